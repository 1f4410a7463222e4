// TMA-pipelined fine-level operator (3-D), sm_100a.
//
// A block is BX warps; each warp is 16 lanes along z times 2 element columns along x, so
// a block covers 2*BX element columns and marches along y, one hex8 element per thread and
// layer.  Per layer a thread (1) x-z transforms the four corners of the new (upper) node
// plane, reusing the transform of the lower plane from the previous layer, (2) applies the
// y stage, E and the sparse transformed element matrix, (3) inverse-transforms along y,
// adding the part that belongs to the lower plane to what the previous layer carried for
// it (all in the transform domain) and carrying the upper part forward, (4) inverse x-z
// transforms the completed plane's part and sums the four in-plane element contributions
// of each node: z by shuffle within the 16-lane half, x by shuffle between halves and
// through shared memory between warps.  Node planes arrive through an NS-deep ring of
// shared-memory stages filled by cp.async.bulk.tensor (TMA) copies issued by one thread,
// each completing on its own mbarrier; a stage holds, for plane p, the tile of u (3
// components), of the element constraint flags and of the element row E[p].  The copy for
// plane p+NS is issued as soon as every thread is done with plane p, so NS-1 planes are in
// flight while the block computes.  Constrained DOFs are masked only in warps where a flag
// is set, from the per-node mask in global memory.  TMA zero-fills everything outside the arrays (negative / past-the-end
// coordinates), and every padding slot of the slot layout holds zero, so the inner loop
// has no bounds checks on loads.
//
// TMA rules respected here: every box starts at an innermost coordinate that is a
// multiple of 16 elements (z tiles start at z0-1 rounded down to 16; the 48-wide box
// covers the 17 nodes the tile needs from any of the 16 possible offsets, and its 48-word
// rows put the two half-warps on disjoint shared-memory banks), the flags use their own
// array with a 16-byte row pitch, all strides are multiples of 16 bytes, and shared-memory
// destinations are 128-byte aligned.  No multicast.
//
// Every mbarrier wait is bounded (2^28 SM cycles, ~0.15 s); after one expiry a thread
// stops waiting altogether and records the error in *err, so the kernel always terminates
// quickly and the host reports a failure instead of the GPU hanging.
#pragma once
#include <cuda.h>

#include "common.cuh"
#include "element_op.cuh"
#include "fine_apply.cuh"

namespace edge {

constexpr int TMA_ZB = 48;  // box width along z (elements)

EDGE_D uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

EDGE_D void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
EDGE_D void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Bounded wait for the phase with the given parity to complete.  Returns false on timeout.
EDGE_D bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
    if (clock64() - t0 > (1LL << 28)) return false;
  }
}
EDGE_D void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          smem_u32(dst)),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}
EDGE_D void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(
          smem_u32(dst)),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}

// Tile of the v3 kernel: warps of 16 z-lanes x 2 x-columns, BX warps -> 2*BX element
// columns per block; z tiles of 15 output nodes, x tiles of 2*BX-1 output columns.
template <typename T, int BX>
struct TmaTile {
  static constexpr int NC = 2 * BX;                      // element columns per block
  static constexpr int NR = NC + 1;                      // node rows (x) per stage
  static constexpr int U_BYTES = 3 * NR * TMA_ZB * (int)sizeof(T);
  static constexpr int F_BYTES = NC * TMA_ZB;            // element constraint flags
  static constexpr int E_BYTES = NC * TMA_ZB * (int)sizeof(T);
  static constexpr int up(int b) { return (b + 127) & ~127; }
  static constexpr int U_OFF = 0;
  static constexpr int F_OFF = up(U_BYTES);
  static constexpr int E_OFF = F_OFF + up(F_BYTES);
  static constexpr int STAGE = E_OFF + up(E_BYTES);
  static constexpr int TX_BYTES = U_BYTES + F_BYTES + E_BYTES;
  static constexpr int X_BYTES = 2 * BX * 16 * 3 * (int)sizeof(T);  // warp-boundary exchange, 2 buffers
};

template <typename T, int BX, int NS>
constexpr int tma_smem_bytes() {
  return NS * TmaTile<T, BX>::STAGE + TmaTile<T, BX>::X_BYTES + 128 + 16 * NS;
}

// x-z Walsh-Hadamard transform of the four corners (bx, bz) of one plane, per component:
// in t[bx][bz][c] -> out t[hx][hz][c].
template <typename T> EDGE_D void wht_xz(T t[2][2][3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int bx = 0; bx < 2; ++bx) {
      const T a = t[bx][0][c], b = t[bx][1][c];
      t[bx][0][c] = a + b;
      t[bx][1][c] = a - b;
    }
#pragma unroll
    for (int hz = 0; hz < 2; ++hz) {
      const T a = t[0][hz][c], b = t[1][hz][c];
      t[0][hz][c] = a + b;
      t[1][hz][c] = a - b;
    }
  }
}

// Sparse transformed element operator: v = E * Khat u on the 24 transform coefficients
// (h = hx | hy<<1 | hz<<2), both indexed [h][c].
template <typename T> EDGE_D void khat_apply(const KHat3<T>& K, T E, const T uh[8][3], T vh[8][3]) {
  T ue[8][3];
#pragma unroll
  for (int h = 1; h < 8; ++h)
#pragma unroll
    for (int c = 0; c < 3; ++c) ue[h][c] = uh[h][c] * E;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    vh[0][c] = T(0);
#pragma unroll
    for (int h = 1; h < 8; ++h) {
      T acc = K.dg[c][h] * ue[h][c];
#pragma unroll
      for (int d = 0; d < 3; ++d)
        if (d != c && (((h >> c) & 1) != ((h >> d) & 1))) acc += K.of[c][d][h] * ue[h ^ (1 << c) ^ (1 << d)][d];
      vh[h][c] = acc;
    }
  }
}

template <typename T, class Epi, int BX, int NS>
__global__ void __launch_bounds__(32 * BX)
k_fine3_tma(const Geo g, const __grid_constant__ CUtensorMap mapU, const __grid_constant__ CUtensorMap mapF,
            const __grid_constant__ CUtensorMap mapE, const T* __restrict__ u, const uint8_t* __restrict__ mask,
            const KHat3<T> K, const int ly, Epi epi, double* part, unsigned* ticket, double* dot_dst, int* err) {
  EDGE_PDL_ENTRY();
  using Tile = TmaTile<T, BX>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  typedef T XArr[2][BX][16][3];
  XArr& sX = *reinterpret_cast<XArr*>(smem + NS * Tile::STAGE);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + NS * Tile::STAGE + Tile::X_BYTES);

  const int lane = threadIdx.x & 31, w = threadIdx.y, tid = threadIdx.x + 32 * w;
  const int zl = lane & 15, xh = lane >> 4;
  const int cx = 2 * w + xh;                               // element column in the block
  const int z0 = blockIdx.x * 15, x0 = blockIdx.y * (2 * BX - 1);
  const int y0 = blockIdx.z * ly;
  const int y1 = min(y0 + ly, g.ny);
  const int ez = z0 - 1 + zl, ex = x0 - 1 + cx;
  const int zs = ((z0 - 1) >= 0) ? ((z0 - 1) & ~15) : -16;
  const int zo = (z0 - 1) - zs;
  const long long n = g.n;
  const int p0 = y0 - 1;
  const int np = y1 - p0 + 1;
  const bool writer = (zl >= 1) && (cx >= 1) && (ez < g.nz) && (ex < g.nx);
  epi.init();
  bool ok = true;

  if (tid == 0) {
    for (int s = 0; s < NS; ++s) mbar_init(&bar[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](int k) {
    const int s = k % NS;
    unsigned char* st = smem + s * Tile::STAGE;
    const int p = p0 + k;
    mbar_expect_tx(&bar[s], Tile::TX_BYTES);
    tma_load_4d(st + Tile::U_OFF, &mapU, zs, x0 - 1, p, 0, &bar[s]);
    tma_load_3d(st + Tile::F_OFF, &mapF, zs, x0 - 1, p, &bar[s]);
    tma_load_3d(st + Tile::E_OFF, &mapE, zs, x0 - 1, p, &bar[s]);
  };
  if (tid == 0)
    for (int k = 0; k < NS && k < np; ++k) issue(k);

  // per-thread offsets into a stage
  const int uoff = cx * TMA_ZB + zo + zl;          // corner (0,0) of this thread, component 0
  constexpr int UC = Tile::NR * TMA_ZB;           // component stride
  const int eoff = cx * TMA_ZB + zo + zl;

  // load the four corners (cx+dx, z+dz) of the plane in stage k, masking constrained DOFs
  // when the element row's flag says some corner is constrained
  auto load_plane = [&](int k, int p, uint8_t fl, T t[2][2][3]) {
    const T* su = reinterpret_cast<const T*>(smem + (k % NS) * Tile::STAGE + Tile::U_OFF) + uoff;
#pragma unroll
    for (int dx = 0; dx < 2; ++dx)
#pragma unroll
      for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int c = 0; c < 3; ++c) t[dx][dz][c] = su[c * UC + dx * TMA_ZB + dz];
    if (__any_sync(0xffffffffu, fl != 0)) {
      if (fl) {
#pragma unroll
        for (int dx = 0; dx < 2; ++dx)
#pragma unroll
          for (int dz = 0; dz < 2; ++dz) {
            const int ii = ex + dx, kk = ez + dz;
            if (ii >= 0 && ii < g.nx && kk >= 0 && kk < g.nz && p >= 0 && p < g.ny) {
              const uint8_t m = __ldg(mask + g.slot3(ii, p, kk));
#pragma unroll
              for (int c = 0; c < 3; ++c)
                if ((m >> c) & 1) t[dx][dz][c] = T(0);
            }
          }
      }
    }
  };
  auto flag_of = [&](int k) -> uint8_t {
    return (smem + (k % NS) * Tile::STAGE + Tile::F_OFF)[eoff];
  };

  T lo[2][2][3];   // x-z transform of the lower plane
  T car[2][2][3];  // transform-domain contributions carried to the next plane
  T own_lo[3];     // this thread's node on the lower plane (masked values)
  if (ok) ok = mbar_wait(&bar[0], 0);
  load_plane(0, p0, flag_of(0), lo);
#pragma unroll
  for (int c = 0; c < 3; ++c) own_lo[c] = lo[0][0][c];
  wht_xz(lo);
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c) car[a][b][c] = T(0);
  double dacc = 0.0;
  const long long s_base = g.slot3(max(ex, 0), 0, max(ez, 0));  // used only by writers

  for (int k = 0; k + 1 < np; ++k) {
    const int ey = p0 + k;
    // epilogue inputs of this layer's output node, loaded before the element math so
    // their latency overlaps it
    typename Epi::Pre pre;
    const bool wr = (ey >= y0) && writer;
    if (wr) pre = epi.pre(s_base + (long long)ey * g.plane);
    if (ok) ok = mbar_wait(&bar[(k + 1) % NS], ((k + 1) / NS) & 1);
    const uint8_t fl = flag_of(k);   // element row ey: covers this layer's 8 corners
    const T Ee = reinterpret_cast<const T*>(smem + (k % NS) * Tile::STAGE + Tile::E_OFF)[eoff];
    T hi[2][2][3];
    // the new plane is also the lower face of element row ey+1, which reuses these values:
    // mask by both rows' flags (row ey may be the ghost row below the grid, flagged 0)
    load_plane(k + 1, ey + 1, fl | flag_of(k + 1), hi);
    T own_hi[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) own_hi[c] = hi[0][0][c];
    wht_xz(hi);
    // y stage -> 8 transform coefficients per component
    T uh[8][3];
#pragma unroll
    for (int hx = 0; hx < 2; ++hx)
#pragma unroll
      for (int hz = 0; hz < 2; ++hz)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          uh[hx | (hz << 2)][c] = lo[hx][hz][c] + hi[hx][hz][c];
          uh[hx | 2 | (hz << 2)][c] = lo[hx][hz][c] - hi[hx][hz][c];
        }
    T vh[8][3];
    khat_apply(K, Ee, uh, vh);
    // inverse y stage: by = 0 part completes this plane (with the carried part), by = 1 is carried
    T cur[2][2][3];
#pragma unroll
    for (int hx = 0; hx < 2; ++hx)
#pragma unroll
      for (int hz = 0; hz < 2; ++hz)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const T a = vh[hx | (hz << 2)][c], b = vh[hx | 2 | (hz << 2)][c];
          cur[hx][hz][c] = car[hx][hz][c] + (a + b);
          car[hx][hz][c] = a - b;
        }
    wht_xz(cur);  // now cur[ax][az][c]: contribution of this element column to plane ey
    // z-combine: node ez gets az=0 of own column and az=1 of column ez-1 (lane-1 in this half)
    T gx[2][3];
#pragma unroll
    for (int ax = 0; ax < 2; ++ax)
#pragma unroll
      for (int c = 0; c < 3; ++c) gx[ax][c] = cur[ax][0][c] + __shfl_up_sync(0xffffffffu, cur[ax][1][c], 1, 16);
    // x-combine: column cx gets ax=0 of itself and ax=1 of column cx-1
    T fromL[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) fromL[c] = __shfl_up_sync(0xffffffffu, gx[1][c], 16);  // lanes 16..31
    const int xb = k & 1;
    if (xh == 1)
#pragma unroll
      for (int c = 0; c < 3; ++c) sX[xb][w][zl][c] = gx[1][c];
    __syncthreads();
    if (tid == 0 && k + NS < np) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(k + NS);
    }
    if (xh == 0) {
#pragma unroll
      for (int c = 0; c < 3; ++c) fromL[c] = (w > 0) ? sX[xb][w - 1][zl][c] : T(0);
    }
    if (wr) {
      // own node = corner (0,0) of element row ey; its flag fl says whether it may be constrained
      const long long s_out = s_base + (long long)ey * g.plane;
      T own[3], Au[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        Au[c] = gx[0][c] + fromL[c];
        own[c] = own_lo[c];
      }
      if (fl) {
        const uint8_t m = __ldg(mask + s_out);
#pragma unroll
        for (int c = 0; c < 3; ++c)
          if ((m >> c) & 1) {
            own[c] = __ldg(u + c * n + s_out);
            Au[c] = own[c];
          }
      }
      epi.apply(s_out, own, Au, pre, dacc);
    }
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) lo[a][b][c] = hi[a][b][c];
#pragma unroll
    for (int c = 0; c < 3; ++c) own_lo[c] = own_hi[c];
  }
  if (!ok) atomicOr(err, 1);
  finish_dot(epi, dacc, part, ticket, dot_dst);
}

}  // namespace edge
