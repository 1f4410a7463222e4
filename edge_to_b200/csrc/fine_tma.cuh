// TMA-pipelined fine-level operator (3-D), sm_100a.
//
// Same tiling and arithmetic as k_fine3_wht (fine_apply.cuh): a block of 32 lanes (z) x
// BX warps (x) marches along y, one hex8 element per thread and layer, Walsh-Hadamard
// element operator, node sums by warp shuffle (z) and shared memory (x).  What changes is
// how the node planes arrive: an NS-deep ring of shared-memory stages is filled by
// cp.async.bulk.tensor (TMA) copies issued by one thread, each stage completing on its own
// mbarrier.  A stage holds, for node plane p, the tile of u (3 components), of the BC
// mask and of the element row E[p]; the copy for plane p+NS is issued as soon as every
// thread has finished with plane p, so NS-1 planes are always in flight while the block
// computes.  TMA zero-fills everything outside the arrays (negative / past-the-end
// coordinates), and every padding slot of the slot layout holds zero, so the inner loop
// has no bounds checks on loads.
//
// TMA rules respected here: every box starts at an innermost coordinate that is a
// multiple of 16 elements (z tiles start at z0-1 rounded down to 16; the 48-wide box
// covers the 33 nodes the tile needs from any of the 16 possible offsets), the mask uses
// its own array with a 16-byte row pitch, all strides are multiples of 16 bytes, and
// shared-memory destinations are 128-byte aligned.  No multicast.
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

template <typename T, int BX>
struct TmaTile {
  static constexpr int NR = BX + 1;                                   // node rows (x) per stage
  static constexpr int U_BYTES = 3 * NR * TMA_ZB * (int)sizeof(T);
  static constexpr int M_BYTES = NR * TMA_ZB;
  static constexpr int E_BYTES = BX * TMA_ZB * (int)sizeof(T);
  static constexpr int up(int b) { return (b + 127) & ~127; }
  static constexpr int U_OFF = 0;
  static constexpr int M_OFF = up(U_BYTES);
  static constexpr int E_OFF = M_OFF + up(M_BYTES);
  static constexpr int STAGE = E_OFF + up(E_BYTES);
  static constexpr int TX_BYTES = U_BYTES + M_BYTES + E_BYTES;
};

template <typename T, int BX, int NS>
constexpr int tma_smem_bytes() {
  return NS * TmaTile<T, BX>::STAGE + 2 * 2 * 3 * BX * 33 * (int)sizeof(T) + 128 + 16 * NS;
}

template <typename T, class Epi, int BX, int NS>
__global__ void __launch_bounds__(32 * BX)
k_fine3_tma(const Geo g, const __grid_constant__ CUtensorMap mapU, const __grid_constant__ CUtensorMap mapM,
            const __grid_constant__ CUtensorMap mapE, const T* __restrict__ u, const uint8_t* __restrict__ mask,
            const KHat3<T> K, const int ly, Epi epi, double* part, unsigned* ticket, double* dot_dst, int* err) {
  using Tile = TmaTile<T, BX>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  typedef T GArr[2][2][3][BX][33];
  GArr& sG = *reinterpret_cast<GArr*>(smem + NS * Tile::STAGE);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + NS * Tile::STAGE + 2 * 2 * 3 * BX * 33 * sizeof(T));

  const int lane = threadIdx.x, wx = threadIdx.y, tid = lane + 32 * wx;
  const int z0 = blockIdx.x * 31, x0 = blockIdx.y * (BX - 1);
  const int y0 = blockIdx.z * ly;
  const int y1 = min(y0 + ly, g.ny);
  const int ez = z0 - 1 + lane, ex = x0 - 1 + wx;
  const int zs = ((z0 - 1) >= 0) ? ((z0 - 1) & ~15) : -16;  // box start, multiple of 16
  const int zo = (z0 - 1) - zs;                              // offset of node z0-1 in the box
  const long long n = g.n;
  const int p0 = y0 - 1;          // first plane
  const int np = y1 - p0 + 1;     // planes p0 .. y1
  epi.init();
  bool ok = true;

  if (tid == 0) {
    for (int s = 0; s < NS; ++s) mbar_init(&bar[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](int k) {  // plane p0 + k into stage k % NS
    const int s = k % NS;
    unsigned char* st = smem + s * Tile::STAGE;
    const int p = p0 + k;
    mbar_expect_tx(&bar[s], Tile::TX_BYTES);
    tma_load_4d(st + Tile::U_OFF, &mapU, zs, x0 - 1, p, 0, &bar[s]);
    tma_load_3d(st + Tile::M_OFF, &mapM, zs, x0 - 1, p, &bar[s]);
    tma_load_3d(st + Tile::E_OFF, &mapE, zs, x0 - 1, p, &bar[s]);
  };
  if (tid == 0)
    for (int k = 0; k < NS && k < np; ++k) issue(k);

  auto U = [&](int k, int c, int row, int z) -> T {
    const T* su = reinterpret_cast<const T*>(smem + (k % NS) * Tile::STAGE + Tile::U_OFF);
    return su[(c * Tile::NR + row) * TMA_ZB + z];
  };
  auto M = [&](int k, int row, int z) -> uint8_t {
    const uint8_t* sm = smem + (k % NS) * Tile::STAGE + Tile::M_OFF;
    return sm[row * TMA_ZB + z];
  };
  auto Eel = [&](int k) -> T {
    const T* se = reinterpret_cast<const T*>(smem + (k % NS) * Tile::STAGE + Tile::E_OFF);
    return se[wx * TMA_ZB + zo + lane];
  };

  // lower plane p0 into registers (masked); ml = BC bits of this thread's own node
  T ul[2][2][3];
  uint8_t ml = 0;
  if (ok) ok = mbar_wait(&bar[0], 0);
#pragma unroll
  for (int dx = 0; dx < 2; ++dx)
#pragma unroll
    for (int dz = 0; dz < 2; ++dz) {
      const uint8_t m = M(0, wx + dx, zo + lane + dz);
      if (dx == 0 && dz == 0) ml = m;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const T v = U(0, c, wx + dx, zo + lane + dz);
        ul[dx][dz][c] = ((m >> c) & 1) ? T(0) : v;
      }
    }
  T acc[3] = {T(0), T(0), T(0)};
  double dacc = 0.0;
  for (int k = 0; k + 1 < np; ++k) {  // layer ey = p0 + k uses planes k (E) and k+1 (upper u)
    const int ey = p0 + k;
    if (ok) ok = mbar_wait(&bar[(k + 1) % NS], ((k + 1) / NS) & 1);
    T uu[2][2][3];
    uint8_t mu = 0;
#pragma unroll
    for (int dx = 0; dx < 2; ++dx)
#pragma unroll
      for (int dz = 0; dz < 2; ++dz) {
        const uint8_t m = M(k + 1, wx + dx, zo + lane + dz);
        if (dx == 0 && dz == 0) mu = m;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const T v = U(k + 1, c, wx + dx, zo + lane + dz);
          uu[dx][dz][c] = ((m >> c) & 1) ? T(0) : v;
        }
      }
    const T Ee = Eel(k);
    T u8[8][3], f[8][3];
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const int bx = b & 1, by = (b >> 1) & 1, bz = (b >> 2) & 1;
#pragma unroll
      for (int c = 0; c < 3; ++c) u8[b][c] = by ? uu[bx][bz][c] : ul[bx][bz][c];
    }
    elem3_apply(K, Ee, u8, f);
    T gz[2][2][3];
#pragma unroll
    for (int ax = 0; ax < 2; ++ax)
#pragma unroll
      for (int ay = 0; ay < 2; ++ay)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const T up = __shfl_up_sync(0xffffffffu, f[ax | (ay << 1) | 4][c], 1);
          gz[ax][ay][c] = f[ax | (ay << 1)][c] + up;
        }
    const int gb = k & 1;
#pragma unroll
    for (int ay = 0; ay < 2; ++ay)
#pragma unroll
      for (int c = 0; c < 3; ++c) sG[gb][ay][c][wx][lane] = gz[1][ay][c];
    __syncthreads();
    // every thread is done with stage k (its E row, and its u as last layer's upper plane)
    if (tid == 0 && k + NS < np) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(k + NS);
    }
    T tot[2][3];
#pragma unroll
    for (int ay = 0; ay < 2; ++ay)
#pragma unroll
      for (int c = 0; c < 3; ++c) tot[ay][c] = gz[0][ay][c] + (wx > 0 ? sG[gb][ay][c][wx - 1][lane] : T(0));
    if (ey >= y0 && lane >= 1 && wx >= 1 && ez < g.nz && ex < g.nx) {
      const long long s = g.slot3(ex, ey, ez);
      const uint8_t m = ml;
      T own[3], Au[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        own[c] = ul[0][0][c];
        Au[c] = acc[c] + tot[0][c];
        if ((m >> c) & 1) {
          own[c] = __ldg(u + c * n + s);
          Au[c] = own[c];
        }
      }
      epi(s, 3, own, Au, dacc);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[c] = tot[1][c];
#pragma unroll
    for (int dx = 0; dx < 2; ++dx)
#pragma unroll
      for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int c = 0; c < 3; ++c) ul[dx][dz][c] = uu[dx][dz][c];
    ml = mu;
  }
  if (!ok) atomicOr(err, 1);
  finish_dot(epi, dacc, part, ticket, dot_dst);
}

}  // namespace edge
