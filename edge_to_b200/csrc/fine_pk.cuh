// Packed-pair fine-level operator (3-D, FP32), sm_100a.
//
// Same algorithm as k_fine3_tma (transform-domain element operator, y-marching blocks,
// TMA-staged node planes, carry of the upper-face part in registers), but every thread
// owns TWO neighbouring element columns (x = c, c+1) and keeps their values side by side
// in float2 registers, so the whole element operator runs on the packed FP32 pipe
// (add/sub/mul/fma .f32x2: one instruction for both elements).  The two elements share
// their middle node row, which the thread completes by itself (one scalar add per
// component); only the row towards the left neighbour pair crosses lanes (a shuffle
// between half-warps, shared memory between warps).
//
// Tile: a warp is 16 z-lanes x 2 pairs, a block BX warps = 4*BX element columns, which
// produce 4*BX-1 node rows (the first row is the halo of the block to the left); z tiles
// of 15 nodes as in k_fine3_tma.  Stage contents for plane p: u (3 components) over
// 4*BX+1 node rows x 24 z-words, E over 4*BX element columns x 24 z-words, and the element
// constraint flags over 4*BX columns x 48 bytes.
//
// TMA rules: the u and E boxes start at z0-1 rounded down to a multiple of 4 words (16
// bytes for FP32), the byte-wide flag box at z0-1 rounded down to 16; box rows are 96 and
// 48 bytes; strides are multiples of 16 bytes; stage buffers are 128-byte aligned; no
// multicast.  Every mbarrier wait is bounded as in k_fine3_tma.
//
// Shared-memory banks: the two pairs of a warp read node rows two apart, 48 words, so
// their 16-lane halves fall on disjoint bank halves.
#pragma once
#include "fine_tma.cuh"

namespace edge {

constexpr int PK_ZB = 24;  // u / E box width along z (FP32 words)
constexpr int PK_FB = 48;  // flag box width (bytes)

struct P2 {
  float2 v;
};
EDGE_D P2 operator+(P2 a, P2 b) { return {__fadd2_rn(a.v, b.v)}; }
EDGE_D P2 operator-(P2 a, P2 b) {
  unsigned long long x, y, d;
  memcpy(&x, &a.v, 8);
  memcpy(&y, &b.v, 8);
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(x), "l"(y));
  P2 r;
  memcpy(&r.v, &d, 8);
  return r;
}
EDGE_D P2 operator*(P2 a, P2 b) { return {__fmul2_rn(a.v, b.v)}; }
EDGE_D P2 pfma(P2 a, P2 b, P2 c) { return {__ffma2_rn(a.v, b.v, c.v)}; }
EDGE_D P2 pk(float a, float b) { return {make_float2(a, b)}; }

// Transformed element operator with both coefficients of a pair equal (host-duplicated).
struct KHat3P {
  P2 dg[3][8];
  P2 of[3][3][8];
};

template <int BX>
struct PkTile {
  static constexpr int NC = 4 * BX;  // element columns per block
  static constexpr int NR = NC + 1;  // node rows per stage
  static constexpr int U_BYTES = 3 * NR * PK_ZB * 4;
  static constexpr int F_BYTES = NC * PK_FB;
  static constexpr int E_BYTES = NC * PK_ZB * 4;
  static constexpr int up(int b) { return (b + 127) & ~127; }
  static constexpr int U_OFF = 0;
  static constexpr int F_OFF = up(U_BYTES);
  static constexpr int E_OFF = F_OFF + up(F_BYTES);
  static constexpr int STAGE = E_OFF + up(E_BYTES);
  static constexpr int TX_BYTES = U_BYTES + F_BYTES + E_BYTES;
  static constexpr int X_BYTES = 2 * BX * 16 * 3 * 4;  // [2][BX][16][3] floats
};

template <int BX, int NS>
constexpr int pk_smem_bytes() {
  return NS * PkTile<BX>::STAGE + PkTile<BX>::X_BYTES + 128 + 16 * NS;
}

// v = E * Khat u on the packed transform coefficients (h = hx | hy<<1 | hz<<2).
EDGE_D void khat_apply_pk(const KHat3P& K, P2 E, const P2 uh[8][3], P2 vh[8][3]) {
  P2 ue[8][3];
#pragma unroll
  for (int h = 1; h < 8; ++h)
#pragma unroll
    for (int c = 0; c < 3; ++c) ue[h][c] = uh[h][c] * E;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    vh[0][c] = pk(0.f, 0.f);
#pragma unroll
    for (int h = 1; h < 8; ++h) {
      P2 acc = K.dg[c][h] * ue[h][c];
#pragma unroll
      for (int d = 0; d < 3; ++d)
        if (d != c && (((h >> c) & 1) != ((h >> d) & 1))) acc = pfma(K.of[c][d][h], ue[h ^ (1 << c) ^ (1 << d)][d], acc);
      vh[h][c] = acc;
    }
  }
}

template <class Epi, int BX, int NS, int MINB>
__global__ void __launch_bounds__(32 * BX, MINB)
k_fine3_pk(const Geo g, const __grid_constant__ CUtensorMap mapU, const __grid_constant__ CUtensorMap mapF,
           const __grid_constant__ CUtensorMap mapE, const float* __restrict__ u, const uint8_t* __restrict__ mask,
           const KHat3P K, const int ly, Epi epi, double* part, unsigned* ticket, double* dot_dst, int* err) {
  EDGE_PDL_ENTRY();
  using Tile = PkTile<BX>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  typedef float XArr[2][BX][16][3];
  XArr& sX = *reinterpret_cast<XArr*>(smem + NS * Tile::STAGE);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + NS * Tile::STAGE + Tile::X_BYTES);

  const int lane = threadIdx.x & 31, w = threadIdx.y, tid = threadIdx.x + 32 * w;
  const int zl = lane & 15, xh = lane >> 4;
  const int c0 = 2 * (2 * w + xh);                       // first element column of the pair
  const int z0 = blockIdx.x * 15, x0 = blockIdx.y * (4 * BX - 1);
  const int y0 = blockIdx.z * ly;
  const int y1 = min(y0 + ly, g.ny);
  const int ez = z0 - 1 + zl, exa = x0 - 1 + c0;
  const int zs4 = (z0 >= 1) ? ((z0 - 1) & ~3) : -4;
  const int zo4 = (z0 - 1) - zs4;
  const int zs16 = (z0 >= 1) ? ((z0 - 1) & ~15) : -16;
  const int zo16 = (z0 - 1) - zs16;
  const long long n = g.n;
  const int p0 = y0 - 1;
  const int np = y1 - p0 + 1;
  const bool zok = (zl >= 1) && (ez < g.nz);
  const bool writerA = zok && (c0 >= 1) && (exa < g.nx);
  const bool writerB = zok && (exa + 1 < g.nx);
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
    tma_load_4d(st + Tile::U_OFF, &mapU, zs4, x0 - 1, p, 0, &bar[s]);
    tma_load_3d(st + Tile::F_OFF, &mapF, zs16, x0 - 1, p, &bar[s]);
    tma_load_3d(st + Tile::E_OFF, &mapE, zs4, x0 - 1, p, &bar[s]);
  };
  if (tid == 0)
    for (int k = 0; k < NS && k < np; ++k) issue(k);

  constexpr int UC = Tile::NR * PK_ZB;  // component stride in a stage (words)
  const int uoff = c0 * PK_ZB + zo4 + zl;
  const int foff = c0 * PK_FB + zo16 + zl;

  // The 3 node rows x 2 z of plane `p` (stage k), masked on constrained DOFs when `fl` says
  // some corner of the pair may be constrained; returns the packed corners and the
  // thread's two own nodes (rows c0, c0+1 at z = ez).
  auto load_plane = [&](int k, int p, uint8_t fl, P2 t[2][2][3], float ownA[3], float ownB[3]) {
    const float* su = reinterpret_cast<const float*>(smem + (k % NS) * Tile::STAGE + Tile::U_OFF) + uoff;
    float s[3][2][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int c = 0; c < 3; ++c) s[r][dz][c] = su[c * UC + r * PK_ZB + dz];
    if (__any_sync(0xffffffffu, fl != 0)) {
      if (fl) {
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int dz = 0; dz < 2; ++dz) {
            const int ii = exa + r, kk = ez + dz;
            if (ii >= 0 && ii < g.nx && kk >= 0 && kk < g.nz && p >= 0 && p < g.ny) {
              const uint8_t m = __ldg(mask + g.slot3(ii, p, kk));
#pragma unroll
              for (int c = 0; c < 3; ++c)
                if ((m >> c) & 1) s[r][dz][c] = 0.f;
            }
          }
      }
    }
#pragma unroll
    for (int dx = 0; dx < 2; ++dx)
#pragma unroll
      for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int c = 0; c < 3; ++c) t[dx][dz][c] = pk(s[dx][dz][c], s[dx + 1][dz][c]);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      ownA[c] = s[0][0][c];
      ownB[c] = s[1][0][c];
    }
  };
  auto flags_of = [&](int k, uint8_t& fa, uint8_t& fb) {
    const uint8_t* sf = smem + (k % NS) * Tile::STAGE + Tile::F_OFF + foff;
    fa = sf[0];
    fb = sf[PK_FB];
  };

  P2 lo[2][2][3];   // x-z transform of the lower plane
  P2 car[2][2][3];  // transform-domain contributions carried to the next plane
  float ownA_lo[3], ownB_lo[3];
  if (ok) ok = mbar_wait(&bar[0], 0);
  {
    uint8_t fa, fb;
    flags_of(0, fa, fb);
    load_plane(0, p0, fa | fb, lo, ownA_lo, ownB_lo);
  }
  wht_xz(lo);
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c) car[a][b][c] = pk(0.f, 0.f);
  double dacc = 0.0;
  // output slots in plane 0 (used only by writers; exa + 1 >= 0 always, exa may be -1)
  const long long sA_base = g.slot3(max(exa, 0), 0, max(ez, 0));
  const long long sB_base = g.slot3(exa + 1, 0, max(ez, 0));

  for (int k = 0; k + 1 < np; ++k) {
    const int ey = p0 + k;
    const long long sA = sA_base + (long long)ey * g.plane;
    const long long sB = sB_base + (long long)ey * g.plane;
    // epilogue inputs of this layer's two output nodes, loaded before the element math so
    // their latency overlaps it
    const bool wrA = (ey >= y0) && writerA, wrB = (ey >= y0) && writerB;
    typename Epi::Pre preA, preB;
    if (wrA) preA = epi.pre(sA);
    if (wrB) preB = epi.pre(sB);
    if (ok) ok = mbar_wait(&bar[(k + 1) % NS], ((k + 1) / NS) & 1);
    uint8_t fa, fb, fa1, fb1;
    flags_of(k, fa, fb);       // element row ey
    flags_of(k + 1, fa1, fb1); // element row ey + 1 (shares the new plane)
    const float* sE = reinterpret_cast<const float*>(smem + (k % NS) * Tile::STAGE + Tile::E_OFF) + uoff;
    const P2 Ee = pk(sE[0], sE[PK_ZB]);
    P2 hi[2][2][3];
    float ownA_hi[3], ownB_hi[3];
    load_plane(k + 1, ey + 1, fa | fb | fa1 | fb1, hi, ownA_hi, ownB_hi);
    wht_xz(hi);
    P2 uh[8][3];
#pragma unroll
    for (int hx = 0; hx < 2; ++hx)
#pragma unroll
      for (int hz = 0; hz < 2; ++hz)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          uh[hx | (hz << 2)][c] = lo[hx][hz][c] + hi[hx][hz][c];
          uh[hx | 2 | (hz << 2)][c] = lo[hx][hz][c] - hi[hx][hz][c];
        }
    P2 vh[8][3];
    khat_apply_pk(K, Ee, uh, vh);
    P2 cur[2][2][3];
#pragma unroll
    for (int hx = 0; hx < 2; ++hx)
#pragma unroll
      for (int hz = 0; hz < 2; ++hz)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const P2 a = vh[hx | (hz << 2)][c], b = vh[hx | 2 | (hz << 2)][c];
          cur[hx][hz][c] = car[hx][hz][c] + (a + b);
          car[hx][hz][c] = a - b;
        }
    wht_xz(cur);  // cur[ax][az][c]: contributions of the pair's two elements to plane ey
    // z-combine: node ez gets az=0 of its own element and az=1 of element ez-1 (lane-1)
    P2 gx[2][3];
#pragma unroll
    for (int ax = 0; ax < 2; ++ax)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float2 up = cur[ax][1][c].v;
        const P2 sh = pk(__shfl_up_sync(0xffffffffu, up.x, 1, 16), __shfl_up_sync(0xffffffffu, up.y, 1, 16));
        gx[ax][c] = cur[ax][0][c] + sh;
      }
    // x-combine: row c0+1 = ax=1 of element a + ax=0 of element b (in-thread);
    // row c0 = ax=0 of element a + ax=1 of the left pair's element b.
    float AuA[3], AuB[3], fromL[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      AuB[c] = gx[1][c].v.x + gx[0][c].v.y;
      fromL[c] = __shfl_up_sync(0xffffffffu, gx[1][c].v.y, 16);  // lanes 16..31
    }
    const int xb = k & 1;
    if (xh == 1)
#pragma unroll
      for (int c = 0; c < 3; ++c) sX[xb][w][zl][c] = gx[1][c].v.y;
    __syncthreads();
    if (tid == 0 && k + NS < np) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(k + NS);
    }
    if (xh == 0) {
#pragma unroll
      for (int c = 0; c < 3; ++c) fromL[c] = (w > 0) ? sX[xb][w - 1][zl][c] : 0.f;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) AuA[c] = gx[0][c].v.x + fromL[c];
    {
      if (wrA) {
        float own[3], Au[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          own[c] = ownA_lo[c];
          Au[c] = AuA[c];
        }
        if (fa) {
          const uint8_t m = __ldg(mask + sA);
#pragma unroll
          for (int c = 0; c < 3; ++c)
            if ((m >> c) & 1) {
              own[c] = __ldg(u + c * n + sA);
              Au[c] = own[c];
            }
        }
        epi.apply(sA, own, Au, preA, dacc);
      }
      if (wrB) {
        float own[3], Au[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          own[c] = ownB_lo[c];
          Au[c] = AuB[c];
        }
        if (fb) {
          const uint8_t m = __ldg(mask + sB);
#pragma unroll
          for (int c = 0; c < 3; ++c)
            if ((m >> c) & 1) {
              own[c] = __ldg(u + c * n + sB);
              Au[c] = own[c];
            }
        }
        epi.apply(sB, own, Au, preB, dacc);
      }
    }
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) lo[a][b][c] = hi[a][b][c];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      ownA_lo[c] = ownA_hi[c];
      ownB_lo[c] = ownB_hi[c];
    }
  }
  if (!ok) atomicOr(err, 1);
  finish_dot(epi, dacc, part, ticket, dot_dst);
}

}  // namespace edge
