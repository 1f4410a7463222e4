// Coarse levels of the geometric multigrid.
//
// Level l >= 1 operators are stored as compact symmetric stencils.  Neighbour
// directions are numbered nb = (dz+1) + 3(dx+1) + 9(dy+1) in 3-D and (dx+1) + 3(dy+1)
// in 2-D; the centre is nb = 13 / 4 and nb > centre are the "upper" directions.  Since
// A_l is symmetric, only the upper triangle of the centre block and the blocks towards the
// upper neighbours are stored, coefficient-major (one array of n slots per coefficient, so
// one thread per node reads them coalesced):
//   3-D: 6 centre (00 01 02 11 12 22) + 13 x 9 = 123 arrays, 2-D: 3 + 4 x 4 = 19 arrays.
// The block towards a lower neighbour J = I - d is the transpose of J's stored block for +d.
// This replaces the reference's fixed-81/18-nnz CSR (core/_mgm_cuda.py:69-221): same
// values, no index arrays, half the coefficients.
//
// Transfers restate restriction_{2d,3d}_kernel / prolongation_{2d,3d}_kernel
// (core/_templated_cuda.cu:232-475): full weighting 1, 1/2, 1/4, 1/8 by Manhattan
// distance, divided by the coarse node's boundary total (8, 6, 4.5, 3.375 in 3-D;
// 4, 3, 2.25 in 2-D); prolongation divides each parent's value by its total and
// averages over the in-range parents.
//
// Galerkin operators restate get_restricted_{3d,2d}_l0_nnz_based and _l1p_nnz_based
// (core/_mgm_cuda.cu:1-649): A_{l+1} = R A_l R^T with R as above on both sides; level 1
// is formed from E, K0 and the BC mask with constrained fine DOFs contributing the
// identity.  Here level 1 is gathered per (coarse node, neighbour) from the fine
// elements whose coarse cube holds both nodes: an element with lower corner 2m+s
// (per axis) maps its corners onto the coarse cube {m, m+1} with weights
// P_s = [[1,0],[1/2,1/2]] (s=0) or [[1/2,1/2],[0,1]] (s=1), so its contribution is
// E_e * (P_s^T K0 P_s), eight 24x24 tables computed once on the host; elements that
// touch a constrained DOF are projected with their masked K0 directly.
#pragma once
#include "common.cuh"
#include "fine_apply.cuh"

namespace edge {

EDGE_HD double bnd_total3(int nb) { return nb == 3 ? 3.375 : nb == 2 ? 4.5 : nb == 1 ? 6.0 : 8.0; }
EDGE_HD double bnd_total2(int nb) { return nb == 2 ? 2.25 : nb == 1 ? 3.0 : 4.0; }
EDGE_HD double dist_w(int d) { return d == 0 ? 1.0 : d == 1 ? 0.5 : d == 2 ? 0.25 : 0.125; }
EDGE_D int is_bnd(int i, int n) { return (i == 0 || i == n - 1) ? 1 : 0; }
// 1 / bnd_total: the transfers multiply by these instead of dividing (a divide in FP64 is a
// long instruction sequence; the results differ from the division by rounding only)
template <typename T> EDGE_D T inv_bnd_total3(int nb) {
  return nb == 3 ? T(1.0 / 3.375) : nb == 2 ? T(1.0 / 4.5) : nb == 1 ? T(1.0 / 6.0) : T(0.125);
}
template <typename T> EDGE_D T inv_bnd_total2(int nb) {
  return nb == 2 ? T(1.0 / 2.25) : nb == 1 ? T(1.0 / 3.0) : T(0.25);
}
// arithmetic type of a transfer producing TO: FP64 for FP64 vectors, FP32 otherwise
template <typename TO> struct TransferT {
  using type = float;
};
template <> struct TransferT<double> {
  using type = double;
};

// ------------------------------------------------------------------ symmetric stencil access
constexpr int NST3 = 123;
constexpr int NST2 = 19;
EDGE_HD int nst(int dim) { return dim == 3 ? NST3 : NST2; }
EDGE_HD int centre_nb(int dim) { return dim == 3 ? 13 : 4; }
// index of centre coefficient (c, d) in the symmetric 3x3 / 2x2 storage
EDGE_HD int cidx(int dim, int c, int d) {
  if (c > d) { int t = c; c = d; d = t; }
  return dim == 3 ? (c == 0 ? d : (c == 1 ? 2 + d : 5)) : (c == 0 ? d : 2);
}
// array index of coefficient (c, d) of the block towards upper direction nb
EDGE_HD int uidx(int dim, int nb, int c, int d) {
  return dim == 3 ? 6 + (nb - 14) * 9 + c * 3 + d : 3 + (nb - 5) * 4 + c * 2 + d;
}
EDGE_HD void nb_dir(int dim, int nb, int& dx, int& dy, int& dz) {
  if (dim == 3) {
    dz = nb % 3 - 1;
    dx = (nb / 3) % 3 - 1;
    dy = nb / 9 - 1;
  } else {
    dx = nb % 3 - 1;
    dy = nb / 3 - 1;
    dz = 0;
  }
}
EDGE_HD long long nb_off(const Geo& g, int nb) {
  int dx, dy, dz;
  nb_dir(g.dim, nb, dx, dy, dz);
  return g.dim == 3 ? (long long)dy * g.plane + (long long)dx * g.pz + dz : (long long)dy * g.pz + dx;
}
// A[I, I+dir(nb)](c, d) with I at slot s; the caller guarantees I+dir(nb) is in the grid.
template <typename TS>
EDGE_D double st_get(const Geo& g, const TS* __restrict__ S, long long s, int nb, int c, int d) {
  const int cn = centre_nb(g.dim);
  if (nb == cn) return (double)Conv<double>::from(S[(long long)cidx(g.dim, c, d) * g.n + s]);
  if (nb > cn) return (double)Conv<double>::from(S[(long long)uidx(g.dim, nb, c, d) * g.n + s]);
  const long long sj = s + nb_off(g, nb);
  return (double)Conv<double>::from(S[(long long)uidx(g.dim, 2 * cn - nb, d, c) * g.n + sj]);
}

// ------------------------------------------------------------------ stencil apply (levels >= 1)
// One thread per slot (flat grid); padding slots exit.
template <typename T, typename TS, class Epi>
__global__ void __launch_bounds__(128)
k_st3_apply(const Geo g, const T* __restrict__ u, const TS* __restrict__ S, Epi epi, double* part, unsigned* ticket,
            double* dot_dst) {
  EDGE_PDL_ENTRY();
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n = g.n;
  epi.init();
  double dacc = 0.0;
  const int k = (int)(s % g.pz), i = (int)((s / g.pz) % g.nx), j = (int)(s / g.plane);
  if (s < n && k < g.nz) {
    const typename Epi::Pre pe = epi.pre(s);  // epilogue inputs first: their latency overlaps the stencil
    const T u0 = __ldg(u + s), u1 = __ldg(u + n + s), u2 = __ldg(u + 2 * n + s);
    const T c00 = Conv<T>::from(__ldg(S + s)), c01 = Conv<T>::from(__ldg(S + n + s)),
            c02 = Conv<T>::from(__ldg(S + 2 * n + s)), c11 = Conv<T>::from(__ldg(S + 3 * n + s)),
            c12 = Conv<T>::from(__ldg(S + 4 * n + s)), c22 = Conv<T>::from(__ldg(S + 5 * n + s));
    T Au[3];
    Au[0] = c00 * u0 + c01 * u1 + c02 * u2;
    Au[1] = c01 * u0 + c11 * u1 + c12 * u2;
    Au[2] = c02 * u0 + c12 * u1 + c22 * u2;
#pragma unroll
    for (int nb = 14; nb < 27; ++nb) {
      const int dz = nb % 3 - 1, dx = (nb / 3) % 3 - 1, dy = nb / 9 - 1;
      const long long off = (long long)dy * g.plane + (long long)dx * g.pz + dz;
      const TS* Sb = S + (long long)(6 + (nb - 14) * 9) * n;
      if (i + dx >= 0 && i + dx < g.nx && j + dy >= 0 && j + dy < g.ny && k + dz >= 0 && k + dz < g.nz) {
        const long long sn = s + off;  // upper neighbour: block stored here
        const T v0 = __ldg(u + sn), v1 = __ldg(u + n + sn), v2 = __ldg(u + 2 * n + sn);
#pragma unroll
        for (int c = 0; c < 3; ++c)
          Au[c] += Conv<T>::from(__ldg(Sb + (c * 3 + 0) * n + s)) * v0 +
                   Conv<T>::from(__ldg(Sb + (c * 3 + 1) * n + s)) * v1 +
                   Conv<T>::from(__ldg(Sb + (c * 3 + 2) * n + s)) * v2;
      }
      if (i - dx >= 0 && i - dx < g.nx && j - dy >= 0 && j - dy < g.ny && k - dz >= 0 && k - dz < g.nz) {
        const long long sm = s - off;  // lower neighbour: transpose of its block for +d
        const T v0 = __ldg(u + sm), v1 = __ldg(u + n + sm), v2 = __ldg(u + 2 * n + sm);
#pragma unroll
        for (int c = 0; c < 3; ++c)
          Au[c] += Conv<T>::from(__ldg(Sb + (0 * 3 + c) * n + sm)) * v0 +
                   Conv<T>::from(__ldg(Sb + (1 * 3 + c) * n + sm)) * v1 +
                   Conv<T>::from(__ldg(Sb + (2 * 3 + c) * n + sm)) * v2;
      }
    }
    T own[3] = {u0, u1, u2};
    epi.apply(s, own, Au, pe, dacc);
  }
  finish_dot(epi, dacc, part, ticket, dot_dst);
}

// Two consecutive z-slots per thread (s0 even, s1 = s0 + 1; the padded row length is a
// multiple of 4, so both lie in one (x, y) row): the centre blocks, the stored upper blocks,
// the dz = 0 lower blocks and the dz = 0 neighbour values load as pairs (8 bytes for FP32,
// 4 bytes for a BF16 stencil copy).  A warp covers 64 slots of one row,
// so the (x, y) range tests of a direction are warp-uniform branches; the z range test is
// a select on values loaded from inside the array (a z neighbour outside the grid is the
// row's padding or the next row's first slot).  Same sums in the same order per node as
// k_st3_apply.
template <typename T, typename TS, class Epi>
__global__ void __launch_bounds__(128)
k_st3_apply2(const Geo g, const T* __restrict__ u, const TS* __restrict__ S, Epi epi, double* part, unsigned* ticket,
             double* dot_dst) {
  EDGE_PDL_ENTRY();
  using T2 = typename V2<T>::type;
  const long long s0 = 2 * (blockIdx.x * (long long)blockDim.x + threadIdx.x);
  const long long n = g.n;
  epi.init();
  double dacc = 0.0;
  if (s0 < n) {
    const int k0 = (int)(s0 % g.pz), i = (int)((s0 / g.pz) % g.nx), j = (int)(s0 / g.plane);
    const bool ok0 = k0 < g.nz, ok1 = k0 + 1 < g.nz;
    // epilogue inputs of both slots first (s0 + 1 < n: n is even), overlapping the stencil loads
    const typename Epi::Pre pe0 = epi.pre(s0), pe1 = epi.pre(s0 + 1);
    auto ld2 = [&](const T* a, long long s) { return reinterpret_cast<const T2*>(a + s)[0]; };
    auto lds2 = [&](const TS* a, long long s) -> T2 {
      if constexpr (std::is_same<TS, T>::value) {
        return reinterpret_cast<const T2*>(a + s)[0];
      } else if constexpr (std::is_same<TS, __nv_bfloat16>::value) {
        // s is even and the coefficient arrays start on even slots: one 4-byte load
        const __nv_bfloat162 h = __ldg(reinterpret_cast<const __nv_bfloat162*>(a + s));
        T2 r;
        r.x = Conv<T>::from(__low2bfloat16(h));
        r.y = Conv<T>::from(__high2bfloat16(h));
        return r;
      } else {
        T2 r;
        r.x = Conv<T>::from(__ldg(a + s));
        r.y = Conv<T>::from(__ldg(a + s + 1));
        return r;
      }
    };
    T2 uc[3], Au[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) uc[c] = ld2(u + c * n, s0);
    {
      T2 cc[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) cc[q] = lds2(S + q * n, s0);
      // rows of the symmetric centre block: (c00 c01 c02; c01 c11 c12; c02 c12 c22)
      Au[0].x = cc[0].x * uc[0].x + cc[1].x * uc[1].x + cc[2].x * uc[2].x;
      Au[0].y = cc[0].y * uc[0].y + cc[1].y * uc[1].y + cc[2].y * uc[2].y;
      Au[1].x = cc[1].x * uc[0].x + cc[3].x * uc[1].x + cc[4].x * uc[2].x;
      Au[1].y = cc[1].y * uc[0].y + cc[3].y * uc[1].y + cc[4].y * uc[2].y;
      Au[2].x = cc[2].x * uc[0].x + cc[4].x * uc[1].x + cc[5].x * uc[2].x;
      Au[2].y = cc[2].y * uc[0].y + cc[4].y * uc[1].y + cc[5].y * uc[2].y;
    }
#pragma unroll
    for (int nb = 14; nb < 27; ++nb) {
      const int dz = nb % 3 - 1, dx = (nb / 3) % 3 - 1, dy = nb / 9 - 1;
      const long long off = (long long)dy * g.plane + (long long)dx * g.pz + dz;
      const TS* Sb = S + (long long)(6 + (nb - 14) * 9) * n;
      if (i + dx >= 0 && i + dx < g.nx && j + dy >= 0 && j + dy < g.ny) {  // upper neighbour
        const bool z0 = k0 + dz >= 0 && k0 + dz < g.nz, z1 = k0 + 1 + dz >= 0 && k0 + 1 + dz < g.nz;
        const long long sn = s0 + off;
        // dz = +1 at the end of the last row would read one slot past the array: clamp
        // (that value is masked by z1 anyway)
        const long long sn1 = sn + 1 < n ? sn + 1 : n - 1;
        T2 v[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (dz == 0) {
            v[c] = ld2(u + c * n, sn);
          } else {
            v[c].x = __ldg(u + c * n + sn);
            v[c].y = __ldg(u + c * n + sn1);
          }
          v[c].x = z0 ? v[c].x : T(0);
          v[c].y = z1 ? v[c].y : T(0);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const T2 a = lds2(Sb + (c * 3 + 0) * n, s0), b = lds2(Sb + (c * 3 + 1) * n, s0),
                   d = lds2(Sb + (c * 3 + 2) * n, s0);
          Au[c].x += a.x * v[0].x + b.x * v[1].x + d.x * v[2].x;
          Au[c].y += a.y * v[0].y + b.y * v[1].y + d.y * v[2].y;
        }
      }
      if (i - dx >= 0 && i - dx < g.nx && j - dy >= 0 && j - dy < g.ny) {  // lower neighbour
        const bool z0 = k0 - dz >= 0 && k0 - dz < g.nz, z1 = k0 + 1 - dz >= 0 && k0 + 1 - dz < g.nz;
        const long long sm = s0 - off;  // sm >= -1 when the (x, y) test holds: clamp the pair start
        const long long sa = sm < 0 ? 0 : sm;
        T2 v[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (dz == 0) {  // off is even (plane and pz are multiples of 4): sm is an aligned pair start >= 0
            v[c] = ld2(u + c * n, sm);
          } else {
            v[c].x = __ldg(u + c * n + sa);
            v[c].y = __ldg(u + c * n + sm + 1);
          }
          v[c].x = z0 ? v[c].x : T(0);
          v[c].y = z1 ? v[c].y : T(0);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          T2 a, b, d;
          if (dz == 0) {
            a = lds2(Sb + (0 * 3 + c) * n, sm);
            b = lds2(Sb + (1 * 3 + c) * n, sm);
            d = lds2(Sb + (2 * 3 + c) * n, sm);
          } else {
            a.x = Conv<T>::from(__ldg(Sb + (0 * 3 + c) * n + sa));
            a.y = Conv<T>::from(__ldg(Sb + (0 * 3 + c) * n + sm + 1));
            b.x = Conv<T>::from(__ldg(Sb + (1 * 3 + c) * n + sa));
            b.y = Conv<T>::from(__ldg(Sb + (1 * 3 + c) * n + sm + 1));
            d.x = Conv<T>::from(__ldg(Sb + (2 * 3 + c) * n + sa));
            d.y = Conv<T>::from(__ldg(Sb + (2 * 3 + c) * n + sm + 1));
          }
          Au[c].x += a.x * v[0].x + b.x * v[1].x + d.x * v[2].x;
          Au[c].y += a.y * v[0].y + b.y * v[1].y + d.y * v[2].y;
        }
      }
    }
    if (ok0) {
      T own[3] = {uc[0].x, uc[1].x, uc[2].x}, A[3] = {Au[0].x, Au[1].x, Au[2].x};
      epi.apply(s0, own, A, pe0, dacc);
    }
    if (ok1) {
      T own[3] = {uc[0].y, uc[1].y, uc[2].y}, A[3] = {Au[0].y, Au[1].y, Au[2].y};
      epi.apply(s0 + 1, own, A, pe1, dacc);
    }
  }
  finish_dot(epi, dacc, part, ticket, dot_dst);
}

// BF16 pair (low half: the even slot) -> two FP32 values, exactly
EDGE_D float2 bf16x2_to_f2(uint32_t w) { return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u)); }

// Tile-major BF16 pair copy of a 3-D stencil for k_st3_apply2t: word
// (p >> 5) * STT_TILE + q * 32 + (p & 31) holds coefficient array q of the slot pair p (slots
// 2p and 2p + 1, the low half for slot 2p).  The 32 pairs of a warp form one tile, so every
// coefficient load of a thread is the tile base of its pair plus a constant offset (q * 128
// bytes), with no per-load address arithmetic; a warp's loads stay 128-byte coalesced.
constexpr int STT_TILE = NST3 * 32;  // words per tile of 32 pairs
EDGE_HD long long stt_base(long long p) { return (p >> 5) * STT_TILE + (p & 31); }
EDGE_HD long long stt_words(long long n) { return ((n / 2 + 31) / 32) * STT_TILE; }

// FP32 stencil (NST3 arrays of n slots) -> the tile-major BF16 pair copy (n even; padding
// pairs of the last tile are zero).  Same rounding as the linear BF16 copy.
__global__ void k_stencil_tiled_bf16(long long n, const float* __restrict__ S, unsigned* __restrict__ St,
                                     long long nw) {
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < nw; w += (long long)gridDim.x * blockDim.x) {
    const long long tile = w / STT_TILE;
    const int r = (int)(w - tile * STT_TILE), q = r >> 5;
    const long long s = 2 * (tile * 32 + (r & 31));
    unsigned v = 0u;
    if (s < n) {
      const float2 c = reinterpret_cast<const float2*>(S + (long long)q * n + s)[0];
      v = (unsigned)__bfloat16_as_ushort(Conv<__nv_bfloat16>::from(c.x)) |
          ((unsigned)__bfloat16_as_ushort(Conv<__nv_bfloat16>::from(c.y)) << 16);
    }
    St[w] = v;
  }
}

// k_st3_apply2 on the tile-major BF16 copy: two consecutive z-slots per thread, the thread's
// own coefficient pairs at constant offsets from one base, the transposed blocks of a lower
// neighbour from one base per direction (two for dz = +-1, where the neighbour pair straddles
// two stored pairs), and the three products of a block row on the packed FP32 pipe (both
// slots of the pair in one instruction).  Same terms as k_st3_apply2 summed in the same order
// (each block row: a v0, + b v1, + d v2, then added to the sum), with the packed instructions'
// own rounding of each step.
// The x += omega D^-1 (b - A x) sweep is held to 64 registers (8 blocks per SM instead of 7
// at its unbounded 71; 4 bytes of spill).
template <class Epi> struct StTiledMinBlocks {
  static constexpr int value = 1;
};
template <typename T, typename TB, typename TD, typename TX, bool DOT, typename TV>
struct StTiledMinBlocks<EpiJacobiAdd<T, TB, TD, TX, DOT, TV>> {
  static constexpr int value = 8;
};
template <class Epi>
__global__ void __launch_bounds__(128, StTiledMinBlocks<Epi>::value)
k_st3_apply2t(const Geo g, const float* __restrict__ u, const unsigned* __restrict__ St, Epi epi, double* part,
              unsigned* ticket, double* dot_dst) {
  EDGE_PDL_ENTRY();
  using T = float;
  using T2 = float2;
  const long long p = blockIdx.x * 128LL + threadIdx.x;  // slot pair
  const long long s0 = 2 * p;
  const long long n = g.n;
  epi.init();
  double dacc = 0.0;
  if (s0 < n) {
    const int k0 = (int)(s0 % g.pz), i = (int)((s0 / g.pz) % g.nx), j = (int)(s0 / g.plane);
    const bool ok0 = k0 < g.nz, ok1 = k0 + 1 < g.nz;
    const typename Epi::Pre pe0 = epi.pre(s0), pe1 = epi.pre(s0 + 1);
    const unsigned* own = St + stt_base(p);
    auto ld2 = [&](const T* a, long long s) { return reinterpret_cast<const T2*>(a + s)[0]; };
    auto lo = [](unsigned w) { return __uint_as_float(w << 16); };
    auto hi = [](unsigned w) { return __uint_as_float(w & 0xffff0000u); };
    auto row = [](T2 a, T2 b, T2 d, const T2* v) {
      return __ffma2_rn(d, v[2], __ffma2_rn(b, v[1], __fmul2_rn(a, v[0])));
    };
    T2 uc[3], Au[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) uc[c] = ld2(u + c * n, s0);
    {
      T2 cc[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) cc[q] = bf16x2_to_f2(__ldg(own + q * 32));
      Au[0] = row(cc[0], cc[1], cc[2], uc);
      Au[1] = row(cc[1], cc[3], cc[4], uc);
      Au[2] = row(cc[2], cc[4], cc[5], uc);
    }
#pragma unroll
    for (int nb = 14; nb < 27; ++nb) {
      const int dz = nb % 3 - 1, dx = (nb / 3) % 3 - 1, dy = nb / 9 - 1;
      const long long off = (long long)dy * g.plane + (long long)dx * g.pz + dz;
      const int qb = 6 + (nb - 14) * 9;
      if (i + dx >= 0 && i + dx < g.nx && j + dy >= 0 && j + dy < g.ny) {  // upper neighbour
        const bool z0 = k0 + dz >= 0 && k0 + dz < g.nz, z1 = k0 + 1 + dz >= 0 && k0 + 1 + dz < g.nz;
        const long long sn = s0 + off;
        const long long sn1 = sn + 1 < n ? sn + 1 : n - 1;
        T2 v[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (dz == 0) {
            v[c] = ld2(u + c * n, sn);
          } else {
            v[c].x = __ldg(u + c * n + sn);
            v[c].y = __ldg(u + c * n + sn1);
          }
          v[c].x = z0 ? v[c].x : T(0);
          v[c].y = z1 ? v[c].y : T(0);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c)
          Au[c] = __fadd2_rn(Au[c], row(bf16x2_to_f2(__ldg(own + (qb + c * 3 + 0) * 32)),
                                        bf16x2_to_f2(__ldg(own + (qb + c * 3 + 1) * 32)),
                                        bf16x2_to_f2(__ldg(own + (qb + c * 3 + 2) * 32)), v));
      }
      if (i - dx >= 0 && i - dx < g.nx && j - dy >= 0 && j - dy < g.ny) {  // lower neighbour
        const bool z0 = k0 - dz >= 0 && k0 - dz < g.nz, z1 = k0 + 1 - dz >= 0 && k0 + 1 - dz < g.nz;
        const long long sm = s0 - off;  // >= -1 here; odd exactly when dz != 0
        const long long sa = sm < 0 ? 0 : sm;
        T2 v[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (dz == 0) {
            v[c] = ld2(u + c * n, sm);
          } else {
            v[c].x = __ldg(u + c * n + sa);
            v[c].y = __ldg(u + c * n + sm + 1);
          }
          v[c].x = z0 ? v[c].x : T(0);
          v[c].y = z1 ? v[c].y : T(0);
        }
        if (dz == 0) {  // the neighbour pair is the stored pair sm / 2
          const unsigned* lb = St + stt_base(sm >> 1);
#pragma unroll
          for (int c = 0; c < 3; ++c)
            Au[c] = __fadd2_rn(Au[c], row(bf16x2_to_f2(__ldg(lb + (qb + 0 * 3 + c) * 32)),
                                          bf16x2_to_f2(__ldg(lb + (qb + 1 * 3 + c) * 32)),
                                          bf16x2_to_f2(__ldg(lb + (qb + 2 * 3 + c) * 32)), v));
        } else {  // slot sm: high half of pair (sm - 1) / 2; slot sm + 1: low half of pair (sm + 1) / 2
          const long long pa = (sm - 1) >> 1;
          const unsigned* la = St + stt_base(pa < 0 ? 0 : pa);
          const unsigned* lb = St + stt_base((sm + 1) >> 1);
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const unsigned a0 = __ldg(la + (qb + 0 * 3 + c) * 32), a1 = __ldg(lb + (qb + 0 * 3 + c) * 32);
            const unsigned b0 = __ldg(la + (qb + 1 * 3 + c) * 32), b1 = __ldg(lb + (qb + 1 * 3 + c) * 32);
            const unsigned d0 = __ldg(la + (qb + 2 * 3 + c) * 32), d1 = __ldg(lb + (qb + 2 * 3 + c) * 32);
            Au[c] = __fadd2_rn(Au[c], row(make_float2(hi(a0), lo(a1)), make_float2(hi(b0), lo(b1)),
                                          make_float2(hi(d0), lo(d1)), v));
          }
        }
      }
    }
    if (ok0) {
      T o[3] = {uc[0].x, uc[1].x, uc[2].x}, A[3] = {Au[0].x, Au[1].x, Au[2].x};
      epi.apply(s0, o, A, pe0, dacc);
    }
    if (ok1) {
      T o[3] = {uc[0].y, uc[1].y, uc[2].y}, A[3] = {Au[0].y, Au[1].y, Au[2].y};
      epi.apply(s0 + 1, o, A, pe1, dacc);
    }
  }
  finish_dot(epi, dacc, part, ticket, dot_dst);
}

// Latency-oriented variant for small levels, where a sweep is a handful of dependent load
// round trips rather than a bandwidth problem: four lanes per node share the 26 neighbour
// terms (term t = 4m + lane; terms 0..12 are the stored upper blocks, 13..25 the transposed
// blocks of the lower neighbours), every load is unconditional (a neighbour outside the grid
// reads this node's own slot and is replaced by zero), the four partial sums are combined
// by two xor-shuffles (the same fixed order on every lane, so results are reproducible) and
// lane 0 of the group adds the centre block and runs the epilogue.
template <typename T, typename TS, class Epi>
__global__ void __launch_bounds__(128)
k_st3_apply_q(const Geo g, const T* __restrict__ u, const TS* __restrict__ S, Epi epi, double* part, unsigned* ticket,
              double* dot_dst) {
  EDGE_PDL_ENTRY();
  const long long s0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 2;
  const int q = threadIdx.x & 3;
  const long long n = g.n;
  epi.init();
  double dacc = 0.0;
  const long long s = s0 < n ? s0 : n - 1;
  const int k = (int)(s % g.pz), i = (int)((s / g.pz) % g.nx), j = (int)(s / g.plane);
  const bool valid = s0 < n && k < g.nz;
  typename Epi::Pre pe{};
  if (q == 0) pe = epi.pre(s);  // the epilogue lane's inputs first (s is clamped into the array)
  T Au[3] = {T(0), T(0), T(0)};
#pragma unroll
  for (int m = 0; m < 7; ++m) {
    const int t = 4 * m + q;
    const bool lower = t >= 13;
    const int nbi = min(lower ? t - 13 : t, 12);
    const int nb = 14 + nbi;
    const int dz = nb % 3 - 1, dx = (nb / 3) % 3 - 1, dy = nb / 9 - 1;
    const int sg = lower ? -1 : 1;
    const bool in = t < 26 && valid && i + sg * dx >= 0 && i + sg * dx < g.nx && j + sg * dy >= 0 &&
                    j + sg * dy < g.ny && k + sg * dz >= 0 && k + sg * dz < g.nz;
    const long long off = sg * ((long long)dy * g.plane + (long long)dx * g.pz + dz);
    const long long sn = in ? s + off : s;
    const TS* Sb = S + (long long)(6 + nbi * 9) * n + (lower ? sn : s);
    const int cs = lower ? 1 : 3, ds = lower ? 3 : 1;
    T v[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const T a = __ldg(u + c * n + sn);
      v[c] = in ? a : T(0);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c)
      Au[c] += Conv<T>::from(__ldg(Sb + (long long)(c * cs) * n)) * v[0] +
               Conv<T>::from(__ldg(Sb + (long long)(c * cs + ds) * n)) * v[1] +
               Conv<T>::from(__ldg(Sb + (long long)(c * cs + 2 * ds) * n)) * v[2];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    Au[c] += __shfl_xor_sync(0xffffffffu, Au[c], 1);
    Au[c] += __shfl_xor_sync(0xffffffffu, Au[c], 2);
  }
  if (q == 0 && valid) {
    const T u0 = __ldg(u + s), u1 = __ldg(u + n + s), u2 = __ldg(u + 2 * n + s);
    const T c00 = Conv<T>::from(__ldg(S + s)), c01 = Conv<T>::from(__ldg(S + n + s)),
            c02 = Conv<T>::from(__ldg(S + 2 * n + s)), c11 = Conv<T>::from(__ldg(S + 3 * n + s)),
            c12 = Conv<T>::from(__ldg(S + 4 * n + s)), c22 = Conv<T>::from(__ldg(S + 5 * n + s));
    Au[0] += c00 * u0 + c01 * u1 + c02 * u2;
    Au[1] += c01 * u0 + c11 * u1 + c12 * u2;
    Au[2] += c02 * u0 + c12 * u1 + c22 * u2;
    T own[3] = {u0, u1, u2};
    epi.apply(s, own, Au, pe, dacc);
  }
  finish_dot(epi, dacc, part, ticket, dot_dst);
}

template <typename T, typename TS, class Epi>
__global__ void __launch_bounds__(128)
k_st2_apply(const Geo g, const T* __restrict__ u, const TS* __restrict__ S, Epi epi, double* part, unsigned* ticket,
            double* dot_dst) {
  EDGE_PDL_ENTRY();
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n = g.n;
  epi.init();
  double dacc = 0.0;
  const int i = (int)(s % g.pz), j = (int)(s / g.pz);
  if (s < n && i < g.nx) {
    const T u0 = __ldg(u + s), u1 = __ldg(u + n + s);
    const T c00 = Conv<T>::from(__ldg(S + s)), c01 = Conv<T>::from(__ldg(S + n + s)),
            c11 = Conv<T>::from(__ldg(S + 2 * n + s));
    T Au[2];
    Au[0] = c00 * u0 + c01 * u1;
    Au[1] = c01 * u0 + c11 * u1;
#pragma unroll
    for (int nb = 5; nb < 9; ++nb) {
      const int dx = nb % 3 - 1, dy = nb / 3 - 1;
      const long long off = (long long)dy * g.pz + dx;
      const TS* Sb = S + (long long)(3 + (nb - 5) * 4) * n;
      if (i + dx >= 0 && i + dx < g.nx && j + dy >= 0 && j + dy < g.ny) {
        const long long sn = s + off;
        const T v0 = __ldg(u + sn), v1 = __ldg(u + n + sn);
        Au[0] += Conv<T>::from(__ldg(Sb + s)) * v0 + Conv<T>::from(__ldg(Sb + n + s)) * v1;
        Au[1] += Conv<T>::from(__ldg(Sb + 2 * n + s)) * v0 + Conv<T>::from(__ldg(Sb + 3 * n + s)) * v1;
      }
      if (i - dx >= 0 && i - dx < g.nx && j - dy >= 0 && j - dy < g.ny) {
        const long long sm = s - off;
        const T v0 = __ldg(u + sm), v1 = __ldg(u + n + sm);
        Au[0] += Conv<T>::from(__ldg(Sb + sm)) * v0 + Conv<T>::from(__ldg(Sb + 2 * n + sm)) * v1;
        Au[1] += Conv<T>::from(__ldg(Sb + n + sm)) * v0 + Conv<T>::from(__ldg(Sb + 3 * n + sm)) * v1;
      }
    }
    T own[2] = {u0, u1};
    epi(s, 2, own, Au, dacc);
  }
  finish_dot(epi, dacc, part, ticket, dot_dst);
}

// Dinv of a stencil level: 1 / centre diagonal.
template <typename TS, typename TD>
__global__ void k_st_dinv(const Geo g, const TS* __restrict__ S, TD* __restrict__ dinv) {
  EDGE_PDL_ENTRY();
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= g.n) return;
  for (int c = 0; c < g.dof; ++c) {
    const double v = (double)Conv<double>::from(S[(long long)cidx(g.dim, c, c) * g.n + s]);
    dinv[c * g.n + s] = Conv<TD>::from(v != 0.0 ? 1.0 / v : 0.0);
  }
}

// ------------------------------------------------------------------ transfers
template <typename TI, typename TO>
// 3-D restriction: one thread per coarse node; blockIdx.y = plane y, the (z, x) pairs of a
// plane flattened over blockIdx.x (z fastest).  The fine z-neighbours 2K and 2K + 1 are one
// aligned pair load (2K is even and rows are padded to a multiple of 4 slots, so 2K + 1 is
// inside the row; it is masked when it is past the last node), 2K - 1 a scalar load.  The
// weights are summed in the order (x, y, z) of the 27-point loop.
__global__ void k_restrict3(const Geo gf, const Geo gc, const TI* __restrict__ in, TO* __restrict__ out) {
  EDGE_PDL_ENTRY();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int J = blockIdx.y;
  if (t >= gc.nz * gc.nx) return;
  const int K = t % gc.nz, I = t / gc.nz;
  using T = typename TransferT<TO>::type;
  using TI2 = typename V2<TI>::type;
  const int nb = is_bnd(I, gc.nx) + is_bnd(J, gc.ny) + is_bnd(K, gc.nz);
  const bool zm = K >= 1, zp = 2 * K + 1 < gf.nz;
  T v[3] = {0, 0, 0};
#pragma unroll
  for (int di = -1; di <= 1; ++di) {
    const int fi = 2 * I + di;
    if (fi < 0 || fi >= gf.nx) continue;
#pragma unroll
    for (int dj = -1; dj <= 1; ++dj) {
      const int fj = 2 * J + dj;
      if (fj < 0 || fj >= gf.ny) continue;
      const T w0 = (T)dist_w(abs(di) + abs(dj)), w1 = (T)dist_w(abs(di) + abs(dj) + 1);
      const long long sf = gf.slot3(fi, fj, 2 * K);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const TI* a = in + c * gf.n + sf;
        const TI2 pr = __ldg(reinterpret_cast<const TI2*>(a));
        if (zm) v[c] += w1 * Conv<T>::from(__ldg(a - 1));
        v[c] += w0 * Conv<T>::from(pr.x);
        if (zp) v[c] += w1 * Conv<T>::from(pr.y);
      }
    }
  }
  const T iw = inv_bnd_total3<T>(nb);
  const long long sc = gc.slot3(I, J, K);
  for (int c = 0; c < 3; ++c) out[c * gc.n + sc] = Conv<TO>::from(v[c] * iw);
}

// The same restriction fused with the coarse level's first damped-Jacobi sweep from zero
// (k_jacobi0): out = R in and x = (w Dinv) out at every coarse node, w = omega * wscale; the
// padding slots of x are not written (they hold zero from allocation and are never read).
template <typename T>
__global__ void k_restrict3_j0(const Geo gf, const Geo gc, const T* __restrict__ in, T* __restrict__ out,
                               const T* __restrict__ dinv, T* __restrict__ x, const double* omega, double wscale) {
  EDGE_PDL_ENTRY();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int J = blockIdx.y;
  if (t >= gc.nz * gc.nx) return;
  const int K = t % gc.nz, I = t / gc.nz;
  using TT = typename TransferT<T>::type;
  using T2 = typename V2<T>::type;
  const int nb = is_bnd(I, gc.nx) + is_bnd(J, gc.ny) + is_bnd(K, gc.nz);
  const bool zm = K >= 1, zp = 2 * K + 1 < gf.nz;
  TT v[3] = {0, 0, 0};
#pragma unroll
  for (int di = -1; di <= 1; ++di) {
    const int fi = 2 * I + di;
    if (fi < 0 || fi >= gf.nx) continue;
#pragma unroll
    for (int dj = -1; dj <= 1; ++dj) {
      const int fj = 2 * J + dj;
      if (fj < 0 || fj >= gf.ny) continue;
      const TT w0 = (TT)dist_w(abs(di) + abs(dj)), w1 = (TT)dist_w(abs(di) + abs(dj) + 1);
      const long long sf = gf.slot3(fi, fj, 2 * K);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const T* a = in + c * gf.n + sf;
        const T2 pr = __ldg(reinterpret_cast<const T2*>(a));
        if (zm) v[c] += w1 * Conv<TT>::from(__ldg(a - 1));
        v[c] += w0 * Conv<TT>::from(pr.x);
        if (zp) v[c] += w1 * Conv<TT>::from(pr.y);
      }
    }
  }
  const TT iw = inv_bnd_total3<TT>(nb);
  const long long sc = gc.slot3(I, J, K);
  const T wt = Conv<T>::from((*omega) * wscale);
  for (int c = 0; c < 3; ++c) {
    const T bv = Conv<T>::from(v[c] * iw);
    out[c * gc.n + sc] = bv;
    x[c * gc.n + sc] = wt * Conv<T>::from(__ldg(dinv + c * gc.n + sc)) * bv;
  }
}

template <typename TI, typename TO>
__global__ void k_restrict2(const Geo gf, const Geo gc, const TI* __restrict__ in, TO* __restrict__ out) {
  EDGE_PDL_ENTRY();
  const int I = blockIdx.x * blockDim.x + threadIdx.x;
  const int J = blockIdx.y;
  if (I >= gc.nx) return;
  using T = typename TransferT<TO>::type;
  const T iw = inv_bnd_total2<T>(is_bnd(I, gc.nx) + is_bnd(J, gc.ny));
  T v[2] = {0, 0};
  for (int di = -1; di <= 1; ++di) {
    const int fi = 2 * I + di;
    if (fi < 0 || fi >= gf.nx) continue;
    for (int dj = -1; dj <= 1; ++dj) {
      const int fj = 2 * J + dj;
      if (fj < 0 || fj >= gf.ny) continue;
      const T w = (T)dist_w(abs(di) + abs(dj));
      const long long sf = gf.slot2(fi, fj);
      for (int c = 0; c < 2; ++c) v[c] += w * Conv<T>::from(in[c * gf.n + sf]);
    }
  }
  const long long sc = gc.slot2(I, J);
  for (int c = 0; c < 2; ++c) out[c * gc.n + sc] = Conv<TO>::from(v[c] * iw);
}

// 3-D prolongation: one thread per coarse node (ci, cj, ck), which writes its fine children
// (2ci + a, 2cj + b, 2ck + c), a, b, c in {0, 1}.  A child's value is the mean of its coarse
// parents (the corners ci..ci+a x cj..cj+b x ck..ck+c that exist), each scaled by the
// reciprocal of its boundary weight total; the eight corner values are loaded once per thread
// instead of once per child, and the two z-children of a fine row are one aligned pair store.
// Launch: blockIdx.y = coarse plane cj, the coarse (z, x) pairs flattened over blockIdx.x.
template <typename TI, typename TO>
__global__ void k_prolong3(const Geo gf, const Geo gc, const TI* __restrict__ in, TO* __restrict__ out) {
  EDGE_PDL_ENTRY();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int cj = blockIdx.y;
  if (t >= gc.nz * gc.nx) return;
  const int ck = t % gc.nz, ci = t / gc.nz;
  using T = typename TransferT<TO>::type;
  using TO2 = typename V2<TO>::type;
  // upper parents that exist, and odd children that exist
  const bool px = ci + 1 < gc.nx, py = cj + 1 < gc.ny, pz = ck + 1 < gc.nz;
  const bool fx = 2 * ci + 1 < gf.nx, fy = 2 * cj + 1 < gf.ny, fz = 2 * ck + 1 < gf.nz;
  T cv[2][2][2][3];  // weighted corner values, 0 where the corner does not exist
#pragma unroll
  for (int x = 0; x < 2; ++x)
#pragma unroll
    for (int y = 0; y < 2; ++y)
#pragma unroll
      for (int z = 0; z < 2; ++z) {
        const bool ex = (x == 0 || px) && (y == 0 || py) && (z == 0 || pz);
        const long long sc = gc.slot3(ci + x, cj + y, ck + z);
        const T iw = inv_bnd_total3<T>(is_bnd(ci + x, gc.nx) + is_bnd(cj + y, gc.ny) + is_bnd(ck + z, gc.nz));
#pragma unroll
        for (int c = 0; c < 3; ++c) cv[x][y][z][c] = ex ? Conv<T>::from(__ldg(in + c * gc.n + sc)) * iw : T(0);
      }
#pragma unroll
  for (int a = 0; a < 2; ++a) {
    if (a == 1 && !fx) continue;
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      if (b == 1 && !fy) continue;
      // parents per axis: 1, or 2 for an odd child whose upper parent exists; 1/cnt is exact
      const int cxy = (1 + (a == 1 && px)) * (1 + (b == 1 && py));
      const T ic0 = T(1) / T(cxy), ic1 = T(1) / T(cxy * (1 + pz));
      const long long sf = gf.slot3(2 * ci + a, 2 * cj + b, 2 * ck);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        T v0 = 0, v1 = 0;  // the even and the odd z-child
#pragma unroll
        for (int x = 0; x <= a; ++x)
#pragma unroll
          for (int y = 0; y <= b; ++y) {
            v0 += cv[x][y][0][c];
            v1 += cv[x][y][0][c];
            v1 += cv[x][y][1][c];
          }
        TO* o = out + c * gf.n + sf;
        if (fz) {
          TO2 w;
          w.x = Conv<TO>::from(v0 * ic0);
          w.y = Conv<TO>::from(v1 * ic1);
          *reinterpret_cast<TO2*>(o) = w;
        } else {
          o[0] = Conv<TO>::from(v0 * ic0);
        }
      }
    }
  }
}

template <typename TI, typename TO>
__global__ void k_prolong2(const Geo gf, const Geo gc, const TI* __restrict__ in, TO* __restrict__ out) {
  EDGE_PDL_ENTRY();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= gf.nx) return;
  using T = typename TransferT<TO>::type;
  T v[2] = {0, 0};
  int cnt = 0;
  for (int ci = i / 2; ci <= i / 2 + (i & 1); ++ci) {
    if (ci >= gc.nx) continue;
    for (int cj = j / 2; cj <= j / 2 + (j & 1); ++cj) {
      if (cj >= gc.ny) continue;
      const T iw = inv_bnd_total2<T>(is_bnd(ci, gc.nx) + is_bnd(cj, gc.ny));
      const long long sc = gc.slot2(ci, cj);
      for (int c = 0; c < 2; ++c) v[c] += Conv<T>::from(in[c * gc.n + sc]) * iw;
      ++cnt;
    }
  }
  const T ic = cnt ? T(1) / T(cnt) : T(0);
  const long long sf = gf.slot2(i, j);
  for (int c = 0; c < 2; ++c) out[c * gf.n + sf] = Conv<TO>::from(v[c] * ic);
}

// ------------------------------------------------------------------ Galerkin, level 0 -> 1
// Element constraint flags: flag[slot(e)] = 1 if any corner DOF of element e is constrained.
__global__ void k_elem_flags(const Geo g, const uint8_t* __restrict__ mask, uint8_t* __restrict__ flag) {
  EDGE_PDL_ENTRY();
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= g.n) return;
  uint8_t f = 0;
  if (g.dim == 3) {
    const int k = (int)(s % g.pz), i = (int)((s / g.pz) % g.nx), j = (int)(s / g.plane);
    if (k < g.nz - 1 && i < g.nx - 1 && j < g.ny - 1)
      for (int b = 0; b < 8; ++b) f |= mask[g.slot3(i + (b & 1), j + ((b >> 1) & 1), k + ((b >> 2) & 1))];
  } else {
    const int i = (int)(s % g.pz), j = (int)(s / g.pz);
    if (i < g.nx - 1 && j < g.ny - 1)
      for (int b = 0; b < 4; ++b) f |= mask[g.slot2(i + (b & 1), j + ((b >> 1) & 1))];
  }
  flag[s] = f ? 1 : 0;
}

// Store a computed block V (dof x dof, row-major) for centre/upper direction nb.
template <typename TS>
EDGE_D void store_block(const Geo& g, TS* S, long long s, int nb, const double* V, bool valid) {
  const int d = g.dof;
  if (nb == centre_nb(g.dim)) {
    for (int a = 0; a < d; ++a)
      for (int b = a; b < d; ++b) S[(long long)cidx(g.dim, a, b) * g.n + s] = Conv<TS>::from(valid ? V[a * d + b] : 0.0);
  } else {
    for (int a = 0; a < d; ++a)
      for (int b = 0; b < d; ++b) S[(long long)uidx(g.dim, nb, a, b) * g.n + s] = Conv<TS>::from(valid ? V[a * d + b] : 0.0);
  }
}

EDGE_D double pw(int s, int a, int c) {  // 1-D corner weight P_s[a][c]
  return s == 0 ? (a == 0 ? (c == 0 ? 1.0 : 0.0) : 0.5) : (a == 0 ? 0.5 : (c == 1 ? 1.0 : 0.0));
}

// One thread per (coarse node, neighbour nb = blockIdx.y).  Q: 8 parity tables [s][24][24]
// (bit-order corners), K0b: dense element matrix in bit order.
template <typename TE, typename TS>
__global__ void __launch_bounds__(128)
k_galerkin3_l0(const Geo gf, const Geo gc, const TE* __restrict__ E, const uint8_t* __restrict__ mask,
               const uint8_t* __restrict__ eflag, const double* __restrict__ Q, const double* __restrict__ K0b,
               TS* __restrict__ S) {
  EDGE_PDL_ENTRY();
  const long long sc = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int nb = 13 + blockIdx.y;  // centre and upper directions only
  if (sc >= gc.n) return;
  const int Kz = (int)(sc % gc.pz), Ix = (int)((sc / gc.pz) % gc.nx), Jy = (int)(sc / gc.plane);
  const int dz = nb % 3 - 1, dx = (nb / 3) % 3 - 1, dy = nb / 9 - 1;
  double V[9];
  for (int q = 0; q < 9; ++q) V[q] = 0.0;
  const int I[3] = {Ix, Jy, Kz};
  const int Jn[3] = {Ix + dx, Jy + dy, Kz + dz};
  const int ncn[3] = {gc.nx, gc.ny, gc.nz};
  const int nfn[3] = {gf.nx, gf.ny, gf.nz};
  bool valid = Kz < gc.nz;
  for (int d = 0; d < 3; ++d) valid = valid && Jn[d] >= 0 && Jn[d] < ncn[d];
  if (valid) {
    // elements: per axis m in [max(I,J)-1, min(I,J)], parity s in {0,1}
    int mlo[3], mhi[3];
    for (int d = 0; d < 3; ++d) {
      mlo[d] = max(I[d], Jn[d]) - 1;
      mhi[d] = min(I[d], Jn[d]);
    }
    for (int my = mlo[1]; my <= mhi[1]; ++my)
      for (int sy = 0; sy < 2; ++sy) {
        const int ly = 2 * my + sy;
        if (ly < 0 || ly >= nfn[1] - 1) continue;
        for (int mx = mlo[0]; mx <= mhi[0]; ++mx)
          for (int sx = 0; sx < 2; ++sx) {
            const int lx = 2 * mx + sx;
            if (lx < 0 || lx >= nfn[0] - 1) continue;
            for (int mz = mlo[2]; mz <= mhi[2]; ++mz)
              for (int sz = 0; sz < 2; ++sz) {
                const int lz = 2 * mz + sz;
                if (lz < 0 || lz >= nfn[2] - 1) continue;
                const long long se = gf.slot3(lx, ly, lz);
                const double Ee = (double)Conv<double>::from(E[se]);
                const int cI = (I[0] - mx) | ((I[1] - my) << 1) | ((I[2] - mz) << 2);
                const int cJ = (Jn[0] - mx) | ((Jn[1] - my) << 1) | ((Jn[2] - mz) << 2);
                const int par = sx | (sy << 1) | (sz << 2);
                if (!eflag[se]) {
                  const double* Qs = Q + par * 576;
                  for (int c = 0; c < 3; ++c)
                    for (int d = 0; d < 3; ++d) V[c * 3 + d] += Ee * Qs[(cI * 3 + c) * 24 + cJ * 3 + d];
                } else {
                  const int sv[3] = {sx, sy, sz};
                  for (int a = 0; a < 8; ++a) {
                    double wa = 1.0;
                    for (int d = 0; d < 3; ++d) wa *= pw(sv[d], (a >> d) & 1, (cI >> d) & 1);
                    if (wa == 0.0) continue;
                    const uint8_t ma = mask[gf.slot3(lx + (a & 1), ly + ((a >> 1) & 1), lz + ((a >> 2) & 1))];
                    for (int b = 0; b < 8; ++b) {
                      double wb = 1.0;
                      for (int d = 0; d < 3; ++d) wb *= pw(sv[d], (b >> d) & 1, (cJ >> d) & 1);
                      if (wb == 0.0) continue;
                      const uint8_t mb = mask[gf.slot3(lx + (b & 1), ly + ((b >> 1) & 1), lz + ((b >> 2) & 1))];
                      for (int c = 0; c < 3; ++c) {
                        if ((ma >> c) & 1) continue;
                        for (int d = 0; d < 3; ++d) {
                          if ((mb >> d) & 1) continue;
                          V[c * 3 + d] += Ee * wa * wb * K0b[(a * 3 + c) * 24 + b * 3 + d];
                        }
                      }
                    }
                  }
                }
              }
          }
      }
    // identity rows/columns of constrained fine DOFs
    int flo[3], fhi[3];
    for (int d = 0; d < 3; ++d) {
      flo[d] = max(max(2 * I[d], 2 * Jn[d]) - 1, 0);
      fhi[d] = min(min(2 * I[d], 2 * Jn[d]) + 1, nfn[d] - 1);
    }
    for (int fy = flo[1]; fy <= fhi[1]; ++fy)
      for (int fx = flo[0]; fx <= fhi[0]; ++fx)
        for (int fz = flo[2]; fz <= fhi[2]; ++fz) {
          const uint8_t m = mask[gf.slot3(fx, fy, fz)];
          if (!m) continue;
          const int f3[3] = {fx, fy, fz};
          double w = 1.0;
          for (int d = 0; d < 3; ++d) w *= (f3[d] == 2 * I[d] ? 1.0 : 0.5) * (f3[d] == 2 * Jn[d] ? 1.0 : 0.5);
          for (int c = 0; c < 3; ++c)
            if ((m >> c) & 1) V[c * 3 + c] += w;
        }
    const double WI = bnd_total3(is_bnd(I[0], ncn[0]) + is_bnd(I[1], ncn[1]) + is_bnd(I[2], ncn[2]));
    const double WJ = bnd_total3(is_bnd(Jn[0], ncn[0]) + is_bnd(Jn[1], ncn[1]) + is_bnd(Jn[2], ncn[2]));
    for (int q = 0; q < 9; ++q) V[q] = V[q] / WI / WJ;
  }
  store_block(gc, S, sc, nb, V, valid);
}

template <typename TE, typename TS>
__global__ void __launch_bounds__(128)
k_galerkin2_l0(const Geo gf, const Geo gc, const TE* __restrict__ E, const uint8_t* __restrict__ mask,
               const uint8_t* __restrict__ eflag, const double* __restrict__ Q, const double* __restrict__ K0b,
               TS* __restrict__ S) {
  EDGE_PDL_ENTRY();
  const long long sc = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int nb = 4 + blockIdx.y;  // centre and upper directions only
  if (sc >= gc.n) return;
  const int Ix = (int)(sc % gc.pz), Jy = (int)(sc / gc.pz);
  const int dx = nb % 3 - 1, dy = nb / 3 - 1;
  double V[4] = {0, 0, 0, 0};
  const int I[2] = {Ix, Jy};
  const int Jn[2] = {Ix + dx, Jy + dy};
  const int ncn[2] = {gc.nx, gc.ny};
  const int nfn[2] = {gf.nx, gf.ny};
  bool valid = Ix < gc.nx;
  for (int d = 0; d < 2; ++d) valid = valid && Jn[d] >= 0 && Jn[d] < ncn[d];
  if (valid) {
    int mlo[2], mhi[2];
    for (int d = 0; d < 2; ++d) {
      mlo[d] = max(I[d], Jn[d]) - 1;
      mhi[d] = min(I[d], Jn[d]);
    }
    for (int my = mlo[1]; my <= mhi[1]; ++my)
      for (int sy = 0; sy < 2; ++sy) {
        const int ly = 2 * my + sy;
        if (ly < 0 || ly >= nfn[1] - 1) continue;
        for (int mx = mlo[0]; mx <= mhi[0]; ++mx)
          for (int sx = 0; sx < 2; ++sx) {
            const int lx = 2 * mx + sx;
            if (lx < 0 || lx >= nfn[0] - 1) continue;
            const long long se = gf.slot2(lx, ly);
            const double Ee = (double)Conv<double>::from(E[se]);
            const int cI = (I[0] - mx) | ((I[1] - my) << 1);
            const int cJ = (Jn[0] - mx) | ((Jn[1] - my) << 1);
            const int par = sx | (sy << 1);
            if (!eflag[se]) {
              const double* Qs = Q + par * 64;
              for (int c = 0; c < 2; ++c)
                for (int d = 0; d < 2; ++d) V[c * 2 + d] += Ee * Qs[(cI * 2 + c) * 8 + cJ * 2 + d];
            } else {
              const int sv[2] = {sx, sy};
              for (int a = 0; a < 4; ++a) {
                double wa = 1.0;
                for (int d = 0; d < 2; ++d) wa *= pw(sv[d], (a >> d) & 1, (cI >> d) & 1);
                if (wa == 0.0) continue;
                const uint8_t ma = mask[gf.slot2(lx + (a & 1), ly + ((a >> 1) & 1))];
                for (int b = 0; b < 4; ++b) {
                  double wb = 1.0;
                  for (int d = 0; d < 2; ++d) wb *= pw(sv[d], (b >> d) & 1, (cJ >> d) & 1);
                  if (wb == 0.0) continue;
                  const uint8_t mb = mask[gf.slot2(lx + (b & 1), ly + ((b >> 1) & 1))];
                  for (int c = 0; c < 2; ++c) {
                    if ((ma >> c) & 1) continue;
                    for (int d = 0; d < 2; ++d) {
                      if ((mb >> d) & 1) continue;
                      V[c * 2 + d] += Ee * wa * wb * K0b[(a * 2 + c) * 8 + b * 2 + d];
                    }
                  }
                }
              }
            }
          }
      }
    int flo[2], fhi[2];
    for (int d = 0; d < 2; ++d) {
      flo[d] = max(max(2 * I[d], 2 * Jn[d]) - 1, 0);
      fhi[d] = min(min(2 * I[d], 2 * Jn[d]) + 1, nfn[d] - 1);
    }
    for (int fy = flo[1]; fy <= fhi[1]; ++fy)
      for (int fx = flo[0]; fx <= fhi[0]; ++fx) {
        const uint8_t m = mask[gf.slot2(fx, fy)];
        if (!m) continue;
        const int f2[2] = {fx, fy};
        double w = 1.0;
        for (int d = 0; d < 2; ++d) w *= (f2[d] == 2 * I[d] ? 1.0 : 0.5) * (f2[d] == 2 * Jn[d] ? 1.0 : 0.5);
        for (int c = 0; c < 2; ++c)
          if ((m >> c) & 1) V[c * 2 + c] += w;
      }
    const double WI = bnd_total2(is_bnd(I[0], ncn[0]) + is_bnd(I[1], ncn[1]));
    const double WJ = bnd_total2(is_bnd(Jn[0], ncn[0]) + is_bnd(Jn[1], ncn[1]));
    for (int q = 0; q < 4; ++q) V[q] = V[q] / WI / WJ;
  }
  store_block(gc, S, sc, nb, V, valid);
}

// ------------------------------------------------------------------ Galerkin, stencil level l -> l+1
template <typename TS>
__global__ void __launch_bounds__(128)
k_galerkin3_st(const Geo gf, const Geo gc, const TS* __restrict__ Sf, TS* __restrict__ Sc) {
  EDGE_PDL_ENTRY();
  const long long sc = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int nb = 13 + blockIdx.y;
  if (sc >= gc.n) return;
  const int Kz = (int)(sc % gc.pz), Ix = (int)((sc / gc.pz) % gc.nx), Jy = (int)(sc / gc.plane);
  const int dz = nb % 3 - 1, dx = (nb / 3) % 3 - 1, dy = nb / 9 - 1;
  const int I[3] = {Ix, Jy, Kz};
  const int Jn[3] = {Ix + dx, Jy + dy, Kz + dz};
  const int ncn[3] = {gc.nx, gc.ny, gc.nz};
  const int nfn[3] = {gf.nx, gf.ny, gf.nz};
  bool valid = Kz < gc.nz;
  for (int d = 0; d < 3; ++d) valid = valid && Jn[d] >= 0 && Jn[d] < ncn[d];
  double V[9];
  for (int q = 0; q < 9; ++q) V[q] = 0.0;
  if (valid) {
    for (int iy = max(2 * I[1] - 1, 0); iy <= min(2 * I[1] + 1, nfn[1] - 1); ++iy)
      for (int ix = max(2 * I[0] - 1, 0); ix <= min(2 * I[0] + 1, nfn[0] - 1); ++ix)
        for (int iz = max(2 * I[2] - 1, 0); iz <= min(2 * I[2] + 1, nfn[2] - 1); ++iz) {
          const double wi = dist_w(abs(ix - 2 * I[0]) + abs(iy - 2 * I[1]) + abs(iz - 2 * I[2]));
          const long long si = gf.slot3(ix, iy, iz);
          const int fi[3] = {ix, iy, iz};
          int jlo[3], jhi[3];
          for (int d = 0; d < 3; ++d) {
            jlo[d] = max(max(2 * Jn[d] - 1, fi[d] - 1), 0);
            jhi[d] = min(min(2 * Jn[d] + 1, fi[d] + 1), nfn[d] - 1);
          }
          for (int jy = jlo[1]; jy <= jhi[1]; ++jy)
            for (int jx = jlo[0]; jx <= jhi[0]; ++jx)
              for (int jz = jlo[2]; jz <= jhi[2]; ++jz) {
                const double wj = dist_w(abs(jx - 2 * Jn[0]) + abs(jy - 2 * Jn[1]) + abs(jz - 2 * Jn[2]));
                const int fnb = (jz - iz + 1) + 3 * (jx - ix + 1) + 9 * (jy - iy + 1);
                const double w = wi * wj;
                for (int c = 0; c < 3; ++c)
                  for (int d = 0; d < 3; ++d) V[c * 3 + d] += w * st_get(gf, Sf, si, fnb, c, d);
              }
        }
    const double WI = bnd_total3(is_bnd(I[0], ncn[0]) + is_bnd(I[1], ncn[1]) + is_bnd(I[2], ncn[2]));
    const double WJ = bnd_total3(is_bnd(Jn[0], ncn[0]) + is_bnd(Jn[1], ncn[1]) + is_bnd(Jn[2], ncn[2]));
    for (int q = 0; q < 9; ++q) V[q] = V[q] / WI / WJ;
  }
  store_block(gc, Sc, sc, nb, V, valid);
}

// One axis of the Galerkin product: So = R_a Si R_a^T, with R_a the 1-D full weighting along
// axis a (weight 1 at distance 0 and 1/2 at distance 1, divided by the coarse node's total: 2
// inside, 1.5 at either end) and the identity along the other two axes.  The restriction of
// k_galerkin3_st is the product of the three: its weights are 1/2^d by Manhattan distance d and
// its totals 8 (3/4)^k with k = the node's end axes, the per-axis factors multiplied out, and
// its fine index sets are per-axis intervals.  So three passes (x, y, z; FP64 intermediates)
// give the same R A R^T with at most 7 fine (i, j) pairs per output (node, direction) instead
// of up to 27 x 8; only the summation order differs.  One thread per (output slot, centre or
// upper direction nb = 13 + blockIdx.y); padding slots store zeros.  AX: 0 = x, 1 = y, 2 = z.
template <int AX, typename TI, typename TO>
__global__ void __launch_bounds__(128)
k_galerkin3_axis(const Geo gi, const Geo go, const TI* __restrict__ Si, TO* __restrict__ So) {
  EDGE_PDL_ENTRY();
  const long long so = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int nb = 13 + blockIdx.y;
  if (so >= go.n) return;
  const int Kz = (int)(so % go.pz), Ix = (int)((so / go.pz) % go.nx), Jy = (int)(so / go.plane);
  const int dz = nb % 3 - 1, dx = (nb / 3) % 3 - 1, dy = nb / 9 - 1;
  const int I[3] = {Ix, Jy, Kz};
  const int Jn[3] = {Ix + dx, Jy + dy, Kz + dz};
  const int no[3] = {go.nx, go.ny, go.nz};
  const int na = AX == 0 ? gi.nx : AX == 1 ? gi.ny : gi.nz;  // input nodes along the axis
  bool valid = Kz < go.nz;
  for (int d = 0; d < 3; ++d) valid = valid && Jn[d] >= 0 && Jn[d] < no[d];
  double V[9];
  for (int q = 0; q < 9; ++q) V[q] = 0.0;
  if (valid) {
    const int Ia = I[AX], Ja = Jn[AX];
    for (int ia = max(2 * Ia - 1, 0); ia <= min(2 * Ia + 1, na - 1); ++ia) {
      const double wi = ia == 2 * Ia ? 1.0 : 0.5;
      int fi[3] = {I[0], I[1], I[2]};
      fi[AX] = ia;
      const long long si = gi.slot3(fi[0], fi[1], fi[2]);
      const int jlo = max(max(2 * Ja - 1, ia - 1), 0), jhi = min(min(2 * Ja + 1, ia + 1), na - 1);
      for (int ja = jlo; ja <= jhi; ++ja) {
        const double w = wi * (ja == 2 * Ja ? 1.0 : 0.5);
        int e[3] = {dx, dy, dz};  // the other axes keep the output direction
        e[AX] = ja - ia;
        const int fnb = (e[2] + 1) + 3 * (e[0] + 1) + 9 * (e[1] + 1);
        for (int c = 0; c < 3; ++c)
          for (int d = 0; d < 3; ++d) V[c * 3 + d] += w * st_get(gi, Si, si, fnb, c, d);
      }
    }
    const double WI = is_bnd(Ia, no[AX]) ? 1.5 : 2.0, WJ = is_bnd(Ja, no[AX]) ? 1.5 : 2.0;
    for (int q = 0; q < 9; ++q) V[q] = V[q] / WI / WJ;
  }
  store_block(go, So, so, nb, V, valid);
}

template <typename TS>
__global__ void __launch_bounds__(128)
k_galerkin2_st(const Geo gf, const Geo gc, const TS* __restrict__ Sf, TS* __restrict__ Sc) {
  EDGE_PDL_ENTRY();
  const long long sc = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int nb = 4 + blockIdx.y;
  if (sc >= gc.n) return;
  const int Ix = (int)(sc % gc.pz), Jy = (int)(sc / gc.pz);
  const int dx = nb % 3 - 1, dy = nb / 3 - 1;
  const int I[2] = {Ix, Jy};
  const int Jn[2] = {Ix + dx, Jy + dy};
  const int ncn[2] = {gc.nx, gc.ny};
  const int nfn[2] = {gf.nx, gf.ny};
  bool valid = Ix < gc.nx;
  for (int d = 0; d < 2; ++d) valid = valid && Jn[d] >= 0 && Jn[d] < ncn[d];
  double V[4] = {0, 0, 0, 0};
  if (valid) {
    for (int iy = max(2 * I[1] - 1, 0); iy <= min(2 * I[1] + 1, nfn[1] - 1); ++iy)
      for (int ix = max(2 * I[0] - 1, 0); ix <= min(2 * I[0] + 1, nfn[0] - 1); ++ix) {
        const double wi = dist_w(abs(ix - 2 * I[0]) + abs(iy - 2 * I[1]));
        const long long si = gf.slot2(ix, iy);
        const int fi[2] = {ix, iy};
        int jlo[2], jhi[2];
        for (int d = 0; d < 2; ++d) {
          jlo[d] = max(max(2 * Jn[d] - 1, fi[d] - 1), 0);
          jhi[d] = min(min(2 * Jn[d] + 1, fi[d] + 1), nfn[d] - 1);
        }
        for (int jy = jlo[1]; jy <= jhi[1]; ++jy)
          for (int jx = jlo[0]; jx <= jhi[0]; ++jx) {
            const double wj = dist_w(abs(jx - 2 * Jn[0]) + abs(jy - 2 * Jn[1]));
            const int fnb = (jx - ix + 1) + 3 * (jy - iy + 1);
            const double w = wi * wj;
            for (int c = 0; c < 2; ++c)
              for (int d = 0; d < 2; ++d) V[c * 2 + d] += w * st_get(gf, Sf, si, fnb, c, d);
          }
      }
    const double WI = bnd_total2(is_bnd(I[0], ncn[0]) + is_bnd(I[1], ncn[1]));
    const double WJ = bnd_total2(is_bnd(Jn[0], ncn[0]) + is_bnd(Jn[1], ncn[1]));
    for (int q = 0; q < 4; ++q) V[q] = V[q] / WI / WJ;
  }
  store_block(gc, Sc, sc, nb, V, valid);
}

// ------------------------------------------------------------------ coarsest level: dense FP64
// Dense row-major A (nd x nd) from a stencil level; dense DOF index = node_index*dof + c with
// node_index the unpadded lexicographic index (j, i, k) of the reference.
template <typename TS>
__global__ void k_st_to_dense(const Geo g, const TS* __restrict__ S, double* __restrict__ A, int nd) {
  EDGE_PDL_ENTRY();
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= g.n) return;
  const int dof = g.dof;
  int i, j, k = 0;
  if (g.dim == 3) {
    k = (int)(s % g.pz);
    i = (int)((s / g.pz) % g.nx);
    j = (int)(s / g.plane);
    if (k >= g.nz) return;
  } else {
    i = (int)(s % g.pz);
    j = (int)(s / g.pz);
    if (i >= g.nx) return;
  }
  auto didx = [&](int ii, int jj, int kk) -> long long {
    return g.dim == 3 ? ((long long)jj * g.nx * g.nz + (long long)ii * g.nz + kk) : ((long long)jj * g.nx + ii);
  };
  const long long row_node = didx(i, j, k);
  const int nnb = g.dim == 3 ? 27 : 9;
  for (int nb = 0; nb < nnb; ++nb) {
    int di, dj, dk;
    nb_dir(g.dim, nb, di, dj, dk);
    if (g.dim == 3 && (k + dk < 0 || k + dk >= g.nz)) continue;
    if (i + di < 0 || i + di >= g.nx || j + dj < 0 || j + dj >= g.ny) continue;
    const long long col_node = didx(i + di, j + dj, k + dk);
    for (int c = 0; c < dof; ++c)
      for (int d = 0; d < dof; ++d) A[(row_node * dof + c) * nd + col_node * dof + d] = st_get(g, S, s, nb, c, d);
  }
}

// Blocked right-looking Cholesky (lower) of an SPD nd x nd row-major FP64 matrix, tile
// size CB.  Per tile column K: k_chol_diag factors the diagonal tile in shared memory,
// k_chol_panel solves the tiles below it, k_chol_update applies the symmetric rank-CB
// update to the trailing lower triangle.  `status` is set to 1 on a non-positive pivot
// (the pivot is then replaced by 1 so the factor stays finite).
constexpr int CB = 32;

__global__ void __launch_bounds__(CB * CB / 4) k_chol_diag(double* A, int nd, int K, int* status) {
  EDGE_PDL_ENTRY();
  __shared__ double t[CB][CB + 1];
  const int k0 = K * CB;
  const int m = min(CB, nd - k0);
  for (int q = threadIdx.x; q < CB * CB; q += blockDim.x) {
    const int r = q / CB, c = q % CB;
    t[r][c] = (r < m && c < m) ? A[(long long)(k0 + r) * nd + k0 + c] : (r == c ? 1.0 : 0.0);
  }
  __syncthreads();
  for (int k = 0; k < CB; ++k) {
    if (threadIdx.x == 0) {
      double d = t[k][k];
      if (!(d > 0.0)) {
        if (k < m) *status = 1;
        d = 1.0;
      }
      t[k][k] = sqrt(d);
    }
    __syncthreads();
    const double p = t[k][k];
    for (int i = k + 1 + threadIdx.x; i < CB; i += blockDim.x) t[i][k] /= p;
    __syncthreads();
    for (int q = threadIdx.x; q < CB * CB; q += blockDim.x) {
      const int i = q / CB, j = q % CB;
      if (i > k && j > k && j <= i) t[i][j] -= t[i][k] * t[j][k];
    }
    __syncthreads();
  }
  for (int q = threadIdx.x; q < CB * CB; q += blockDim.x) {
    const int r = q / CB, c = q % CB;
    if (r < m && c < m) A[(long long)(k0 + r) * nd + k0 + c] = (c <= r) ? t[r][c] : 0.0;
  }
}

// Tile row I = K+1+blockIdx.x: X L_KK^T = A_IK  (X overwrites A_IK)
__global__ void __launch_bounds__(CB * CB / 4) k_chol_panel(double* A, int nd, int K) {
  EDGE_PDL_ENTRY();
  __shared__ double L[CB][CB + 1];
  __shared__ double X[CB][CB + 1];
  const int k0 = K * CB;
  const int i0 = (K + 1 + blockIdx.x) * CB;
  const int mk = min(CB, nd - k0), mi = min(CB, nd - i0);
  for (int q = threadIdx.x; q < CB * CB; q += blockDim.x) {
    const int r = q / CB, c = q % CB;
    L[r][c] = (r < mk && c < mk) ? A[(long long)(k0 + r) * nd + k0 + c] : (r == c ? 1.0 : 0.0);
    X[r][c] = (r < mi && c < mk) ? A[(long long)(i0 + r) * nd + k0 + c] : 0.0;
  }
  __syncthreads();
  // row r of X: x_r[c] = (a_r[c] - sum_{j<c} x_r[j] L[c][j]) / L[c][c], one thread per row
  for (int r = threadIdx.x; r < CB; r += blockDim.x) {
    for (int c = 0; c < CB; ++c) {
      double v = X[r][c];
      for (int j = 0; j < c; ++j) v -= X[r][j] * L[c][j];
      X[r][c] = v / L[c][c];
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < CB * CB; q += blockDim.x) {
    const int r = q / CB, c = q % CB;
    if (r < mi && c < mk) A[(long long)(i0 + r) * nd + k0 + c] = X[r][c];
  }
}

// Trailing update A_IJ -= A_IK A_JK^T for K < J <= I; blockIdx.x enumerates (I, J).
__global__ void __launch_bounds__(CB * CB / 4) k_chol_update(double* A, int nd, int K, int nt) {
  EDGE_PDL_ENTRY();
  __shared__ double P[CB][CB + 1];
  __shared__ double Q[CB][CB + 1];
  const int m = nt - K - 1;  // tiles below K
  int q = blockIdx.x, I = 0;
  while (q >= I + 1) {  // triangular enumeration: (I, J) with 0 <= J <= I < m
    q -= I + 1;
    ++I;
  }
  const int J = q;
  if (I >= m) return;
  const int k0 = K * CB, i0 = (K + 1 + I) * CB, j0 = (K + 1 + J) * CB;
  const int mk = min(CB, nd - k0), mi = min(CB, nd - i0), mj = min(CB, nd - j0);
  for (int t = threadIdx.x; t < CB * CB; t += blockDim.x) {
    const int r = t / CB, c = t % CB;
    P[r][c] = (r < mi && c < mk) ? A[(long long)(i0 + r) * nd + k0 + c] : 0.0;
    Q[r][c] = (r < mj && c < mk) ? A[(long long)(j0 + r) * nd + k0 + c] : 0.0;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < CB * CB; t += blockDim.x) {
    const int r = t / CB, c = t % CB;
    if (r >= mi || c >= mj) continue;
    if (I == J && c > r) continue;
    double v = 0.0;
#pragma unroll 8
    for (int k = 0; k < CB; ++k) v += P[r][k] * Q[c][k];
    A[(long long)(i0 + r) * nd + j0 + c] -= v;
  }
}

// U = L^T (row-major), so that both substitutions below read rows.
__global__ void k_transpose_lower(const double* __restrict__ L, double* __restrict__ U, int nd) {
  EDGE_PDL_ENTRY();
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= (long long)nd * nd) return;
  const int r = (int)(q / nd), c = (int)(q % nd);
  U[(long long)c * nd + r] = (c <= r) ? L[q] : 0.0;
}

// Column `col` of A^-1 = L^-T L^-1 e_col, one block per column.  U = L^T row-major.
__global__ void __launch_bounds__(256) k_chol_inverse(const double* __restrict__ L, const double* __restrict__ U,
                                                      double* __restrict__ X, int nd) {
  EDGE_PDL_ENTRY();
  extern __shared__ double y[];
  const int col = blockIdx.x;
  const int t = threadIdx.x, nt = blockDim.x;
  for (int i = t; i < nd; i += nt) y[i] = (i == col) ? 1.0 : 0.0;
  __syncthreads();
  for (int k = col; k < nd; ++k) {  // L y = e_col (y_i = 0 for i < col)
    const double yk = y[k] / U[(long long)k * nd + k];
    __syncthreads();
    if (t == 0) y[k] = yk;
    for (int i = k + 1 + t; i < nd; i += nt) y[i] -= U[(long long)k * nd + i] * yk;
    __syncthreads();
  }
  for (int k = nd - 1; k >= 0; --k) {  // L^T x = y
    const double xk = y[k] / L[(long long)k * nd + k];
    __syncthreads();
    if (t == 0) y[k] = xk;
    for (int i = t; i < k; i += nt) y[i] -= L[(long long)k * nd + i] * xk;
    __syncthreads();
  }
  for (int i = t; i < nd; i += nt) X[(long long)i * nd + col] = y[i];
}

// x = Ainv b on the coarsest level: b and x in slot layout (types TB/TX), Ainv dense FP64.
// Each block first gathers b into shared memory in dense order (nd * sizeof(TB) bytes of
// dynamic shared memory), then one warp per dense row.
template <typename TB, typename TX>
__global__ void k_coarse_solve(const Geo g, const double* __restrict__ Ainv, int nd, const TB* __restrict__ b,
                               TX* __restrict__ x) {
  EDGE_PDL_ENTRY();
  extern __shared__ __align__(16) unsigned char coarse_smem[];
  TB* bs = reinterpret_cast<TB*>(coarse_smem);
  const int dof = g.dof;
  auto slot_of = [&](int dn) -> long long {
    const int node = dn / dof;
    if (g.dim == 3) {
      const int k = node % g.nz, i = (node / g.nz) % g.nx, j = node / (g.nz * g.nx);
      return g.slot3(i, j, k);
    }
    const int i = node % g.nx, j = node / g.nx;
    return g.slot2(i, j);
  };
  for (int c = threadIdx.x; c < nd; c += blockDim.x) bs[c] = b[(c % dof) * g.n + slot_of(c)];
  __syncthreads();
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= nd) return;
  const double* __restrict__ a = Ainv + (long long)row * nd;
  double acc = 0.0;
  for (int c = lane; c < nd; c += 32) acc += a[c] * (double)Conv<double>::from(bs[c]);
  acc = warp_sum(acc);
  if (lane == 0) x[(row % dof) * g.n + slot_of(row)] = Conv<TX>::from(acc);
}

}  // namespace edge
