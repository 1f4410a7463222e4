// Fine-level (level 0) matrix-free operator K(E) with boundary conditions, fused with
// the epilogues the solver needs (plain product, product + dot, residual, damped
// Jacobi sweep, last post-smoothing sweep with the correction add).
//
// Semantics follow mat_vec_node_basis_parallel_wcon (core/_ops.py:330-368,
// core/_templated_cuda.cu:782-834): constrained DOFs contribute nothing as columns and
// their rows are the identity, so (A u)_c = u_c on a constrained DOF.
//
// Two implementations:
//  * k_fine3_wht / k_fine2_wht: element-centric tiles.  A block is 32 lanes along the
//    fastest axis (z in 3-D, x in 2-D) times BX warps along x (3-D) and marches along y.
//    Each thread computes one element per y-layer with the Walsh-Hadamard element
//    operator (element_op.cuh), adds the four in-plane contributions of every node
//    with a warp shuffle (z) and shared memory (x), and carries the upper-face
//    contributions to the next plane in registers.  No atomics: every output is a
//    fixed-order sum.  Tiles overlap by one element column on their low side.
//  * k_fine3_dense / k_fine2_dense: one thread per node, dense K0 rows over its 2^d
//    elements.  Works for any element matrix; used when K0 lacks the box structure and
//    as an independent cross-check.
#pragma once
#include "common.cuh"
#include "element_op.cuh"

namespace edge {

// ------------------------------------------------------------------ epilogues
// Each epilogue receives the node slot s, the node's input values `own` (raw on
// constrained components) and the operator output Au (identity rows applied).
// kIoBytes: algorithmic bytes per DOF the epilogue reads/writes besides the input vector.
template <typename T, typename TO> struct EpiStore {
  TO* out;
  long long n;
  static constexpr bool kDot = false;
  static constexpr int kIoBytes = sizeof(TO);
  EDGE_D void init() {}
  EDGE_D void operator()(long long s, int dof, const T* own, const T* Au, double& acc) const {
    for (int c = 0; c < dof; ++c) out[c * n + s] = Conv<TO>::from(Au[c]);
  }
  struct Pre {};
  EDGE_D Pre pre(long long) const { return {}; }
  EDGE_D void apply(long long s, const T* own, const T* Au, const Pre&, double& acc) const {
    operator()(s, 3, own, Au, acc);
  }
};

// out = A u and acc += u . (A u)   (PCG: q = A p, p.q)
template <typename T> struct EpiStoreDot {
  T* out;
  long long n;
  static constexpr bool kDot = true;
  static constexpr int kIoBytes = sizeof(T);
  EDGE_D void init() {}
  EDGE_D void operator()(long long s, int dof, const T* own, const T* Au, double& acc) const {
    for (int c = 0; c < dof; ++c) {
      out[c * n + s] = Au[c];
      acc += (double)own[c] * (double)Au[c];
    }
  }  struct Pre {};
  EDGE_D Pre pre(long long) const { return {}; }
  EDGE_D void apply(long long s, const T* own, const T* Au, const Pre&, double& acc) const {
    operator()(s, 3, own, Au, acc);
  }
};

// r = b - A u
template <typename T, typename TB, typename TO> struct EpiResid {
  const TB* b;
  TO* r;
  long long n;
  static constexpr bool kDot = false;
  static constexpr int kIoBytes = sizeof(TB) + sizeof(TO);
  EDGE_D void init() {}
  EDGE_D void operator()(long long s, int dof, const T* own, const T* Au, double& acc) const {
    for (int c = 0; c < dof; ++c) r[c * n + s] = Conv<TO>::from(Conv<T>::from(b[c * n + s]) - Au[c]);
  }
  struct Pre {
    T b[3];
  };
  EDGE_D Pre pre(long long s) const {
    Pre p;
    for (int c = 0; c < 3; ++c) p.b[c] = Conv<T>::from(b[c * n + s]);
    return p;
  }
  EDGE_D void apply(long long s, const T* own, const T* Au, const Pre& p, double& acc) const {
    for (int c = 0; c < 3; ++c) r[c * n + s] = Conv<TO>::from(p.b[c] - Au[c]);
  }
};

// xo = u + w * Dinv * (b - A u),  w = omega * wscale (omega read from device memory)
template <typename T, typename TB, typename TD> struct EpiJacobi {
  const TB* b;
  const TD* dinv;
  T* xo;
  const double* omega;
  double wscale;
  long long n;
  T w;
  static constexpr bool kDot = false;
  static constexpr int kIoBytes = sizeof(TB) + sizeof(TD) + sizeof(T);
  EDGE_D void init() { w = Conv<T>::from(__ldg(omega) * wscale); }
  EDGE_D void operator()(long long s, int dof, const T* own, const T* Au, double& acc) const {
    for (int c = 0; c < dof; ++c) {
      const long long q = c * n + s;
      xo[q] = own[c] + w * Conv<T>::from(dinv[q]) * (Conv<T>::from(b[q]) - Au[c]);
    }
  }
  struct Pre {
    T b[3], d[3];
  };
  EDGE_D Pre pre(long long s) const {
    Pre p;
    for (int c = 0; c < 3; ++c) {
      p.b[c] = Conv<T>::from(b[c * n + s]);
      p.d[c] = Conv<T>::from(dinv[c * n + s]);
    }
    return p;
  }
  EDGE_D void apply(long long s, const T* own, const T* Au, const Pre& p, double& acc) const {
    for (int c = 0; c < 3; ++c) xo[c * n + s] = own[c] + w * p.d[c] * (p.b[c] - Au[c]);
  }
};

// Last post-smoothing sweep fused with the correction: xo = xbase + e + w Dinv (b - A e),
// with e = u.  With kDot, acc += dotv . xo (the PCG's r.z at level 0).
template <typename T, typename TB, typename TD, typename TX, bool DOT, typename TV = TB> struct EpiJacobiAdd {
  const TB* b;
  const TD* dinv;
  const TX* xbase;
  TX* xo;
  const TV* dotv;
  const double* omega;
  double wscale;
  long long n;
  T w;
  static constexpr bool kDot = DOT;
  static constexpr int kIoBytes = sizeof(TB) + sizeof(TD) + 2 * sizeof(TX) + (DOT ? sizeof(TV) : 0);
  EDGE_D void init() { w = Conv<T>::from(__ldg(omega) * wscale); }
  EDGE_D void operator()(long long s, int dof, const T* own, const T* Au, double& acc) const {
    for (int c = 0; c < dof; ++c) {
      const long long q = c * n + s;
      T e = own[c] + w * Conv<T>::from(dinv[q]) * (Conv<T>::from(b[q]) - Au[c]);
      TX v = Conv<TX>::from(Conv<T>::from(xbase[q]) + e);
      xo[q] = v;
      if (DOT) acc += (double)dotv[q] * (double)v;
    }
  }
  struct Pre {
    T b[3], d[3], xb[3];
    TV dv[DOT ? 3 : 1];
  };
  EDGE_D Pre pre(long long s) const {
    Pre p;
    for (int c = 0; c < 3; ++c) {
      const long long q = c * n + s;
      p.b[c] = Conv<T>::from(b[q]);
      p.d[c] = Conv<T>::from(dinv[q]);
      p.xb[c] = Conv<T>::from(xbase[q]);
      if constexpr (DOT) p.dv[c] = dotv[q];
    }
    return p;
  }
  EDGE_D void apply(long long s, const T* own, const T* Au, const Pre& p, double& acc) const {
    for (int c = 0; c < 3; ++c) {
      const T e = own[c] + w * p.d[c] * (p.b[c] - Au[c]);
      const TX v = Conv<TX>::from(p.xb[c] + e);
      xo[c * n + s] = v;
      if constexpr (DOT) acc += (double)p.dv[c] * (double)v;
    }
  }
};

struct DotSink {
  double* dst;
  EDGE_D void operator()(double t) const { *dst = t; }
};

template <class Epi>
EDGE_D void finish_dot(const Epi&, double acc, double* part, unsigned* ticket, double* dst) {
  if constexpr (Epi::kDot) {
    __shared__ double sh[32];
    double bt = block_sum(acc, sh);
    grid_reduce_finish(bt, part, ticket, DotSink{dst});
  }
}

// ------------------------------------------------------------------ 3-D tiled WHT kernel
template <typename T, typename TE, class Epi, int BX>
__global__ void __launch_bounds__(32 * BX)
k_fine3_wht(const Geo g, const T* __restrict__ u, const TE* __restrict__ E, const uint8_t* __restrict__ mask,
            const KHat3<T> K, const int ly, Epi epi, double* part, unsigned* ticket, double* dot_dst) {
  EDGE_PDL_ENTRY();
  __shared__ T sU[2][3][BX + 1][34];
  __shared__ T sG[2][2][3][BX][33];
  const int lane = threadIdx.x, wx = threadIdx.y, tid = lane + 32 * wx;
  const int z0 = blockIdx.x * 31, x0 = blockIdx.y * (BX - 1);
  const int y0 = blockIdx.z * ly;
  const int y1 = min(y0 + ly, g.ny);
  const int ez = z0 - 1 + lane, ex = x0 - 1 + wx;
  const long long n = g.n;
  epi.init();

  auto stage = [&](int buf, int p) {
    for (int t = tid; t < (BX + 1) * 33; t += 32 * BX) {
      const int tz = t % 33, tx = t / 33;
      const int kz = z0 - 1 + tz, ix = x0 - 1 + tx;
      T v0 = T(0), v1 = T(0), v2 = T(0);
      if (p >= 0 && p < g.ny && kz >= 0 && kz < g.nz && ix >= 0 && ix < g.nx) {
        const long long s = g.slot3(ix, p, kz);
        const uint8_t m = __ldg(mask + s);
        v0 = (m & 1) ? T(0) : __ldg(u + s);
        v1 = (m & 2) ? T(0) : __ldg(u + s + n);
        v2 = (m & 4) ? T(0) : __ldg(u + s + 2 * n);
      }
      sU[buf][0][tx][tz] = v0;
      sU[buf][1][tx][tz] = v1;
      sU[buf][2][tx][tz] = v2;
    }
  };

  T ul[2][2][3];
  T acc[3] = {T(0), T(0), T(0)};
  double dacc = 0.0;
  stage(0, y0 - 1);
  __syncthreads();
#pragma unroll
  for (int dx = 0; dx < 2; ++dx)
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
      for (int c = 0; c < 3; ++c) ul[dx][dz][c] = sU[0][c][wx + dx][lane + dz];

  int buf = 1;
  for (int ey = y0 - 1; ey < y1; ++ey, buf ^= 1) {
    stage(buf, ey + 1);
    __syncthreads();
    T uu[2][2][3];
#pragma unroll
    for (int dx = 0; dx < 2; ++dx)
#pragma unroll
      for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int c = 0; c < 3; ++c) uu[dx][dz][c] = sU[buf][c][wx + dx][lane + dz];
    T Ee = T(0);
    if (ez >= 0 && ez < g.nz - 1 && ex >= 0 && ex < g.nx - 1 && ey >= 0 && ey < g.ny - 1)
      Ee = Conv<T>::from(__ldg(E + g.slot3(ex, ey, ez)));
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
#pragma unroll
    for (int ay = 0; ay < 2; ++ay)
#pragma unroll
      for (int c = 0; c < 3; ++c) sG[buf][ay][c][wx][lane] = gz[1][ay][c];
    __syncthreads();
    T tot[2][3];
#pragma unroll
    for (int ay = 0; ay < 2; ++ay)
#pragma unroll
      for (int c = 0; c < 3; ++c) tot[ay][c] = gz[0][ay][c] + (wx > 0 ? sG[buf][ay][c][wx - 1][lane] : T(0));
    if (ey >= y0 && lane >= 1 && wx >= 1 && ez < g.nz && ex < g.nx) {
      const long long s = g.slot3(ex, ey, ez);
      const uint8_t m = __ldg(mask + s);
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
  }
  finish_dot(epi, dacc, part, ticket, dot_dst);
}

// ------------------------------------------------------------------ 2-D tiled WHT kernel
template <typename T, typename TE, class Epi, int NW>
__global__ void __launch_bounds__(32 * NW)
k_fine2_wht(const Geo g, const T* __restrict__ u, const TE* __restrict__ E, const uint8_t* __restrict__ mask,
            const KHat2<T> K, const int ly, Epi epi, double* part, unsigned* ticket, double* dot_dst) {
  EDGE_PDL_ENTRY();
  constexpr int NT = 32 * NW;
  __shared__ T sU[2][2][NT + 2];
  __shared__ T sG[2][2][2][NT + 1];
  const int t = threadIdx.x;
  const int x0 = blockIdx.x * (NT - 1);
  const int y0 = blockIdx.y * ly;
  const int y1 = min(y0 + ly, g.ny);
  const int ex = x0 - 1 + t;
  const long long n = g.n;
  epi.init();

  auto stage = [&](int buf, int p) {
    for (int q = t; q < NT + 1; q += NT) {
      const int ix = x0 - 1 + q;
      T v0 = T(0), v1 = T(0);
      if (p >= 0 && p < g.ny && ix >= 0 && ix < g.nx) {
        const long long s = g.slot2(ix, p);
        const uint8_t m = __ldg(mask + s);
        v0 = (m & 1) ? T(0) : __ldg(u + s);
        v1 = (m & 2) ? T(0) : __ldg(u + s + n);
      }
      sU[buf][0][q] = v0;
      sU[buf][1][q] = v1;
    }
  };

  T ul[2][2];
  T acc[2] = {T(0), T(0)};
  double dacc = 0.0;
  stage(0, y0 - 1);
  __syncthreads();
#pragma unroll
  for (int dx = 0; dx < 2; ++dx)
#pragma unroll
    for (int c = 0; c < 2; ++c) ul[dx][c] = sU[0][c][t + dx];
  int buf = 1;
  for (int ey = y0 - 1; ey < y1; ++ey, buf ^= 1) {
    stage(buf, ey + 1);
    __syncthreads();
    T uu[2][2];
#pragma unroll
    for (int dx = 0; dx < 2; ++dx)
#pragma unroll
      for (int c = 0; c < 2; ++c) uu[dx][c] = sU[buf][c][t + dx];
    T Ee = T(0);
    if (ex >= 0 && ex < g.nx - 1 && ey >= 0 && ey < g.ny - 1) Ee = Conv<T>::from(__ldg(E + g.slot2(ex, ey)));
    T u4[4][2], f[4][2];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int bx = b & 1, by = (b >> 1) & 1;
#pragma unroll
      for (int c = 0; c < 2; ++c) u4[b][c] = by ? uu[bx][c] : ul[bx][c];
    }
    elem2_apply(K, Ee, u4, f);
#pragma unroll
    for (int ay = 0; ay < 2; ++ay)
#pragma unroll
      for (int c = 0; c < 2; ++c) sG[buf][ay][c][t] = f[1 | (ay << 1)][c];
    __syncthreads();
    T tot[2][2];
#pragma unroll
    for (int ay = 0; ay < 2; ++ay)
#pragma unroll
      for (int c = 0; c < 2; ++c) tot[ay][c] = f[ay << 1][c] + (t > 0 ? sG[buf][ay][c][t - 1] : T(0));
    if (ey >= y0 && t >= 1 && ex < g.nx) {
      const long long s = g.slot2(ex, ey);
      const uint8_t m = __ldg(mask + s);
      T own[2], Au[2];
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        own[c] = ul[0][c];
        Au[c] = acc[c] + tot[0][c];
        if ((m >> c) & 1) {
          own[c] = __ldg(u + c * n + s);
          Au[c] = own[c];
        }
      }
      epi(s, 2, own, Au, dacc);
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) acc[c] = tot[1][c];
#pragma unroll
    for (int dx = 0; dx < 2; ++dx)
#pragma unroll
      for (int c = 0; c < 2; ++c) ul[dx][c] = uu[dx][c];
  }
  finish_dot(epi, dacc, part, ticket, dot_dst);
}

// ------------------------------------------------------------------ dense node-centric kernels
// K0b: element matrix with corners in bit order, row-major (2^d*dof)^2, in global memory.
template <typename T, typename TE, class Epi>
__global__ void __launch_bounds__(128)
k_fine3_dense(const Geo g, const T* __restrict__ u, const TE* __restrict__ E, const uint8_t* __restrict__ mask,
              const T* __restrict__ K0b, Epi epi, double* part, unsigned* ticket, double* dot_dst) {
  EDGE_PDL_ENTRY();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  const int j = blockIdx.z;
  const long long n = g.n;
  epi.init();
  double dacc = 0.0;
  if (k < g.nz) {
    const long long s = g.slot3(i, j, k);
    T Au[3] = {T(0), T(0), T(0)};
    for (int a = 0; a < 8; ++a) {  // this node is corner a of element (i-ax, j-ay, k-az)
      const int ax = a & 1, ay = (a >> 1) & 1, az = (a >> 2) & 1;
      const int li = i - ax, lj = j - ay, lk = k - az;
      if (li < 0 || lj < 0 || lk < 0 || li >= g.nx - 1 || lj >= g.ny - 1 || lk >= g.nz - 1) continue;
      const T Ee = Conv<T>::from(__ldg(E + g.slot3(li, lj, lk)));
      T r[3] = {T(0), T(0), T(0)};
      for (int b = 0; b < 8; ++b) {
        const long long sb = g.slot3(li + (b & 1), lj + ((b >> 1) & 1), lk + ((b >> 2) & 1));
        const uint8_t mb = __ldg(mask + sb);
        for (int d = 0; d < 3; ++d) {
          if ((mb >> d) & 1) continue;
          const T ub = __ldg(u + d * n + sb);
          for (int c = 0; c < 3; ++c) r[c] += __ldg(K0b + (a * 3 + c) * 24 + b * 3 + d) * ub;
        }
      }
      for (int c = 0; c < 3; ++c) Au[c] += Ee * r[c];
    }
    const uint8_t m = __ldg(mask + s);
    T own[3];
    for (int c = 0; c < 3; ++c) {
      own[c] = __ldg(u + c * n + s);
      if ((m >> c) & 1) Au[c] = own[c];
    }
    epi(s, 3, own, Au, dacc);
  }
  finish_dot(epi, dacc, part, ticket, dot_dst);
}

template <typename T, typename TE, class Epi>
__global__ void __launch_bounds__(128)
k_fine2_dense(const Geo g, const T* __restrict__ u, const TE* __restrict__ E, const uint8_t* __restrict__ mask,
              const T* __restrict__ K0b, Epi epi, double* part, unsigned* ticket, double* dot_dst) {
  EDGE_PDL_ENTRY();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  const long long n = g.n;
  epi.init();
  double dacc = 0.0;
  if (i < g.nx) {
    const long long s = g.slot2(i, j);
    T Au[2] = {T(0), T(0)};
    for (int a = 0; a < 4; ++a) {
      const int ax = a & 1, ay = (a >> 1) & 1;
      const int li = i - ax, lj = j - ay;
      if (li < 0 || lj < 0 || li >= g.nx - 1 || lj >= g.ny - 1) continue;
      const T Ee = Conv<T>::from(__ldg(E + g.slot2(li, lj)));
      T r[2] = {T(0), T(0)};
      for (int b = 0; b < 4; ++b) {
        const long long sb = g.slot2(li + (b & 1), lj + ((b >> 1) & 1));
        const uint8_t mb = __ldg(mask + sb);
        for (int d = 0; d < 2; ++d) {
          if ((mb >> d) & 1) continue;
          const T ub = __ldg(u + d * n + sb);
          for (int c = 0; c < 2; ++c) r[c] += __ldg(K0b + (a * 2 + c) * 8 + b * 2 + d) * ub;
        }
      }
      for (int c = 0; c < 2; ++c) Au[c] += Ee * r[c];
    }
    const uint8_t m = __ldg(mask + s);
    T own[2];
    for (int c = 0; c < 2; ++c) {
      own[c] = __ldg(u + c * n + s);
      if ((m >> c) & 1) Au[c] = own[c];
    }
    epi(s, 2, own, Au, dacc);
  }
  finish_dot(epi, dacc, part, ticket, dot_dst);
}

}  // namespace edge
