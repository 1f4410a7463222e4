// Many independent 2-D problems solved in one persistent launch.
//
// k_batch_pcg: a team of C blocks (one block, or a thread block cluster of C blocks) takes
// the next unsolved problem from a queue (one atomicAdd per problem; the host orders the
// problems largest first, so the long solves start first) and runs that problem's whole
// solve before taking the next: PCG with the Krylov vectors, the
// search direction's product and every inner product in FP64, preconditioned by the
// problem's V-cycle in the problem's precision (FP64; or FP32 with the BF16 fine-level Jacobi
// diagonal and BF16 coarse stencils of the mixed path), on the hierarchy that the problem's
// own set-up built (Galerkin stencils, Jacobi diagonals, the coarsest dense inverse).
//
// The V-cycle is the per-problem solver's (pre- and post-smoothing sweeps per level,
// omega * 1.06^level, full-weighting restriction and its interpolation, the exact coarsest
// solve), the PCG recurrence and the residual-driven omega schedule those of
// solvers/_multigrid_cuda.py:188-241.  Every step is one pass of the block over one level's
// nodes (the team's threads striding over them) followed by a team barrier (__syncthreads, or
// the cluster barrier with its release/acquire ordering), which makes the team's global writes
// visible to its next step (data written inside the launch is read with plain loads, never
// through the read-only path); inner products are sums in a fixed order (per block, then over
// the cluster's blocks through distributed shared memory), so a problem's result does not
// depend on the team that solved it or on the other problems.  The PCG loop is bounded by
// maxiter; the queue counter is the only state shared between teams and nothing waits on it
// (the cluster barrier only joins the blocks of one team, which run together).
#pragma once
#include <cooperative_groups.h>

#include "common.cuh"
#include "coarse.cuh"
#include "misc.cuh"

namespace edge {

// The blocks that solve one problem together.  sum(): the team-wide FP64 sum of a per-thread
// value in a fixed order, returned to every thread; `sh` holds 33 + C doubles of shared memory.
template <int C> struct Team {
  static EDGE_D unsigned rank() {
    if constexpr (C == 1) return 0;
    else return cooperative_groups::this_cluster().block_rank();
  }
  static EDGE_D int first() { return (int)(rank() * blockDim.x + threadIdx.x); }
  static EDGE_D int stride() { return C * (int)blockDim.x; }
  static EDGE_D void sync() {
    if constexpr (C == 1) __syncthreads();
    else cooperative_groups::this_cluster().sync();
  }
  static EDGE_D double sum(double v, double* sh) {
    double r = block_sum(v, sh);  // valid in thread 0 of each block
    if constexpr (C == 1) {
      __syncthreads();
      if (threadIdx.x == 0) sh[32] = r;
      __syncthreads();
      r = sh[32];
      __syncthreads();
      return r;
    } else {
      auto cl = cooperative_groups::this_cluster();
      if (threadIdx.x == 0) cl.map_shared_rank(sh + 33, 0)[rank()] = r;
      cl.sync();
      const double* src = cl.map_shared_rank(sh + 33, 0);
      double t = 0.0;
#pragma unroll
      for (int k = 0; k < C; ++k) t += src[k];
      cl.sync();  // rank 0's slots and every block's sh are reused by the next sum
      return t;
    }
  }
};

constexpr int BATCH_MAXL = 8;             // levels 0..7
constexpr int BATCH_COARSE_SMEM = 1024;  // coarsest right-hand sides up to this size are staged in shared memory

struct BatchLevel {
  Geo g;
  void *b, *xa, *xb, *r, *ea, *eb, *res;  // V-cycle vectors (type TV; b unused on level 0)
  const void* S;                          // stencil, levels >= 1 (type TS)
  const void* dinv;                       // Jacobi inverse diagonal (level 0: TD0, else TV)
};

// One problem of the batch: pointers into the problem's own buffers (edge_problem) and the
// solver settings of its multigrid.
struct BatchDesc {
  int n_level, nd, keep_omega, pad0;
  int sweeps[BATCH_MAXL];
  double wscale[BATCH_MAXL];  // 1.06^level
  double omega, min_omega, omega0;
  const uint8_t* mask;
  const double* E64;  // fine-level E in FP64 (the search direction's product)
  const void* ET;     // fine-level E in the V-cycle's type
  const double* K0_64;  // element matrix, corner-bit order, FP64
  const void* K0_T;     // the same in the V-cycle's type
  double *b64, *x64, *r64, *p64, *q64;
  const double* Ainv;
  PcgState* st;
  const int* chol_status;
  BatchLevel lv[BATCH_MAXL];
};

// Fine-level operator of a 2-D problem, one pass of the block over the level's nodes: at
// node (i, j), A u from the 3 x 3 neighbourhood (constrained components of u read as zero)
// and the four surrounding elements' E with the dense element matrix sK (corner-bit order,
// shared memory), in the order of k_fine2_dense; identity rows on constrained DOFs.
// epi(s, own, Au) finishes node slot s (own: the node's raw input values).  Every load of a
// node is unconditional (a neighbour or element outside the grid reads the node's own slot
// and is replaced by zero), so a thread's loads are in flight together: each pass is a few
// round trips to L2 per node, not one per neighbour.
// Input of the fine operator: u itself (ArrIn) or a value computed from other arrays
// (uin(slot, component)).
template <typename T> struct ArrIn {
  const T* u;
  long long n;
  EDGE_D T operator()(long long ss, int c) const { return u[c * n + ss]; }
};

template <int C, typename T, typename TE, class UIn, class F>
EDGE_D void b_fine2(const Geo& g, UIn uin, const TE* E, const uint8_t* mask, const T* sK, F&& epi) {
  const int nn = g.nx * g.ny;
  for (int t = Team<C>::first(); t < nn; t += Team<C>::stride()) {
    const int i = t % g.nx, j = t / g.nx;
    const long long s = g.slot2(i, j);
    T U[3][3][2];
#pragma unroll
    for (int dy = 0; dy < 3; ++dy)
#pragma unroll
      for (int dx = 0; dx < 3; ++dx) {
        const int ii = i + dx - 1, jj = j + dy - 1;
        const bool in = ii >= 0 && ii < g.nx && jj >= 0 && jj < g.ny;
        const long long ss = in ? s + (long long)(dy - 1) * g.pz + (dx - 1) : s;
        const uint8_t mr = __ldg(mask + ss);
        const uint8_t m = in ? mr : (uint8_t)3;
        const T a0 = uin(ss, 0), a1 = uin(ss, 1);
        U[dy][dx][0] = (m & 1) ? T(0) : a0;
        U[dy][dx][1] = (m & 2) ? T(0) : a1;
      }
    T Au[2] = {T(0), T(0)};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int ax = a & 1, ay = a >> 1;
      const int li = i - ax, lj = j - ay;
      const bool ev = li >= 0 && lj >= 0 && li < g.nx - 1 && lj < g.ny - 1;
      const TE Ev = __ldg(E + (ev ? g.slot2(li, lj) : s));
      const T Ee = ev ? Conv<T>::from(Ev) : T(0);
      T r[2] = {T(0), T(0)};
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int bx = b & 1, by = b >> 1;
#pragma unroll
        for (int dd = 0; dd < 2; ++dd) {
          const T ub = U[by - ay + 1][bx - ax + 1][dd];
#pragma unroll
          for (int c = 0; c < 2; ++c) r[c] += sK[(a * 2 + c) * 8 + b * 2 + dd] * ub;
        }
      }
#pragma unroll
      for (int c = 0; c < 2; ++c) Au[c] += Ee * r[c];
    }
    const uint8_t m = __ldg(mask + s);
    T own[2] = {uin(s, 0), uin(s, 1)};
    Au[0] = (m & 1) ? own[0] : Au[0];
    Au[1] = (m & 2) ? own[1] : Au[1];
    epi(s, own, Au);
  }
}

// Symmetric 2-D stencil (levels >= 1), one pass of the block over the level's nodes, the
// sums of k_st2_apply in its order (a neighbour outside the grid reads the node's own slots
// and contributes zero, so no load is conditional).
template <int C, typename T, typename TS, class F>
EDGE_D void b_st2(const Geo& g, const T* u, const TS* S, F&& epi) {
  const long long n = g.n;
  const int nn = g.nx * g.ny;
  for (int t = Team<C>::first(); t < nn; t += Team<C>::stride()) {
    const int i = t % g.nx, j = t / g.nx;
    const long long s = g.slot2(i, j);
    const T u0 = u[s], u1 = u[n + s];
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
      {
        const bool in = i + dx >= 0 && i + dx < g.nx && j + dy >= 0 && j + dy < g.ny;
        const long long sn = in ? s + off : s;
        const T v0 = in ? u[sn] : T(0), v1 = in ? u[n + sn] : T(0);
        Au[0] += Conv<T>::from(__ldg(Sb + s)) * v0 + Conv<T>::from(__ldg(Sb + n + s)) * v1;
        Au[1] += Conv<T>::from(__ldg(Sb + 2 * n + s)) * v0 + Conv<T>::from(__ldg(Sb + 3 * n + s)) * v1;
      }
      {
        const bool in = i - dx >= 0 && i - dx < g.nx && j - dy >= 0 && j - dy < g.ny;
        const long long sm = in ? s - off : s;
        const T v0 = in ? u[sm] : T(0), v1 = in ? u[n + sm] : T(0);
        Au[0] += Conv<T>::from(__ldg(Sb + sm)) * v0 + Conv<T>::from(__ldg(Sb + 2 * n + sm)) * v1;
        Au[1] += Conv<T>::from(__ldg(Sb + n + sm)) * v0 + Conv<T>::from(__ldg(Sb + 3 * n + sm)) * v1;
      }
    }
    T own[2] = {u0, u1};
    epi(s, own, Au);
  }
}

// Full-weighting restriction to the coarse nodes (k_restrict2's sums).
template <int C, typename T>
EDGE_D void b_restrict2(const Geo& gf, const Geo& gc, const T* in, T* out) {
  const int nc = gc.nx * gc.ny;
  for (int t = Team<C>::first(); t < nc; t += Team<C>::stride()) {
    const int I = t % gc.nx, J = t / gc.nx;
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
        for (int c = 0; c < 2; ++c) v[c] += w * in[c * gf.n + sf];
      }
    }
    const long long sc = gc.slot2(I, J);
    for (int c = 0; c < 2; ++c) out[c * gc.n + sc] = v[c] * iw;
  }
}

// Interpolation to the fine nodes (k_prolong2's sums).
template <int C, typename T>
EDGE_D void b_prolong2(const Geo& gf, const Geo& gc, const T* in, T* out) {
  const int nf = gf.nx * gf.ny;
  for (int t = Team<C>::first(); t < nf; t += Team<C>::stride()) {
    const int i = t % gf.nx, j = t / gf.nx;
    T v[2] = {0, 0};
    int cnt = 0;
    for (int ci = i / 2; ci <= i / 2 + (i & 1); ++ci) {
      if (ci >= gc.nx) continue;
      for (int cj = j / 2; cj <= j / 2 + (j & 1); ++cj) {
        if (cj >= gc.ny) continue;
        const T iw = inv_bnd_total2<T>(is_bnd(ci, gc.nx) + is_bnd(cj, gc.ny));
        const long long sc = gc.slot2(ci, cj);
        for (int c = 0; c < 2; ++c) v[c] += in[c * gc.n + sc] * iw;
        ++cnt;
      }
    }
    const T ic = cnt ? T(1) / T(cnt) : T(0);
    const long long sf = gf.slot2(i, j);
    for (int c = 0; c < 2; ++c) out[c * gf.n + sf] = v[c] * ic;
  }
}

// x = Ainv b on the coarsest level (dense order: DOF c of node j * nx + i), one warp per row;
// every block of the team stages b (written before the team's last barrier) for its rows.
template <int C, typename T>
EDGE_D void b_coarse2(const Geo& g, const double* Ainv, int nd, const T* b, T* x, double* sb) {
  auto slot_of = [&](int dn) -> long long {
    const int node = dn >> 1;
    return (long long)(dn & 1) * g.n + g.slot2(node % g.nx, node / g.nx);
  };
  const bool staged = nd <= BATCH_COARSE_SMEM;
  if (staged) {
    for (int c = threadIdx.x; c < nd; c += blockDim.x) sb[c] = (double)b[slot_of(c)];
    __syncthreads();
  }
  const int lane = threadIdx.x & 31, nw = Team<C>::stride() >> 5;
  for (int row = Team<C>::first() >> 5; row < nd; row += nw) {
    const double* a = Ainv + (long long)row * nd;
    double acc = 0.0;
    for (int c = lane; c < nd; c += 32) acc += __ldg(a + c) * (staged ? sb[c] : (double)b[slot_of(c)]);
    acc = warp_sum(acc);
    if (lane == 0) x[slot_of(row)] = Conv<T>::from(acc);
  }
}

template <int C, typename TA, typename TB>
EDGE_D double b_dot(long long nv, const TA* a, const TB* b, double* sh) {
  double acc = 0.0;
  for (long long q = Team<C>::first(); q < nv; q += Team<C>::stride()) acc += (double)a[q] * (double)b[q];
  return Team<C>::sum(acc, sh);
}

// One application of level l's operator (fine: the element operator in TV; coarser: the
// stencil in TS, arithmetic in TV).
template <int C, typename TV, typename TS, class F>
EDGE_D void b_level_op(const BatchDesc& d, int l, const TV* u, const TV* sK, F&& epi) {
  if (l == 0)
    b_fine2<C, TV, TV>(d.lv[0].g, ArrIn<TV>{u, d.lv[0].g.n}, (const TV*)d.ET, d.mask, sK, epi);
  else
    b_st2<C, TV, TS>(d.lv[l].g, u, (const TS*)d.lv[l].S, epi);
}

// Damped-Jacobi pieces with level l's inverse diagonal (type TD); the level's right-hand side
// b has type TB (level 0: the FP64 PCG residual, read in the V-cycle's type).  down: x = w
// Dinv b (k_jacobi0), ns - 1 more sweeps, r = b - A x; with one sweep on level 0 the two are
// one pass (the operator's input w Dinv b computed where it is read, x never stored: fused0).
// up (after the interpolation into e1): ns - 1 sweeps on the correction, then
// out = xb + (e + w Dinv (r - A e)) with xb the down pass's x (recomputed as w Dinv b when
// fused0); with dot, acc += dotv . out (the PCG's r.z) per thread.
template <int C, typename TV, typename TS, typename TD, typename TB>
EDGE_D void b_smooth_level(const BatchDesc& d, int l, const TV* sK, TV w, const TB* b, const TV* xb, TV*& x, TV*& y,
                           TV*& e1, TV*& e2, TV* r, TV* out, bool down, bool fused0, const double* dotv,
                           double& acc) {
  using TM = Team<C>;
  const BatchLevel& Lv = d.lv[l];
  const Geo& g = Lv.g;
  const long long n = g.n, nv = 2 * n;
  const TD* D = (const TD*)Lv.dinv;
  const int ns = d.sweeps[l];
  auto bv = [&](long long q) { return Conv<TV>::from(b[q]); };
  auto wdb = [&](long long q) { return w * Conv<TV>::from(__ldg(D + q)) * bv(q); };
  auto sweep = [&](const TV* bb, const TV* in, TV* o) {
    b_level_op<C, TV, TS>(d, l, in, sK, [&](long long s, const TV* own, const TV* Au) {
      for (int c = 0; c < 2; ++c) {
        const long long q = c * n + s;
        o[q] = own[c] + w * Conv<TV>::from(__ldg(D + q)) * (bb[q] - Au[c]);
      }
    });
    TM::sync();
  };
  auto sweep_b = [&](const TV* in, TV* o) {  // a sweep on the down pass (right-hand side b)
    b_level_op<C, TV, TS>(d, l, in, sK, [&](long long s, const TV* own, const TV* Au) {
      for (int c = 0; c < 2; ++c) {
        const long long q = c * n + s;
        o[q] = own[c] + w * Conv<TV>::from(__ldg(D + q)) * (bv(q) - Au[c]);
      }
    });
    TM::sync();
  };
  if (down) {
    if (fused0) {
      b_fine2<C, TV, TV>(g, [&](long long ss, int c) { return wdb(c * n + ss); }, (const TV*)d.ET, d.mask, sK,
                         [&](long long s, const TV* own, const TV* Au) {
                           for (int c = 0; c < 2; ++c) r[c * n + s] = bv(c * n + s) - Au[c];
                         });
      TM::sync();
      return;
    }
    if (ns >= 1) {
      for (long long q = TM::first(); q < nv; q += TM::stride()) x[q] = wdb(q);
      TM::sync();
      for (int s = 1; s < ns; ++s) {
        sweep_b(x, y);
        TV* t = x;
        x = y;
        y = t;
      }
    } else {
      for (long long q = TM::first(); q < nv; q += TM::stride()) x[q] = TV(0);
      TM::sync();
    }
    b_level_op<C, TV, TS>(d, l, x, sK, [&](long long s, const TV* own, const TV* Au) {
      for (int c = 0; c < 2; ++c) r[c * n + s] = bv(c * n + s) - Au[c];
    });
    TM::sync();
  } else {
    for (int s = 0; s + 1 < ns; ++s) {
      sweep(r, e1, e2);
      TV* t = e1;
      e1 = e2;
      e2 = t;
    }
    auto xbase = [&](long long q) { return fused0 ? wdb(q) : xb[q]; };
    if (ns >= 1) {
      b_level_op<C, TV, TS>(d, l, e1, sK, [&](long long s, const TV* own, const TV* Au) {
        for (int c = 0; c < 2; ++c) {
          const long long q = c * n + s;
          const TV e = own[c] + w * Conv<TV>::from(__ldg(D + q)) * (r[q] - Au[c]);
          const TV v = xbase(q) + e;
          out[q] = v;
          if (dotv) acc += dotv[q] * (double)v;
        }
      });
    } else {
      for (long long q = TM::first(); q < nv; q += TM::stride()) {
        const TV v = Conv<TV>::from((double)xb[q] + (double)e1[q]);
        out[q] = v;
        if (dotv) acc += dotv[q] * (double)v;
      }
    }
    if (!dotv) TM::sync();  // with dot, the team sum that follows is the barrier
  }
}

// z = V-cycle(r) into lv[0].res, r the FP64 PCG residual (read in the V-cycle's type); returns
// this thread's part of r.z, which the caller sums over the team.
template <int C, typename TV, typename TD0, typename TS>
EDGE_D double b_vcycle(const BatchDesc& d, const TV* sK, double omega, double* sb) {
  using TM = Team<C>;
  const int L = d.n_level;
  TV* xcur[BATCH_MAXL];
  const bool fused0 = d.sweeps[0] == 1;
  double acc = 0.0;
  for (int l = 0; l < L; ++l) {
    const BatchLevel& Lv = d.lv[l];
    TV* x = (TV*)Lv.xa;
    TV* y = (TV*)Lv.xb;
    TV* e1 = nullptr;
    TV* e2 = nullptr;
    const TV w = Conv<TV>::from(omega * d.wscale[l]);
    if (l == 0)
      b_smooth_level<C, TV, TS, TD0, double>(d, l, sK, w, d.r64, nullptr, x, y, e1, e2, (TV*)Lv.r, nullptr, true,
                                              fused0, nullptr, acc);
    else
      b_smooth_level<C, TV, TS, TV, TV>(d, l, sK, w, (const TV*)Lv.b, nullptr, x, y, e1, e2, (TV*)Lv.r, nullptr,
                                        true, false, nullptr, acc);
    xcur[l] = x;
    b_restrict2<C, TV>(Lv.g, d.lv[l + 1].g, (const TV*)Lv.r, (TV*)d.lv[l + 1].b);
    TM::sync();
  }
  b_coarse2<C, TV>(d.lv[L].g, d.Ainv, d.nd, (const TV*)d.lv[L].b, (TV*)d.lv[L].res, sb);
  TM::sync();
  for (int l = L - 1; l >= 0; --l) {
    const BatchLevel& Lv = d.lv[l];
    TV* e1 = (TV*)Lv.ea;
    TV* e2 = (TV*)Lv.eb;
    TV* x = nullptr;
    TV* y = nullptr;
    b_prolong2<C, TV>(Lv.g, d.lv[l + 1].g, (const TV*)d.lv[l + 1].res, e1);
    TM::sync();
    const TV w = Conv<TV>::from(omega * d.wscale[l]);
    if (l == 0)
      b_smooth_level<C, TV, TS, TD0, double>(d, l, sK, w, d.r64, xcur[l], x, y, e1, e2, (TV*)Lv.r, (TV*)Lv.res,
                                              false, fused0, d.r64, acc);
    else
      b_smooth_level<C, TV, TS, TV, TV>(d, l, sK, w, (const TV*)Lv.b, xcur[l], x, y, e1, e2, (TV*)Lv.r,
                                        (TV*)Lv.res, false, false, nullptr, acc);
  }
  return acc;
}

template <int C, typename TV, typename TD0, typename TS>
EDGE_D void b_pcg_problem(const BatchDesc& d, const TV* sK, const double* sK64, double tol, int maxiter, double* sh,
                          double* sb) {
  using TM = Team<C>;
  const Geo& g = d.lv[0].g;
  const long long n = g.n, nv = 2 * n;
  double* x = d.x64;
  double* r = d.r64;
  double* p = d.p64;
  double* q = d.q64;
  const double* b = d.b64;
  const TV* z = (const TV*)d.lv[0].res;
  double omega = d.keep_omega ? d.st->omega : d.omega0;
  const double min_omega = d.min_omega, d_omega = d.omega - d.min_omega;
  // r = b - A x (FP64)
  b_fine2<C, double, double>(g, ArrIn<double>{x, n}, d.E64, d.mask, sK64,
                             [&](long long s, const double* own, const double* Au) {
                               for (int c = 0; c < 2; ++c) r[c * n + s] = b[c * n + s] - Au[c];
                             });
  TM::sync();
  const double bb = b_dot<C>(nv, b, b, sh);
  int done = 0, iter = 0;
  double res = 0.0, rz = 0.0, rr = 0.0;
  if (bb == 0.0) done = 1;  // nothing to solve: residual 0, like a converged solve
  if (*d.chol_status) done = 3;
  while (!done) {
    const double rz_new = TM::sum(b_vcycle<C, TV, TD0, TS>(d, sK, omega, sb), sh);
    const double beta = iter == 0 ? 0.0 : rz_new / rz;
    for (long long k = TM::first(); k < nv; k += TM::stride())
      p[k] = iter == 0 ? (double)z[k] : (double)z[k] + beta * p[k];
    TM::sync();
    double acc = 0.0;
    b_fine2<C, double, double>(g, ArrIn<double>{p, n}, d.E64, d.mask, sK64,
                               [&](long long s, const double* own, const double* Au) {
                                 for (int c = 0; c < 2; ++c) {
                                   q[c * n + s] = Au[c];
                                   acc += own[c] * Au[c];
                                 }
                               });
    const double pq = TM::sum(acc, sh);
    const double alpha = rz_new / pq;
    double racc = 0.0;
    for (long long k = TM::first(); k < nv; k += TM::stride()) {
      x[k] = x[k] + alpha * p[k];
      const double rv = r[k] - alpha * q[k];
      r[k] = rv;
      racc += rv * rv;
    }
    rr = TM::sum(racc, sh);
    rz = rz_new;
    ++iter;
    const double R = sqrt(rr) / sqrt(bb);
    res = R;
    if (R < tol) {
      done = 1;
    } else {
      const double Rc = fmin(fmax(R, tol), 1e-1);
      omega = min_omega + d_omega / 2.0 * exp((-Rc + tol) * 500.0);
      if (iter >= maxiter) done = 2;
    }
  }
  if (TM::first() == 0) {
    PcgState* st = d.st;
    st->bb = bb;
    st->rr = rr;
    st->rz = rz;
    st->res = res;
    st->iter = iter;
    st->done = done;
    st->omega = omega;
  }
}

// The batched solve.  C > 1: launched as thread block clusters of C blocks (cluster
// dimension set at launch); rank 0 of a team takes the team's problems from the queue.
EDGE_D long long global_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// tns (may be null): start and end of each problem's solve (global timer, ns), for the
// benchmark's load-balance record.
template <typename TV, typename TD0, typename TS, int BT, int C>
__global__ void __launch_bounds__(BT) k_batch_pcg(const BatchDesc* D, int nprob, unsigned* queue, double tol,
                                                  int maxiter, long long* tns) {
  using TM = Team<C>;
  __shared__ double sh[33 + C];
  __shared__ double sb[BATCH_COARSE_SMEM];
  __shared__ TV sK[64];
  __shared__ double sK64[64];
  __shared__ BatchDesc sd;
  __shared__ int s_idx;
  for (;;) {
    if (TM::first() == 0) s_idx = (int)atomicAdd(queue, 1u);
    TM::sync();
    int idx;
    if constexpr (C == 1) idx = s_idx;
    else idx = *cooperative_groups::this_cluster().map_shared_rank(&s_idx, 0);
    TM::sync();  // every block has read rank 0's s_idx before rank 0 may exit or overwrite it
    if (idx >= nprob) return;
    {
      const int* src = reinterpret_cast<const int*>(D + idx);
      int* dst = reinterpret_cast<int*>(&sd);
      for (int k = threadIdx.x; k < (int)(sizeof(BatchDesc) / sizeof(int)); k += BT) dst[k] = src[k];
    }
    __syncthreads();
    for (int k = threadIdx.x; k < 64; k += BT) {
      sK[k] = reinterpret_cast<const TV*>(sd.K0_T)[k];
      sK64[k] = sd.K0_64[k];
    }
    __syncthreads();
    const long long t0 = global_ns();
    b_pcg_problem<C, TV, TD0, TS>(sd, sK, sK64, tol, maxiter, sh, sb);
    TM::sync();
    if (tns && TM::first() == 0) {
      tns[2 * idx] = t0;
      tns[2 * idx + 1] = global_ns();
    }
  }
}

// ------------------------------------------------------------------ OC updates of many problems
// One block per problem (taken from a queue like the solve): the OC update of k_oc_prep,
// k_oc_floor, k_oc_pass and k_oc_final (TopOpt/_cuda.py:242-280) with every sum a block sum in a
// fixed order and the bisection tree walked by every thread alike; at most 50 passes of
// OC_DEPTH bisection steps (the per-problem loop's bound of 200 steps).
struct BatchOcDesc {
  long long n;
  const double* rho;
  const double* dr;
  double* ocp;
  double* rho_new;
  double A, vol, vf;
};

template <int BT>
__global__ void __launch_bounds__(BT) k_batch_oc(const BatchOcDesc* D, int nprob, unsigned* queue, double move,
                                                 double* lam_out, int* steps_out) {
  using TM = Team<1>;
  __shared__ double sh[34];
  __shared__ int s_idx;
  for (;;) {
    if (threadIdx.x == 0) s_idx = (int)atomicAdd(queue, 1u);
    __syncthreads();
    const int idx = s_idx;
    __syncthreads();
    if (idx >= nprob) return;
    const BatchOcDesc d = D[idx];
    const long long n = d.n;
    double acc = 0.0;
    for (long long i = threadIdx.x; i < n; i += BT) {
      double v = d.rho[i] * sqrt(fmax(-d.dr[i] / d.A, 0.0));
      if (isnan(v)) v = 0.0;
      acc += fabs(v);
      d.ocp[i] = v;
    }
    const bool allzero = TM::sum(acc, sh) == 0.0;
    for (long long i = threadIdx.x; i < n; i += BT) d.ocp[i] = fmax(1e-12, allzero ? 1e-3 : d.ocp[i]);
    __syncthreads();
    double l1 = 1e-9, l2 = 1e9, last = 0.5 * (l1 + l2);
    int steps = 0;
    bool done = false;
    const int max_pass = (200 + OC_DEPTH - 1) / OC_DEPTH;
    for (int pass = 0; pass < max_pass && !done; ++pass) {
      double lam[OC_NODES];
      {
        double L1[OC_NODES], L2[OC_NODES];
        L1[0] = l1;
        L2[0] = l2;
        for (int t = 0; t < OC_NODES; ++t) {
          lam[t] = 0.5 * (L1[t] + L2[t]);
          if (2 * t + 2 < OC_NODES) {
            L1[2 * t + 1] = L1[t];
            L2[2 * t + 1] = lam[t];
            L1[2 * t + 2] = lam[t];
            L2[2 * t + 2] = L2[t];
          }
        }
      }
      double a[OC_NODES];
      for (int t = 0; t < OC_NODES; ++t) a[t] = 0.0;
      for (long long i = threadIdx.x; i < n; i += BT) {
        const double r = d.rho[i], o = d.ocp[i];
        for (int t = 0; t < OC_NODES; ++t) a[t] += oc_rho(r, o, lam[t], move) * d.A;
      }
      double sums[OC_NODES];
      for (int t = 0; t < OC_NODES; ++t) sums[t] = TM::sum(a[t], sh);
      int t = 0;
      for (int dd = 0; dd < OC_DEPTH; ++dd) {
        if (!((l2 - l1) / (l2 + l1) > 1e-4)) {
          done = true;
          break;
        }
        const double mid = 0.5 * (l1 + l2);
        const bool valid = (sums[t] / d.vol <= d.vf);
        if (valid) l2 = mid;
        else l1 = mid;
        last = mid;
        steps += 1;
        t = 2 * t + (valid ? 1 : 2);
      }
      if (!((l2 - l1) / (l2 + l1) > 1e-4)) done = true;
    }
    for (long long i = threadIdx.x; i < n; i += BT) d.rho_new[i] = oc_rho(d.rho[i], d.ocp[i], last, move);
    if (threadIdx.x == 0) {
      lam_out[idx] = last;
      steps_out[idx] = steps;
    }
    __syncthreads();
  }
}

// User node order (reference numbering of the real nx_r x ny_r grid) <-> slots of a grid that
// may be larger (padded): slots outside the real grid are zero.
__global__ void k_user_to_slots_pad(const Geo g, int nxr, int nyr, const double* __restrict__ user,
                                    double* __restrict__ v) {
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= g.n) return;
  const int i = (int)(s % g.pz), j = (int)(s / g.pz);
  const bool ok = i < nxr && j < nyr;
  const long long node = (long long)j * nxr + i;
  for (int c = 0; c < 2; ++c) v[c * g.n + s] = ok ? user[node * 2 + c] : 0.0;
}
__global__ void k_slots_to_user_pad(const Geo g, int nxr, int nyr, const double* __restrict__ v,
                                    double* __restrict__ user) {
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= g.n) return;
  const int i = (int)(s % g.pz), j = (int)(s / g.pz);
  if (i >= nxr || j >= nyr) return;
  const long long node = (long long)j * nxr + i;
  for (int c = 0; c < 2; ++c) user[node * 2 + c] = v[c * g.n + s];
}

// Per-problem results of a batched call into contiguous arrays: residual, iterations, stop
// reason, and the scalar the post-processing left in scal[2] (the compliance).
__global__ void k_batch_gather(const BatchDesc* D, const double* const* scal, int nprob, double* res, double* comp,
                               int* iters, int* done) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nprob) return;
  const PcgState* st = D[i].st;
  res[i] = st->res;
  iters[i] = st->iter;
  done[i] = st->done;
  comp[i] = scal[i][2];
}

}  // namespace edge
