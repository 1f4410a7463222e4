// Element-wise and reduction kernels of the SIMP loop: layout conversion, density
// filter and its transpose, SIMP material law, element sensitivities, compliance,
// OC bisection, PCG vector updates.
#pragma once
#include "common.cuh"
#include "element_op.cuh"

namespace edge {

// ------------------------------------------------------------------ layout conversion
// User vectors are the reference's interleaved node-major arrays: v[node*dof + c] with
// node = j*nx*nz + i*nz + k (3-D) or j*nx + i (2-D).
EDGE_D bool node_of_slot(const Geo& g, long long s, int& i, int& j, int& k, long long& node) {
  if (g.dim == 3) {
    k = (int)(s % g.pz);
    i = (int)((s / g.pz) % g.nx);
    j = (int)(s / g.plane);
    if (k >= g.nz) return false;
    node = ((long long)j * g.nx + i) * g.nz + k;
  } else {
    k = 0;
    i = (int)(s % g.pz);
    j = (int)(s / g.pz);
    if (i >= g.nx) return false;
    node = (long long)j * g.nx + i;
  }
  return true;
}

template <typename TO>
__global__ void k_user_to_slots(const Geo g, const double* __restrict__ user, TO* __restrict__ v) {
  EDGE_PDL_ENTRY();
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= g.n) return;
  int i, j, k;
  long long node;
  const bool ok = node_of_slot(g, s, i, j, k, node);
  for (int c = 0; c < g.dof; ++c) v[c * g.n + s] = Conv<TO>::from(ok ? user[node * g.dof + c] : 0.0);
}

template <typename TI>
__global__ void k_slots_to_user(const Geo g, const TI* __restrict__ v, double* __restrict__ user) {
  EDGE_PDL_ENTRY();
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= g.n) return;
  int i, j, k;
  long long node;
  if (!node_of_slot(g, s, i, j, k, node)) return;
  for (int c = 0; c < g.dof; ++c) user[node * g.dof + c] = (double)Conv<double>::from(v[c * g.n + s]);
}

// Per-node constraint bits from the reference's per-DOF boolean array.
__global__ void k_mask_from_user(const Geo g, const uint8_t* __restrict__ cons, uint8_t* __restrict__ mask) {
  EDGE_PDL_ENTRY();
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= g.n) return;
  int i, j, k;
  long long node;
  uint8_t m = 0;
  if (node_of_slot(g, s, i, j, k, node))
    for (int c = 0; c < g.dof; ++c) m |= (cons[node * g.dof + c] ? 1 : 0) << c;
  mask[s] = m;
}

// Element constraint flags with rows padded to 16 bytes (the TMA source of the fine
// kernel): f(i,j,k) = 1 if any existing corner (i+a, j+b, k+c), a,b,c in {0,1}, of the
// element slot has a constrained DOF.  Slots past the last element (ghosts) are flagged
// from their existing corners, so f(i,j,k) always covers node (i,j,k) itself.
__global__ void k_flag_pitch16(const Geo g, const uint8_t* __restrict__ mask, uint8_t* __restrict__ f16, int mpz) {
  EDGE_PDL_ENTRY();
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= g.n) return;
  int i, j, k;
  long long node;
  if (!node_of_slot(g, s, i, j, k, node)) return;
  uint8_t f = 0;
  for (int b = 0; b < 8; ++b) {
    const int ii = i + (b & 1), jj = j + ((b >> 1) & 1), kk = k + ((b >> 2) & 1);
    if (ii < g.nx && jj < g.ny && kk < g.nz) f |= mask[g.slot3(ii, jj, kk)];
  }
  f16[((long long)j * g.nx + i) * mpz + k] = f ? 1 : 0;
}

// Element arrays: user order e = i*nely*nelz + j*nelz + k (3-D), i*nely + j (2-D)
// (core/_geom.py:17-18, 43-46) <-> node-aligned slots.
EDGE_D long long user_elem(const Geo& g, int i, int j, int k) {
  const int nely = g.ny - 1;
  if (g.dim == 3) return ((long long)i * nely + j) * (g.nz - 1) + k;
  return (long long)i * nely + j;
}

template <typename TO>
__global__ void k_elem_user_to_slots(const Geo g, const double* __restrict__ user, TO* __restrict__ v) {
  EDGE_PDL_ENTRY();
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= g.n) return;
  int i, j, k;
  long long node;
  double val = 0.0;
  if (node_of_slot(g, s, i, j, k, node) && i < g.nx - 1 && j < g.ny - 1 && (g.dim == 2 || k < g.nz - 1))
    val = user[user_elem(g, i, j, k)];
  v[s] = Conv<TO>::from(val);
}

// A real grid embedded in the lower corner of a larger (padded) grid g: gr holds the real
// grid's node counts.  The user arrays are the real grid's (its own numbering); slots of g
// outside the real grid read zero and are not written back.
EDGE_D bool real_node_of_slot(const Geo& g, const Geo& gr, long long s, int& i, int& j, int& k, long long& node) {
  long long np;
  if (!node_of_slot(g, s, i, j, k, np)) return false;
  if (i >= gr.nx || j >= gr.ny || (g.dim == 3 && k >= gr.nz)) return false;
  node = g.dim == 3 ? ((long long)j * gr.nx + i) * gr.nz + k : (long long)j * gr.nx + i;
  return true;
}
template <typename TO>
__global__ void k_user_to_slots_emb(const Geo g, const Geo gr, const double* __restrict__ user, TO* __restrict__ v) {
  EDGE_PDL_ENTRY();
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= g.n) return;
  int i, j, k;
  long long node;
  const bool ok = real_node_of_slot(g, gr, s, i, j, k, node);
  for (int c = 0; c < g.dof; ++c) v[c * g.n + s] = Conv<TO>::from(ok ? user[node * g.dof + c] : 0.0);
}
template <typename TI>
__global__ void k_slots_to_user_emb(const Geo g, const Geo gr, const TI* __restrict__ v, double* __restrict__ user) {
  EDGE_PDL_ENTRY();
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= g.n) return;
  int i, j, k;
  long long node;
  if (!real_node_of_slot(g, gr, s, i, j, k, node)) return;
  for (int c = 0; c < g.dof; ++c) user[node * g.dof + c] = (double)Conv<double>::from(v[c * g.n + s]);
}
// Element array of the real grid (the reference's element order) into g's slots; padding
// elements (and slots without an element) get zero.
template <typename TO>
__global__ void k_elem_user_to_slots_emb(const Geo g, const Geo gr, const double* __restrict__ user,
                                         TO* __restrict__ v) {
  EDGE_PDL_ENTRY();
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= g.n) return;
  int i, j, k;
  long long node;
  double val = 0.0;
  if (node_of_slot(g, s, i, j, k, node) && i < gr.nx - 1 && j < gr.ny - 1 && (g.dim == 2 || k < gr.nz - 1))
    val = user[user_elem(gr, i, j, k)];
  v[s] = Conv<TO>::from(val);
}

// ------------------------------------------------------------------ density filter
// Cone filter (geom/_filters.py:72-161, core/_filter.py:78-124): taps o_k with global
// weights w_k; (H rho)_e = sum_k w_k rho_{e+o_k} / sum_{in-bounds k} w_k.
constexpr int MAX_TAPS = 128;
struct Taps {
  int n;
  int off[MAX_TAPS][3];  // (dx, dy, dz) in element units
  double w[MAX_TAPS];
};

// Forward filter fused with the SIMP law (MaterialModels.py:47-60):
//   rho_f = H rho (user order), E = clip(rho_f^p, void, 1) written in slot layout
//   (types TE1 and optional TE2 for a second precision).
template <typename TE1, typename TE2>
__global__ void k_filter_material(const Geo g, const Taps taps, const double* __restrict__ rho,
                                  double* __restrict__ rho_f, TE1* __restrict__ E1, TE2* __restrict__ E2,
                                  double penalty, double vmin, int plain) {
  EDGE_PDL_ENTRY();
  const int nelx = g.nx - 1, nely = g.ny - 1, nelz = g.dim == 3 ? g.nz - 1 : 1;
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nel = (long long)nelx * nely * nelz;
  if (e >= nel) return;
  int i, j, k;
  if (g.dim == 3) {
    k = (int)(e % nelz);
    j = (int)((e / nelz) % nely);
    i = (int)(e / ((long long)nelz * nely));
  } else {
    k = 0;
    j = (int)(e % nely);
    i = (int)(e / nely);
  }
  double sv = 0.0, sw = 0.0;
  for (int t = 0; t < taps.n; ++t) {
    const int ii = i + taps.off[t][0], jj = j + taps.off[t][1], kk = k + taps.off[t][2];
    if (ii < 0 || ii >= nelx || jj < 0 || jj >= nely || kk < 0 || kk >= nelz) continue;
    const double w = taps.w[t];
    sv += w * __ldg(rho + user_elem(g, ii, jj, kk));
    sw += w;
  }
  const double rf = sw > 0.0 ? sv / sw : 0.0;
  rho_f[e] = rf;
  double Ev;
  if (plain) {
    Ev = fmin(fmax(rf, vmin), 1.0);
  } else {
    Ev = fmin(fmax(pow(rf, penalty), vmin), 1.0);
  }
  const long long s = g.dim == 3 ? g.slot3(i, j, k) : g.slot2(i, j);
  E1[s] = Conv<TE1>::from(Ev);
  if (E2) E2[s] = Conv<TE2>::from(Ev);
}

// Filter only (H rho), user order in and out.
__global__ void k_filter(const Geo g, const Taps taps, const double* __restrict__ in, double* __restrict__ out) {
  EDGE_PDL_ENTRY();
  const int nelx = g.nx - 1, nely = g.ny - 1, nelz = g.dim == 3 ? g.nz - 1 : 1;
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nel = (long long)nelx * nely * nelz;
  if (e >= nel) return;
  int i, j, k;
  if (g.dim == 3) {
    k = (int)(e % nelz);
    j = (int)((e / nelz) % nely);
    i = (int)(e / ((long long)nelz * nely));
  } else {
    k = 0;
    j = (int)(e % nely);
    i = (int)(e / nely);
  }
  double sv = 0.0, sw = 0.0;
  for (int t = 0; t < taps.n; ++t) {
    const int ii = i + taps.off[t][0], jj = j + taps.off[t][1], kk = k + taps.off[t][2];
    if (ii < 0 || ii >= nelx || jj < 0 || jj >= nely || kk < 0 || kk >= nelz) continue;
    sv += taps.w[t] * __ldg(in + user_elem(g, ii, jj, kk));
    sw += taps.w[t];
  }
  out[e] = sw > 0.0 ? sv / sw : 0.0;
}

// Normaliser N_e = sum of in-bounds weights (core/_filter.py:6-40).
__global__ void k_filter_norm(const Geo g, const Taps taps, double* __restrict__ N) {
  EDGE_PDL_ENTRY();
  const int nelx = g.nx - 1, nely = g.ny - 1, nelz = g.dim == 3 ? g.nz - 1 : 1;
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nel = (long long)nelx * nely * nelz;
  if (e >= nel) return;
  int i, j, k;
  if (g.dim == 3) {
    k = (int)(e % nelz);
    j = (int)((e / nelz) % nely);
    i = (int)(e / ((long long)nelz * nely));
  } else {
    k = 0;
    j = (int)(e % nely);
    i = (int)(e / nely);
  }
  double sw = 0.0;
  for (int t = 0; t < taps.n; ++t) {
    const int ii = i + taps.off[t][0], jj = j + taps.off[t][1], kk = k + taps.off[t][2];
    if (ii < 0 || ii >= nelx || jj < 0 || jj >= nely || kk < 0 || kk >= nelz) continue;
    sw += taps.w[t];
  }
  N[e] = sw;
}

// Transpose: (H^T v)_e = sum_k (w_k / N_{e+o_k}) v_{e+o_k} (core/_filter.py:42-76).
__global__ void k_filter_T(const Geo g, const Taps taps, const double* __restrict__ N, const double* __restrict__ in,
                           double* __restrict__ out) {
  EDGE_PDL_ENTRY();
  const int nelx = g.nx - 1, nely = g.ny - 1, nelz = g.dim == 3 ? g.nz - 1 : 1;
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nel = (long long)nelx * nely * nelz;
  if (e >= nel) return;
  int i, j, k;
  if (g.dim == 3) {
    k = (int)(e % nelz);
    j = (int)((e / nelz) % nely);
    i = (int)(e / ((long long)nelz * nely));
  } else {
    k = 0;
    j = (int)(e % nely);
    i = (int)(e / nely);
  }
  double sv = 0.0;
  for (int t = 0; t < taps.n; ++t) {
    const int ii = i + taps.off[t][0], jj = j + taps.off[t][1], kk = k + taps.off[t][2];
    if (ii < 0 || ii >= nelx || jj < 0 || jj >= nely || kk < 0 || kk >= nelz) continue;
    const long long q = user_elem(g, ii, jj, kk);
    sv += (taps.w[t] / __ldg(N + q)) * __ldg(in + q);
  }
  out[e] = sv;
}

// ------------------------------------------------------------------ sensitivities
// dk_e = -u_e^T K0 u_e (core/_ops.py:5-13) from the solution in slot layout, and
// optionally g_e = p clip(rho_f, void, 1)^(p-1) dk_e (MaterialModels.py:62-73).
// `wht` selects the transform form; otherwise K0b (bit-order dense) is used.
template <typename TU>
__global__ void k_dk(const Geo g, const TU* __restrict__ U, KHat3<double> K3, KHat2<double> K2,
                     const double* __restrict__ K0b, int wht, double* __restrict__ dk, const double* __restrict__ rho_f,
                     double* __restrict__ gout, double penalty, double vmin) {
  EDGE_PDL_ENTRY();
  const int nelx = g.nx - 1, nely = g.ny - 1, nelz = g.dim == 3 ? g.nz - 1 : 1;
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nel = (long long)nelx * nely * nelz;
  if (e >= nel) return;
  double val;
  if (g.dim == 3) {
    const int k = (int)(e % nelz), j = (int)((e / nelz) % nely), i = (int)(e / ((long long)nelz * nely));
    double u[8][3];
    for (int b = 0; b < 8; ++b) {
      const long long s = g.slot3(i + (b & 1), j + ((b >> 1) & 1), k + ((b >> 2) & 1));
      for (int c = 0; c < 3; ++c) u[b][c] = (double)Conv<double>::from(U[c * g.n + s]);
    }
    if (wht) {
      val = -elem3_energy(K3, u);
    } else {
      double acc = 0.0;
      for (int r = 0; r < 24; ++r) {
        double t = 0.0;
        for (int q = 0; q < 24; ++q) t += K0b[r * 24 + q] * u[q / 3][q % 3];
        acc += u[r / 3][r % 3] * t;
      }
      val = -acc;
    }
  } else {
    const int j = (int)(e % nely), i = (int)(e / nely);
    double u[4][2];
    for (int b = 0; b < 4; ++b) {
      const long long s = g.slot2(i + (b & 1), j + ((b >> 1) & 1));
      for (int c = 0; c < 2; ++c) u[b][c] = (double)Conv<double>::from(U[c * g.n + s]);
    }
    if (wht) {
      val = -elem2_energy(K2, u);
    } else {
      double acc = 0.0;
      for (int r = 0; r < 8; ++r) {
        double t = 0.0;
        for (int q = 0; q < 8; ++q) t += K0b[r * 8 + q] * u[q / 2][q % 2];
        acc += u[r / 2][r % 2] * t;
      }
      val = -acc;
    }
  }
  if (dk) dk[e] = val;
  if (gout) gout[e] = penalty * pow(fmin(fmax(rho_f[e], vmin), 1.0), penalty - 1.0) * val;
}

// Fine diagonal of K(E) with BCs (core/_ops.py:45-76): sum over the node's elements of
// E_e K0[(a,c),(a,c)], 1 on constrained DOFs; writes Dinv = 1/diag in type TD.
template <typename TE, typename TD>
__global__ void k_fine_dinv(const Geo g, const TE* __restrict__ E, const uint8_t* __restrict__ mask,
                            const double* __restrict__ K0diag /* [corner][c] bit order */, TD* __restrict__ dinv,
                            double* __restrict__ diag_out) {
  EDGE_PDL_ENTRY();
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= g.n) return;
  int i, j, k;
  long long node;
  const bool ok = node_of_slot(g, s, i, j, k, node);
  const int dof = g.dof;
  double d[3] = {0, 0, 0};
  if (ok) {
    const int nc = g.dim == 3 ? 8 : 4;
    for (int a = 0; a < nc; ++a) {
      const int li = i - (a & 1), lj = j - ((a >> 1) & 1), lk = k - ((a >> 2) & 1);
      if (li < 0 || lj < 0 || li >= g.nx - 1 || lj >= g.ny - 1) continue;
      if (g.dim == 3 && (lk < 0 || lk >= g.nz - 1)) continue;
      const double Ee = (double)Conv<double>::from(E[g.dim == 3 ? g.slot3(li, lj, lk) : g.slot2(li, lj)]);
      for (int c = 0; c < dof; ++c) d[c] += Ee * K0diag[a * dof + c];
    }
    const uint8_t m = mask[s];
    for (int c = 0; c < dof; ++c)
      if ((m >> c) & 1) d[c] = 1.0;
  }
  for (int c = 0; c < dof; ++c) {
    dinv[c * g.n + s] = Conv<TD>::from(ok ? 1.0 / d[c] : 0.0);
    if (diag_out && ok) diag_out[node * dof + c] = d[c];
  }
}

// ------------------------------------------------------------------ reductions
template <typename TA, typename TB>
__global__ void k_dot(long long n, const TA* __restrict__ a, const TB* __restrict__ b, double* part, unsigned* ticket,
                      double* dst) {
  EDGE_PDL_ENTRY();
  double acc = 0.0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    acc += (double)Conv<double>::from(a[q]) * (double)Conv<double>::from(b[q]);
  __shared__ double sh[32];
  double bt = block_sum(acc, sh);
  grid_reduce_finish(bt, part, ticket, DotSink{dst});
}

// ------------------------------------------------------------------ PCG device scalars
struct PcgState {
  double rz;      // r.z used by the current iteration's alpha / beta
  double rz_new;  // r.z of the latest V-cycle
  double pq;      // p.(A p)
  double rr;      // r.r
  double bb;      // f.f
  double alpha, beta;
  double res;     // ||r|| / ||f||
  double omega;   // smoother weight for the next V-cycle
  double tol, min_omega, d_omega;
  double last_replace;      // ||r||/||f|| at the last true-residual replacement (mixed precision)
  int iter, maxiter, done;  // done: 1 converged, 2 maxiter
  int n_true;               // replacements made inside the iteration loop
  // residual update folded into the next iteration's first fine launch (mixed path): pend =
  // a search direction's product exists whose update is still to be applied; xa = the alpha
  // of the solution update x32 += alpha p still to be applied (0: none)
  int pend;
  double xa;
};

// x += alpha p ; r -= alpha q ; rr = r.r with alpha = rz_new / pq.  The finisher
// updates res / omega / done as solvers/_multigrid_cuda.py:219-227 and moves rz_new to rz.
// With r32 != nullptr the updated residual is also written in FP32 (the V-cycle input of
// the mixed-precision solver).

// Finisher of the x/r update: new r.r, residual, iteration count, stop reason and the
// next V-cycle's smoother weight (solvers/_multigrid_cuda.py:219-227).
struct PcgXrFin {
  PcgState* st;
  double alpha;
  EDGE_D void operator()(double t) const {
    st->alpha = alpha;
    st->rz = st->rz_new;
    st->rr = t;
    const double R = sqrt(t) / sqrt(st->bb);
    st->res = R;
    st->iter += 1;
    if (R < st->tol) {
      st->done = 1;
    } else {
      const double Rc = fmin(fmax(R, st->tol), 1e-1);
      st->omega = st->min_omega + st->d_omega / 2.0 * exp((-Rc + st->tol) * 500.0);
      if (st->iter >= st->maxiter) st->done = 2;
    }
  }
};

template <typename TX, typename TP>
__global__ void k_pcg_xr(long long n, TX* __restrict__ x, const TP* __restrict__ p, TX* __restrict__ r,
                         const TP* __restrict__ q, PcgState* st, double* part, unsigned* ticket,
                         float* __restrict__ r32) {
  EDGE_PDL_ENTRY();
  using X2 = typename V2<TX>::type;
  using P2v = typename V2<TP>::type;
  const double alpha = st->rz_new / st->pq;
  double acc = 0.0;
  const long long n2 = n >> 1;
  X2* __restrict__ x2 = reinterpret_cast<X2*>(x);
  X2* __restrict__ r2 = reinterpret_cast<X2*>(r);
  const P2v* __restrict__ p2 = reinterpret_cast<const P2v*>(p);
  const P2v* __restrict__ q2 = reinterpret_cast<const P2v*>(q);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n2; i += (long long)gridDim.x * blockDim.x) {
    const P2v pv = p2[i], qv = q2[i];
    X2 xv = x2[i], rv = r2[i];
    xv.x = Conv<TX>::from((double)xv.x + alpha * (double)pv.x);
    xv.y = Conv<TX>::from((double)xv.y + alpha * (double)pv.y);
    const double r0 = (double)rv.x - alpha * (double)qv.x, r1 = (double)rv.y - alpha * (double)qv.y;
    rv.x = Conv<TX>::from(r0);
    rv.y = Conv<TX>::from(r1);
    x2[i] = xv;
    r2[i] = rv;
    if (r32) reinterpret_cast<float2*>(r32)[i] = make_float2((float)r0, (float)r1);
    acc += r0 * r0 + r1 * r1;
  }
  if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {  // odd length (not produced by this library)
    const long long i = n - 1;
    x[i] = Conv<TX>::from((double)x[i] + alpha * (double)p[i]);
    const double ri = (double)r[i] - alpha * (double)q[i];
    r[i] = Conv<TX>::from(ri);
    if (r32) r32[i] = (float)ri;
    acc += ri * ri;
  }
  __shared__ double sh[32];
  double bt = block_sum(acc, sh);
  grid_reduce_finish(bt, part, ticket, PcgXrFin{st, alpha});
}

// Mixed precision: the same update with the solution kept as an FP32 increment since the last
// residual replacement (x32 += alpha p); the FP64 solution is only touched when k_fold_x adds
// the increment in, before every true residual and at the end of the solve.  This variant
// keeps an FP64 residual recurrence (edge_set_residual32(0)); k_pcg_xr32 is the default.
__global__ void k_pcg_xr_lag(long long n, float* __restrict__ x32, const float* __restrict__ p,
                             double* __restrict__ r, const float* __restrict__ q, PcgState* st, double* part,
                             unsigned* ticket, float* __restrict__ r32) {
  EDGE_PDL_ENTRY();
  const double alpha = st->rz_new / st->pq;
  const float af = (float)alpha;
  double acc = 0.0;
  const long long n2 = n >> 1;
  float2* __restrict__ x2 = reinterpret_cast<float2*>(x32);
  double2* __restrict__ r2 = reinterpret_cast<double2*>(r);
  const float2* __restrict__ p2 = reinterpret_cast<const float2*>(p);
  const float2* __restrict__ q2 = reinterpret_cast<const float2*>(q);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n2; i += (long long)gridDim.x * blockDim.x) {
    const float2 pv = p2[i], qv = q2[i];
    float2 xv = x2[i];
    double2 rv = r2[i];
    xv.x += af * pv.x;
    xv.y += af * pv.y;
    rv.x -= alpha * (double)qv.x;
    rv.y -= alpha * (double)qv.y;
    x2[i] = xv;
    r2[i] = rv;
    reinterpret_cast<float2*>(r32)[i] = make_float2((float)rv.x, (float)rv.y);
    acc += rv.x * rv.x + rv.y * rv.y;
  }
  if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
    const long long i = n - 1;
    x32[i] += af * p[i];
    r[i] -= alpha * (double)q[i];
    r32[i] = (float)r[i];
    acc += r[i] * r[i];
  }
  __shared__ double sh[32];
  double bt = block_sum(acc, sh);
  grid_reduce_finish(bt, part, ticket, PcgXrFin{st, alpha});
}

// Mixed precision with an FP32 residual recurrence between the FP64 replacements ("reliable
// updates": the recurrence only has to stay accurate relative to the residual at the last
// replacement, which is at most 100 times the current one): x32 += alpha p, r32 -= alpha q
// as FP32 fused multiply-adds with alpha rounded to FP32, 16-byte accesses, r.r summed per
// four values in FP32 and accumulated in FP64.
//
// p1 != null: p is one of a ping-pong pair, the one the fused product of this iteration wrote
// (iteration parity 0: p1, parity 1: p0).
__global__ void k_pcg_xr32(long long n, float* __restrict__ x32, const float* __restrict__ p0,
                           const float* __restrict__ p1, float* __restrict__ r32, const float* __restrict__ q,
                           PcgState* st, double* part, unsigned* ticket) {
  EDGE_PDL_ENTRY();
  const float* __restrict__ p = (p1 != nullptr && (st->iter & 1) == 0) ? p1 : p0;
  const double alpha = st->rz_new / st->pq;
  const float af = (float)alpha;
  double acc = 0.0;
  const long long n4 = n >> 2;
  float4* __restrict__ x4 = reinterpret_cast<float4*>(x32);
  float4* __restrict__ r4 = reinterpret_cast<float4*>(r32);
  const float4* __restrict__ p4 = reinterpret_cast<const float4*>(p);
  const float4* __restrict__ q4 = reinterpret_cast<const float4*>(q);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
    const float4 pv = p4[i], qv = q4[i];
    float4 xv = x4[i], rv = r4[i];
    xv.x = fmaf(af, pv.x, xv.x);
    xv.y = fmaf(af, pv.y, xv.y);
    xv.z = fmaf(af, pv.z, xv.z);
    xv.w = fmaf(af, pv.w, xv.w);
    rv.x = fmaf(-af, qv.x, rv.x);
    rv.y = fmaf(-af, qv.y, rv.y);
    rv.z = fmaf(-af, qv.z, rv.z);
    rv.w = fmaf(-af, qv.w, rv.w);
    x4[i] = xv;
    r4[i] = rv;
    acc += (double)(rv.x * rv.x + rv.y * rv.y + rv.z * rv.z + rv.w * rv.w);
  }
  if (blockIdx.x == 0 && threadIdx.x < (n & 3)) {  // tail (lengths here are multiples of 4)
    const long long i = 4 * n4 + threadIdx.x;
    x32[i] = fmaf(af, p[i], x32[i]);
    r32[i] = fmaf(-af, q[i], r32[i]);
    acc += (double)r32[i] * (double)r32[i];
  }
  __shared__ double sh[32];
  double bt = block_sum(acc, sh);
  grid_reduce_finish(bt, part, ticket, PcgXrFin{st, alpha});
}

// The pending solution update of the fused residual update (st->xa != 0): x32 += xa p with the
// search direction of the previous iteration (the p buffer k_pcg_xr32 would have read then),
// applied before the solution is folded into FP64 or the solve ends; FP32, k_pcg_xr32's
// arithmetic.
__global__ void k_x32_pend(long long n, float* __restrict__ x32, const float* __restrict__ p0,
                           const float* __restrict__ p1, const PcgState* st) {
  EDGE_PDL_ENTRY();
  const float af = (float)st->xa;
  if (af == 0.f) return;
  const float* __restrict__ p = (st->iter & 1) ? p1 : p0;
  const long long n4 = n >> 2;
  float4* __restrict__ x4 = reinterpret_cast<float4*>(x32);
  const float4* __restrict__ p4 = reinterpret_cast<const float4*>(p);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
    const float4 pv = p4[i];
    float4 xv = x4[i];
    xv.x = fmaf(af, pv.x, xv.x);
    xv.y = fmaf(af, pv.y, xv.y);
    xv.z = fmaf(af, pv.z, xv.z);
    xv.w = fmaf(af, pv.w, xv.w);
    x4[i] = xv;
  }
  if (blockIdx.x == 0 && threadIdx.x < (n & 3)) {
    const long long i = 4 * n4 + threadIdx.x;
    x32[i] = fmaf(af, p[i], x32[i]);
  }
}

// FP32 copy of the replaced residual into the buffer of the ping-pong pair that holds the
// current residual (st->iter's parity).
__global__ void k_r32_par(long long n, const double* __restrict__ r, float* __restrict__ R0, float* __restrict__ R1,
                          const PcgState* st) {
  EDGE_PDL_ENTRY();
  float* __restrict__ o = (st->iter & 1) ? R1 : R0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    o[i] = (float)r[i];
}

// x64 += x32, x32 = 0
__global__ void k_fold_x(long long n, double* __restrict__ x, float* __restrict__ x32) {
  EDGE_PDL_ENTRY();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    x[i] += (double)x32[i];
    x32[i] = 0.f;
  }
}

// Residual replacement: st->rr holds the TRUE residual r.r (b - A x in FP64).  Decides
// convergence on it; otherwise the iteration continues with the replaced residual.
__global__ void k_pcg_true_res(PcgState* st) {
  EDGE_PDL_ENTRY();
  const double R = sqrt(st->rr) / sqrt(st->bb);
  st->res = R;
  st->last_replace = R;
  st->n_true += 1;
  st->xa = 0.0;  // a pending solution update was applied before the replacement
  if (R < st->tol) {
    st->done = 1;
  } else {
    st->done = (st->iter >= st->maxiter) ? 2 : 0;
    const double Rc = fmin(fmax(R, st->tol), 1e-1);
    st->omega = st->min_omega + st->d_omega / 2.0 * exp((-Rc + st->tol) * 500.0);
  }
}

// p = z + beta p, or p = z before the first iteration (iter == 0)
template <typename TP>
__global__ void k_pcg_p(long long n, TP* __restrict__ p, const TP* __restrict__ z, const PcgState* st) {
  EDGE_PDL_ENTRY();
  using P2v = typename V2<TP>::type;
  const bool first = st->iter == 0;
  const double beta = first ? 0.0 : st->rz_new / st->rz;
  const long long n2 = n >> 1;
  P2v* __restrict__ p2 = reinterpret_cast<P2v*>(p);
  const P2v* __restrict__ z2 = reinterpret_cast<const P2v*>(z);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n2; i += (long long)gridDim.x * blockDim.x) {
    const P2v zv = z2[i];
    if (first) {
      p2[i] = zv;
    } else {
      P2v pv = p2[i];
      pv.x = Conv<TP>::from((double)zv.x + beta * (double)pv.x);
      pv.y = Conv<TP>::from((double)zv.y + beta * (double)pv.y);
      p2[i] = pv;
    }
  }
  if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
    const long long i = n - 1;
    p[i] = first ? z[i] : Conv<TP>::from((double)z[i] + beta * (double)p[i]);
  }
}

// Unpreconditioned CG as PCG with z = r: r.z of the current residual is its r.r.
__global__ void k_cg_rz(PcgState* st) {
  EDGE_PDL_ENTRY(); st->rz_new = st->rr; }
// Report the true relative residual ||f - A x|| / ||f|| (st->rr holds the true r.r).
__global__ void k_final_res(PcgState* st) {
  EDGE_PDL_ENTRY(); st->res = st->bb > 0.0 ? sqrt(st->rr) / sqrt(st->bb) : 0.0; }

// FEA_integrals (TopOpt/_solver.py:80-137 with the structured kernel of core/_ops.py:1032-1058):
// per element, strain = B u_e, stress = D strain (D unscaled, as in the reference), strain
// energy = 1/2 w_e u_e^T K0 u_e.  u_e is gathered from the user-layout displacement in the
// reference's corner order (core/_geom.py:20-57); B (nb x nk), D (nb x nb) and K0 (nk x nk) are
// row-major in that order.  One thread per element (a post-processing call, not a hot path).
__global__ void k_fea_integrals(int dim, int nelx, int nely, int nelz, long long nel, const double* __restrict__ U,
                                const double* __restrict__ w, const double* __restrict__ K0,
                                const double* __restrict__ B, const double* __restrict__ D, int nb,
                                double* __restrict__ strain, double* __restrict__ stress, double* __restrict__ energy) {
  EDGE_PDL_ENTRY();
  const int nc = dim == 3 ? 8 : 4, nk = nc * dim;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nel; e += (long long)gridDim.x * blockDim.x) {
    long long nid[8];
    if (dim == 3) {
      const int i = (int)(e / ((long long)nely * nelz)), j = (int)((e / nelz) % nely), k = (int)(e % nelz);
      const long long nx = nelx + 1, nz = nelz + 1;
      auto node = [&](int a, int b, int c) { return (long long)b * nx * nz + (long long)a * nz + c; };
      nid[0] = node(i, j, k);
      nid[1] = node(i + 1, j, k);
      nid[2] = node(i + 1, j + 1, k);
      nid[3] = node(i, j + 1, k);
      nid[4] = node(i, j, k + 1);
      nid[5] = node(i + 1, j, k + 1);
      nid[6] = node(i + 1, j + 1, k + 1);
      nid[7] = node(i, j + 1, k + 1);
    } else {
      const int i = (int)(e / nely), j = (int)(e % nely);
      const long long nx = nelx + 1;
      nid[0] = (long long)j * nx + i;
      nid[1] = (long long)j * nx + i + 1;
      nid[2] = (long long)(j + 1) * nx + i + 1;
      nid[3] = (long long)(j + 1) * nx + i;
    }
    double u[24];
    for (int m = 0; m < nk; ++m) u[m] = U[nid[m / dim] * dim + m % dim];
    double eps[6];
    for (int b = 0; b < nb; ++b) {
      double a = 0.0;
      for (int m = 0; m < nk; ++m) a += B[b * nk + m] * u[m];
      eps[b] = a;
      strain[e * nb + b] = a;
    }
    for (int b = 0; b < nb; ++b) {
      double a = 0.0;
      for (int c = 0; c < nb; ++c) a += D[b * nb + c] * eps[c];
      stress[e * nb + b] = a;
    }
    double en = 0.0;
    for (int m = 0; m < nk; ++m) {
      double a = 0.0;
      for (int n2 = 0; n2 < nk; ++n2) a += K0[m * nk + n2] * u[n2];
      en += u[m] * a;
    }
    energy[e] = 0.5 * w[e] * en;
  }
}

// Loop control of the graph-captured PCG: the while node repeats while no stop reason is set;
// the if node (mixed precision) computes a true residual when the recurrence has converged
// or has dropped by `drop` since the last replacement.
__global__ void k_cond_while(cudaGraphConditionalHandle h, const PcgState* st) {
  EDGE_PDL_ENTRY();
  cudaGraphSetConditional(h, st->done == 0 ? 1u : 0u);
}
__global__ void k_cond_replace(cudaGraphConditionalHandle h, const PcgState* st, double drop) {
  EDGE_PDL_ENTRY();
  cudaGraphSetConditional(h, (st->done == 1 || st->res < drop * st->last_replace) ? 1u : 0u);
}
// The same test with the residual update fused into the iteration's first launch: only once a
// residual update has been applied (not in the first iteration, whose residual is the
// prologue's true residual).
EDGE_HD bool replace_due_xr(const PcgState* st, double drop) {
  return st->pend && (st->done == 1 || st->res < drop * st->last_replace);
}
__global__ void k_cond_replace_xr(cudaGraphConditionalHandle h, const PcgState* st, double drop) {
  EDGE_PDL_ENTRY();
  cudaGraphSetConditional(h, replace_due_xr(st, drop) ? 1u : 0u);
}
// The rest of the iteration (V-cycle below the first launch, the search direction's product)
// runs while the solve is not done.
__global__ void k_cond_rest(cudaGraphConditionalHandle h, const PcgState* st) {
  EDGE_PDL_ENTRY();
  cudaGraphSetConditional(h, st->done == 0 ? 1u : 0u);
}

// ------------------------------------------------------------------ point springs and adjoint sensitivity
// Grounded springs on single DOFs (the compliant-mechanism input/output springs): in the
// slot layout, out[f] += sign * k * x[f] for every unconstrained spring DOF f = c*n + slot,
// and *dot += sum k x[f]^2 when dot is given (the p.Ap term of PCG).  One block.
template <typename TX, typename TO>
__global__ void k_springs(int ns, const long long* __restrict__ flat, const double* __restrict__ kk, long long n,
                          const uint8_t* __restrict__ mask, const TX* __restrict__ x, TO* __restrict__ out,
                          double sign, double* dot) {
  EDGE_PDL_ENTRY();
  __shared__ double sh[32];
  double acc = 0.0;
  for (int t = threadIdx.x; t < ns; t += blockDim.x) {
    const long long f = flat[t];
    const long long s = f % n;
    const int c = (int)(f / n);
    if ((mask[s] >> c) & 1) continue;
    const double xv = (double)Conv<double>::from(x[f]);
    out[f] = Conv<TO>::from((double)Conv<double>::from(out[f]) + sign * kk[t] * xv);
    acc += kk[t] * xv * xv;
  }
  const double tot = block_sum(acc, sh);
  if (dot && threadIdx.x == 0) *dot += tot;
}

// The springs on the diagonal of K (user layout; constrained DOFs keep their 1).
__global__ void k_springs_diag(int ns, const long long* __restrict__ flat, const long long* __restrict__ user,
                               const double* __restrict__ kk, long long n, const uint8_t* __restrict__ mask,
                               double* __restrict__ diag) {
  EDGE_PDL_ENTRY();
  for (int t = threadIdx.x; t < ns; t += blockDim.x) {
    const long long f = flat[t];
    if ((mask[f % n] >> (int)(f / n)) & 1) continue;
    diag[user[t]] += kk[t];
  }
}

// Adjoint sensitivity of a linear functional: dk_e = -v_e^T K0 u_e, by polarisation of the
// element energy: v^T K0 u = ((u+v)^T K0 (u+v) - (u-v)^T K0 (u-v)) / 4.
__global__ void k_dk2(const Geo g, const double* __restrict__ U, const double* __restrict__ V, KHat3<double> K3,
                      KHat2<double> K2, const double* __restrict__ K0b, int wht, double* __restrict__ dk) {
  EDGE_PDL_ENTRY();
  const int nelx = g.nx - 1, nely = g.ny - 1, nelz = g.dim == 3 ? g.nz - 1 : 1;
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nel = (long long)nelx * nely * nelz;
  if (e >= nel) return;
  double val;
  if (g.dim == 3) {
    const int k = (int)(e % nelz), j = (int)((e / nelz) % nely), i = (int)(e / ((long long)nelz * nely));
    double a[8][3], b[8][3];
    for (int q = 0; q < 8; ++q) {
      const long long s = g.slot3(i + (q & 1), j + ((q >> 1) & 1), k + ((q >> 2) & 1));
      for (int c = 0; c < 3; ++c) {
        const double u = U[c * g.n + s], v = V[c * g.n + s];
        a[q][c] = u + v;
        b[q][c] = u - v;
      }
    }
    if (wht) {
      val = -0.25 * (elem3_energy(K3, a) - elem3_energy(K3, b));
    } else {
      double acc = 0.0;
      for (int r = 0; r < 24; ++r) {
        double t = 0.0;
        for (int q = 0; q < 24; ++q) t += K0b[r * 24 + q] * 0.5 * (a[q / 3][q % 3] + b[q / 3][q % 3]);
        acc += 0.5 * (a[r / 3][r % 3] - b[r / 3][r % 3]) * t;
      }
      val = -acc;
    }
  } else {
    const int j = (int)(e % nely), i = (int)(e / nely);
    double a[4][2], b[4][2];
    for (int q = 0; q < 4; ++q) {
      const long long s = g.slot2(i + (q & 1), j + ((q >> 1) & 1));
      for (int c = 0; c < 2; ++c) {
        const double u = U[c * g.n + s], v = V[c * g.n + s];
        a[q][c] = u + v;
        b[q][c] = u - v;
      }
    }
    if (wht) {
      val = -0.25 * (elem2_energy(K2, a) - elem2_energy(K2, b));
    } else {
      double acc = 0.0;
      for (int r = 0; r < 8; ++r) {
        double t = 0.0;
        for (int q = 0; q < 8; ++q) t += K0b[r * 8 + q] * 0.5 * (a[q / 2][q % 2] + b[q / 2][q % 2]);
        acc += 0.5 * (a[r / 2][r % 2] - b[r / 2][r % 2]) * t;
      }
      val = -acc;
    }
  }
  dk[e] = val;
}

// ------------------------------------------------------------------ OC bisection (TopOpt/_cuda.py:242-280)
// ocP = max(1e-12, rho * sqrt(max(-dr/A, 0))) with NaN -> 0; the all-zero fallback of
// MaterialModels.py:87-88 is applied by k_oc_fallback when sum(ocP_raw) == 0.
__global__ void k_oc_prep(long long n, const double* __restrict__ rho, const double* __restrict__ dr, double A,
                          double* __restrict__ ocp, double* part, unsigned* ticket, double* sum_dst) {
  EDGE_PDL_ENTRY();
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double v = rho[i] * sqrt(fmax(-dr[i] / A, 0.0));
    if (isnan(v)) v = 0.0;
    acc += fabs(v);
    ocp[i] = v;
  }
  __shared__ double sh[32];
  double bt = block_sum(acc, sh);
  grid_reduce_finish(bt, part, ticket, DotSink{sum_dst});
}

__global__ void k_oc_floor(long long n, double* __restrict__ ocp, const double* __restrict__ sum) {
  EDGE_PDL_ENTRY();
  const bool allzero = (*sum == 0.0);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double v = allzero ? 1e-3 : ocp[i];
    ocp[i] = fmax(1e-12, v);
  }
}

constexpr int OC_DEPTH = 4;                  // bisection levels resolved per pass
constexpr int OC_NODES = (1 << OC_DEPTH) - 1;
struct OcState {
  double l1, l2, last;
  double vf, vol;
  int steps, done;
  double sums[OC_NODES];
};

EDGE_D double oc_rho(double r, double o, double lam, double move) {
  const double xU = fmin(fmax(r + move, 0.0), 1.0);
  const double xL = fmin(fmax(r - move, 0.0), 1.0);
  return fmax(0.0, fmax(xL, fmin(1.0, fmin(xU, o / lam))));
}

// Evaluate sum(rho_new(lambda) * A) at every node of the next OC_DEPTH levels of the
// bisection tree.  Tree node t (heap order): children 2t+1 (volume ok -> l2 = mid)
// and 2t+2 (l1 = mid).
__global__ void __launch_bounds__(256) k_oc_pass(long long n, const double* __restrict__ rho, const double* __restrict__ ocp,
                                                 double A, double move, OcState* st, double* part, unsigned* ticket) {
  EDGE_PDL_ENTRY();
  if (st->done) return;
  double lam[OC_NODES];
  {
    double L1[OC_NODES], L2[OC_NODES];
    L1[0] = st->l1;
    L2[0] = st->l2;
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
  double acc[OC_NODES];
  for (int t = 0; t < OC_NODES; ++t) acc[t] = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double r = rho[i], o = ocp[i];
    for (int t = 0; t < OC_NODES; ++t) acc[t] += oc_rho(r, o, lam[t], move) * A;
  }
  __shared__ double sh[32];
  __shared__ double bsum[OC_NODES];
  for (int t = 0; t < OC_NODES; ++t) {
    double v = block_sum(acc[t], sh);
    if (threadIdx.x == 0) bsum[t] = v;
  }
  __syncthreads();
  // grid-wide: partials laid out [block][t]
  __shared__ bool am_last;
  const unsigned nblk = gridDim.x;
  if (threadIdx.x == 0) {
    for (int t = 0; t < OC_NODES; ++t) part[(long long)blockIdx.x * OC_NODES + t] = bsum[t];
    __threadfence();
    am_last = (atomicAdd(ticket, 1u) == nblk - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  for (int t = 0; t < OC_NODES; ++t) {
    double a = 0.0;
    for (unsigned b = threadIdx.x; b < nblk; b += blockDim.x) a += ((volatile double*)part)[(long long)b * OC_NODES + t];
    double tot = block_sum(a, sh);
    if (threadIdx.x == 0) st->sums[t] = tot;
  }
  if (threadIdx.x == 0) {
    // walk the tree exactly as the sequential bisection would
    int t = 0;
    double l1 = st->l1, l2 = st->l2;
    for (int d = 0; d < OC_DEPTH; ++d) {
      if (!((l2 - l1) / (l2 + l1) > 1e-4)) {
        st->done = 1;
        break;
      }
      const double mid = 0.5 * (l1 + l2);
      const bool valid = (st->sums[t] / st->vol <= st->vf);
      if (valid) l2 = mid;
      else l1 = mid;
      st->last = mid;
      st->steps += 1;
      t = 2 * t + (valid ? 1 : 2);
    }
    st->l1 = l1;
    st->l2 = l2;
    if (!((l2 - l1) / (l2 + l1) > 1e-4)) st->done = 1;
    *ticket = 0u;
  }
}

// rho_new at the last lambda tried; also sum((rho_new - rho)^2) for the RMS change.
__global__ void k_oc_final(long long n, const double* __restrict__ rho, const double* __restrict__ ocp, double move,
                           const OcState* st, double* __restrict__ rho_new, double* part, unsigned* ticket,
                           double* chg_dst) {
  EDGE_PDL_ENTRY();
  const double lam = st->last;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double r = rho[i];
    const double v = oc_rho(r, ocp[i], lam, move);
    rho_new[i] = v;
    acc += (v - r) * (v - r);
  }
  __shared__ double sh[32];
  double bt = block_sum(acc, sh);
  grid_reduce_finish(bt, part, ticket, DotSink{chg_dst});
}

// Start state of one OC bisection on the device: bracket [1e-9, 1e9] (TopOpt/_cuda.py:260-261).
__global__ void k_oc_state_init(OcState* st, double vf, double vol) {
  EDGE_PDL_ENTRY();
  OcState init{};
  init.l1 = 1e-9;
  init.l2 = 1e9;
  init.last = 0.5 * (init.l1 + init.l2);
  init.vf = vf;
  init.vol = vol;
  *st = init;
}
// Condition of the OC loop inside a graph: bisect again while the bracket is open and fewer
// than max_steps bisection steps ran (the bound of the host loop).
__global__ void k_cond_oc(cudaGraphConditionalHandle h, const OcState* st, int max_steps) {
  EDGE_PDL_ENTRY();
  cudaGraphSetConditional(h, (st->done == 0 && st->steps < max_steps) ? 1u : 0u);
}

// Multi-material SIMP law (PenalizedMultiMaterial, MaterialModels.py:102-205).  rho is the
// n_el x n_mat row-major design of the reference.  With c_m = clip(rho_m, void, 1),
// a_m = c_m^p and b_m = 1 - a_m:
//   E = max(void, sum_m E_m a_m prod_{k != m} b_k)
//   dE/drho_j = p c_j^(p-1) (E_j prod_{k != j} b_k - sum_{m != j} E_m a_m prod_{k != m, j} b_k)
// (the derivative of the sum before its clip, as the reference's backward), and with
// plain != 0: E = clip(sum_m E_m rho_m, void, 1).  One thread per element.
constexpr int MM_MAX = 8;
struct MMat {
  double e[MM_MAX];
};
__global__ void k_mm_law(long long n_el, int n_mat, const double* __restrict__ rho, MMat Em, double vd, double pen,
                         int plain, double* __restrict__ E, double* __restrict__ dE) {
  EDGE_PDL_ENTRY();
  for (long long el = blockIdx.x * (long long)blockDim.x + threadIdx.x; el < n_el;
       el += (long long)gridDim.x * blockDim.x) {
    const double* r = rho + el * n_mat;
    if (plain) {
      double s = 0.0;
      for (int m = 0; m < n_mat; ++m) s += r[m] * Em.e[m];
      E[el] = fmin(fmax(s, vd), 1.0);
      continue;
    }
    double c[MM_MAX], a[MM_MAX], b[MM_MAX];
    for (int m = 0; m < n_mat; ++m) {
      c[m] = fmin(fmax(r[m], vd), 1.0);
      a[m] = pow(c[m], pen);
      b[m] = 1.0 - a[m];
    }
    double s = 0.0;
    for (int m = 0; m < n_mat; ++m) {
      double t = a[m];
      for (int k = 0; k < n_mat; ++k)
        if (k != m) t *= b[k];
      s += t * Em.e[m];
    }
    E[el] = fmax(s, vd);
    if (dE) {
      for (int j = 0; j < n_mat; ++j) {
        const double dj = pen * pow(c[j], pen - 1.0);
        double g = 0.0;
        for (int i = 0; i < n_mat; ++i) {
          double t = 1.0;
          for (int k = 0; k < n_mat; ++k)
            if (k != j) t *= (k == i) ? a[k] : b[k];
          g += (i == j ? dj : -dj) * t * Em.e[i];
        }
        dE[el * n_mat + j] = g;
      }
    }
  }
}

// OC update of an n_el x ns design with one bisection multiplier per column (the multi-material
// update of TopOpt/_cuda.py:242-280 with PenalizedMultiMaterial's ocP and constraint,
// MaterialModels.py:204-225): every column is bisected while any column's gap
// (l2 - l1) / (l2 + l1) exceeds 1e-4 (np.any); column m is feasible when
// sum_e rho_new[e, m] A_e / vol - mass[m] <= 0, or, with a shared mass (rho_mat given), every
// column is when sum_e sum_m rho_new[e, m] A_e rho_mat[m] / vol <= mass[0].  rho_new is the
// design at the last multipliers tried.  One block: sums in a fixed order, the bisection
// state held alike by every thread, at most 200 steps.
struct MmOcCon {
  int ns, shared;
  double mass[MM_MAX], rm[MM_MAX];
};
__global__ void __launch_bounds__(1024) k_oc_multi(long long n, MmOcCon cn, const double* __restrict__ rho,
                                                   const double* __restrict__ ocp, const double* __restrict__ A,
                                                   int a_per_el, double move, double vol,
                                                   double* __restrict__ rho_new, int* steps_out) {
  EDGE_PDL_ENTRY();
  __shared__ double sh[33];
  const int ns = cn.ns;
  double l1[MM_MAX], l2[MM_MAX], lm[MM_MAX];
  for (int m = 0; m < ns; ++m) {
    l1[m] = 1e-9;
    l2[m] = 1e9;
    lm[m] = 0.5 * (l1[m] + l2[m]);
  }
  int steps = 0;
  for (; steps < 200; ++steps) {
    bool open = false;
    for (int m = 0; m < ns; ++m) open = open || ((l2[m] - l1[m]) / (l2[m] + l1[m]) > 1e-4);
    if (!open) break;
    for (int m = 0; m < ns; ++m) lm[m] = 0.5 * (l1[m] + l2[m]);
    double acc[MM_MAX];
    for (int m = 0; m < ns; ++m) acc[m] = 0.0;
    for (long long e = threadIdx.x; e < n; e += blockDim.x) {
      const double a = A[a_per_el ? e : 0];
      for (int m = 0; m < ns; ++m) acc[m] += oc_rho(rho[e * ns + m], ocp[e * ns + m], lm[m], move) * a;
    }
    double V[MM_MAX];
    for (int m = 0; m < ns; ++m) {
      const double t = block_sum(acc[m], sh);
      __syncthreads();
      if (threadIdx.x == 0) sh[32] = t;
      __syncthreads();
      V[m] = sh[32];
      __syncthreads();
    }
    bool valid[MM_MAX];
    if (cn.shared) {
      double tot = 0.0;
      for (int m = 0; m < ns; ++m) tot += V[m] * cn.rm[m];
      const bool ok = tot / vol <= cn.mass[0];
      for (int m = 0; m < ns; ++m) valid[m] = ok;
    } else {
      for (int m = 0; m < ns; ++m) valid[m] = (V[m] / vol - cn.mass[m]) <= 0.0;
    }
    for (int m = 0; m < ns; ++m) {
      if (valid[m]) l2[m] = lm[m];
      else l1[m] = lm[m];
    }
  }
  for (long long e = threadIdx.x; e < n; e += blockDim.x)
    for (int m = 0; m < ns; ++m) rho_new[e * ns + m] = oc_rho(rho[e * ns + m], ocp[e * ns + m], lm[m], move);
  if (steps_out && threadIdx.x == 0) *steps_out = steps;
}

}  // namespace edge
