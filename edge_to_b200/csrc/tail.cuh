// The coarse end of the mixed-precision V-cycle in one persistent launch, sm_100a.
//
// Below the first coarse level every grid is small (12.8M fine DOFs: level 2 has 70,785
// nodes, levels 3 and 4 9,537 and 1,445, the coarsest 225), so launching one kernel per
// smoothing sweep, residual and transfer leaves the GPU mostly waiting on launch latency and
// kernel tails.  k_vcycle_tail runs the whole cycle from level L0 down to the coarsest
// solve and back up as a sequence of grid-stride stages separated by a grid-wide barrier:
//
//   down, per level l:  x = w_l Dinv b (first sweep from zero) [+ sweeps],
//                       r = b - A x, b_{l+1} = R r (with the next level's first sweep fused)
//   coarsest:           res = Ainv b (dense FP64 inverse, one warp per row)
//   up, per level l:    e = P res_{l+1} [+ sweeps on e], res_l = x + e + w_l Dinv (r - A e)
//
// with the arithmetic of the per-launch kernels (k_jacobi0, k_st3_apply with EpiResid /
// EpiJacobi / EpiJacobiAdd, k_restrict3, k_prolong3, k_coarse_solve: the same operations in
// the same order per node), so the cycle is the multi-launch cycle's.  The stencil is the
// symmetric compact storage of coarse.cuh (123 coefficient arrays), read as FP32 or as the
// BF16 copy.
//
// The launch is cooperative (all blocks co-resident, checked by the runtime), and the grid
// barrier is a generation counter in device memory: the last block to arrive resets the
// count and advances the generation; the others spin on it with a clock bound (2^28 cycles,
// about 0.14 s), after which they record an error flag, stop waiting at every later barrier
// and run to the end, so the kernel always terminates and the host reports the failure.
// Every block passes the same barriers in the same order (no early exit).
#pragma once
#include "coarse.cuh"

namespace edge {

constexpr int TAIL_MAX = 8;  // levels L0 .. L (at most 8)

template <typename TS> struct TailLevel {
  Geo g;
  const TS* S;          // stencil (levels < L)
  const float* dinv;    // Jacobi diagonal
  float *b, *xa, *xb, *r, *ea, *eb, *res;
  double ws;            // 1.06^l (the smoother weight factor of the level)
  int nsm;              // sweeps (pre and post), >= 1
};

template <typename TS> struct TailParams {
  int L0, L;  // smoothed levels L0 .. L-1, coarsest L
  TailLevel<TS> lv[TAIL_MAX];
  const double* Ainv;
  int nd;
  const double* omega;
  unsigned* bar;  // [0] arrival count, [1] generation
  int* err;
};

// Grid-wide barrier with a bounded wait (see the file comment).
EDGE_D void tail_barrier(unsigned* bar, int* err) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = bar + 1;
    const unsigned g0 = *gen;
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u);
    if (arrived == gridDim.x - 1) {
      bar[0] = 0u;
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else if (!*(volatile int*)err) {
      const long long t0 = clock64();
      while (*gen == g0) {
        if (clock64() - t0 > (1LL << 28)) {
          atomicOr(err, 4);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

// (A u) at slot s of a level, in k_st3_apply's order (centre block, then for each upper
// direction the upper neighbour's block and the lower neighbour's transposed block).
template <typename TS>
EDGE_D void tail_stencil(const Geo& g, const TS* __restrict__ S, const float* __restrict__ u, long long s, int i, int j,
                         int k, float Au[3]) {
  const long long n = g.n;
  const float u0 = u[s], u1 = u[n + s], u2 = u[2 * n + s];
  const float c00 = Conv<float>::from(__ldg(S + s)), c01 = Conv<float>::from(__ldg(S + n + s)),
              c02 = Conv<float>::from(__ldg(S + 2 * n + s)), c11 = Conv<float>::from(__ldg(S + 3 * n + s)),
              c12 = Conv<float>::from(__ldg(S + 4 * n + s)), c22 = Conv<float>::from(__ldg(S + 5 * n + s));
  Au[0] = c00 * u0 + c01 * u1 + c02 * u2;
  Au[1] = c01 * u0 + c11 * u1 + c12 * u2;
  Au[2] = c02 * u0 + c12 * u1 + c22 * u2;
#pragma unroll
  for (int nb = 14; nb < 27; ++nb) {
    const int dz = nb % 3 - 1, dx = (nb / 3) % 3 - 1, dy = nb / 9 - 1;
    const long long off = (long long)dy * g.plane + (long long)dx * g.pz + dz;
    const TS* Sb = S + (long long)(6 + (nb - 14) * 9) * n;
    if (i + dx >= 0 && i + dx < g.nx && j + dy >= 0 && j + dy < g.ny && k + dz >= 0 && k + dz < g.nz) {
      const long long sn = s + off;
      const float v0 = u[sn], v1 = u[n + sn], v2 = u[2 * n + sn];
#pragma unroll
      for (int c = 0; c < 3; ++c)
        Au[c] += Conv<float>::from(__ldg(Sb + (c * 3 + 0) * n + s)) * v0 +
                 Conv<float>::from(__ldg(Sb + (c * 3 + 1) * n + s)) * v1 +
                 Conv<float>::from(__ldg(Sb + (c * 3 + 2) * n + s)) * v2;
    }
    if (i - dx >= 0 && i - dx < g.nx && j - dy >= 0 && j - dy < g.ny && k - dz >= 0 && k - dz < g.nz) {
      const long long sm = s - off;
      const float v0 = u[sm], v1 = u[n + sm], v2 = u[2 * n + sm];
#pragma unroll
      for (int c = 0; c < 3; ++c)
        Au[c] += Conv<float>::from(__ldg(Sb + (0 * 3 + c) * n + sm)) * v0 +
                 Conv<float>::from(__ldg(Sb + (1 * 3 + c) * n + sm)) * v1 +
                 Conv<float>::from(__ldg(Sb + (2 * 3 + c) * n + sm)) * v2;
    }
  }
}

// the restricted value of coarse node (I, J, K) for all components (k_restrict3's order)
EDGE_D void tail_restrict(const Geo& gf, const Geo& gc, const float* __restrict__ in, int I, int J, int K, float v[3]) {
  const int nb = is_bnd(I, gc.nx) + is_bnd(J, gc.ny) + is_bnd(K, gc.nz);
  const bool zm = K >= 1, zp = 2 * K + 1 < gf.nz;
  v[0] = v[1] = v[2] = 0.f;
#pragma unroll
  for (int di = -1; di <= 1; ++di) {
    const int fi = 2 * I + di;
    if (fi < 0 || fi >= gf.nx) continue;
#pragma unroll
    for (int dj = -1; dj <= 1; ++dj) {
      const int fj = 2 * J + dj;
      if (fj < 0 || fj >= gf.ny) continue;
      const float w0 = (float)dist_w(abs(di) + abs(dj)), w1 = (float)dist_w(abs(di) + abs(dj) + 1);
      const long long sf = gf.slot3(fi, fj, 2 * K);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float* a = in + c * gf.n + sf;
        const float2 pr = *reinterpret_cast<const float2*>(a);
        if (zm) v[c] += w1 * a[-1];
        v[c] += w0 * pr.x;
        if (zp) v[c] += w1 * pr.y;
      }
    }
  }
  const float iw = inv_bnd_total3<float>(nb);
  for (int c = 0; c < 3; ++c) v[c] = v[c] * iw;
}

// the fine children of coarse node (ci, cj, ck) (k_prolong3's order)
EDGE_D void tail_prolong(const Geo& gf, const Geo& gc, const float* __restrict__ in, float* __restrict__ out, int ci,
                         int cj, int ck) {
  const bool px = ci + 1 < gc.nx, py = cj + 1 < gc.ny, pz = ck + 1 < gc.nz;
  const bool fx = 2 * ci + 1 < gf.nx, fy = 2 * cj + 1 < gf.ny, fz = 2 * ck + 1 < gf.nz;
  float cv[2][2][2][3];
#pragma unroll
  for (int x = 0; x < 2; ++x)
#pragma unroll
    for (int y = 0; y < 2; ++y)
#pragma unroll
      for (int z = 0; z < 2; ++z) {
        const bool ex = (x == 0 || px) && (y == 0 || py) && (z == 0 || pz);
        const long long sc = gc.slot3(ci + x, cj + y, ck + z);
        const float iw = inv_bnd_total3<float>(is_bnd(ci + x, gc.nx) + is_bnd(cj + y, gc.ny) + is_bnd(ck + z, gc.nz));
#pragma unroll
        for (int c = 0; c < 3; ++c) cv[x][y][z][c] = ex ? in[c * gc.n + sc] * iw : 0.f;
      }
#pragma unroll
  for (int a = 0; a < 2; ++a) {
    if (a == 1 && !fx) continue;
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      if (b == 1 && !fy) continue;
      const int cxy = (1 + (a == 1 && px)) * (1 + (b == 1 && py));
      const float ic0 = 1.f / (float)cxy, ic1 = 1.f / (float)(cxy * (1 + pz));
      const long long sf = gf.slot3(2 * ci + a, 2 * cj + b, 2 * ck);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float v0 = 0.f, v1 = 0.f;
#pragma unroll
        for (int x = 0; x <= a; ++x)
#pragma unroll
          for (int y = 0; y <= b; ++y) {
            v0 += cv[x][y][0][c];
            v1 += cv[x][y][0][c];
            v1 += cv[x][y][1][c];
          }
        float* o = out + c * gf.n + sf;
        if (fz) {
          *reinterpret_cast<float2*>(o) = make_float2(v0 * ic0, v1 * ic1);
        } else {
          o[0] = v0 * ic0;
        }
      }
    }
  }
}

template <typename TS>
__global__ void __launch_bounds__(256) k_vcycle_tail(const TailParams<TS> T) {
  EDGE_PDL_ENTRY();
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nthr = (long long)gridDim.x * blockDim.x;
  const double om = __ldg(T.omega);
  // pre-smoothed iterate of each level: the buffer the last pre-sweep wrote
  float* xcur[TAIL_MAX];
  // ---- down
  for (int l = T.L0; l < T.L; ++l) {
    const TailLevel<TS>& V = T.lv[l - T.L0];
    const Geo& g = V.g;
    const float w = (float)(om * V.ws);
    if (l == T.L0) {  // first sweep from zero (below L0 it is fused into the restriction)
      for (long long q = tid; q < 3 * g.n; q += nthr) V.xa[q] = (w * V.dinv[q]) * V.b[q];
      tail_barrier(T.bar, T.err);
    }
    float* x = V.xa;
    float* y = V.xb;
    for (int sw = 1; sw < V.nsm; ++sw) {  // further sweeps: y = x + w Dinv (b - A x)
      for (long long s = tid; s < g.n; s += nthr) {
        const int k = (int)(s % g.pz), i = (int)((s / g.pz) % g.nx), j = (int)(s / g.plane);
        if (k >= g.nz) continue;
        float Au[3];
        tail_stencil(g, V.S, x, s, i, j, k, Au);
        for (int c = 0; c < 3; ++c) {
          const long long q = c * g.n + s;
          y[q] = x[q] + w * V.dinv[q] * (V.b[q] - Au[c]);
        }
      }
      tail_barrier(T.bar, T.err);
      float* t = x;
      x = y;
      y = t;
    }
    xcur[l - T.L0] = x;
    // r = b - A x
    for (long long s = tid; s < g.n; s += nthr) {
      const int k = (int)(s % g.pz), i = (int)((s / g.pz) % g.nx), j = (int)(s / g.plane);
      if (k >= g.nz) continue;
      float Au[3];
      tail_stencil(g, V.S, x, s, i, j, k, Au);
      for (int c = 0; c < 3; ++c) V.r[c * g.n + s] = V.b[c * g.n + s] - Au[c];
    }
    tail_barrier(T.bar, T.err);
    // b_{l+1} = R r, and (above the coarsest) the next level's first sweep from zero
    const TailLevel<TS>& C = T.lv[l + 1 - T.L0];
    const Geo& gc = C.g;
    const bool next_smoothed = l + 1 < T.L;
    const float wc = (float)(om * C.ws);
    for (long long t = tid; t < (long long)gc.nz * gc.nx * gc.ny; t += nthr) {
      const int K = (int)(t % gc.nz), I = (int)((t / gc.nz) % gc.nx), J = (int)(t / ((long long)gc.nz * gc.nx));
      float v[3];
      tail_restrict(g, gc, V.r, I, J, K, v);
      const long long sc = gc.slot3(I, J, K);
      for (int c = 0; c < 3; ++c) {
        const long long q = c * gc.n + sc;
        C.b[q] = v[c];
        if (next_smoothed) C.xa[q] = (wc * C.dinv[q]) * v[c];
      }
    }
    tail_barrier(T.bar, T.err);
  }
  // ---- coarsest: res = Ainv b, one warp per dense row
  {
    const TailLevel<TS>& Cl = T.lv[T.L - T.L0];
    const Geo& g = Cl.g;
    const int lane = threadIdx.x & 31;
    const long long nwarp = nthr >> 5;
    auto slot_of = [&](int dn) -> long long {
      const int node = dn / 3;
      const int k = node % g.nz, i = (node / g.nz) % g.nx, j = node / (g.nz * g.nx);
      return g.slot3(i, j, k);
    };
    for (long long row = tid >> 5; row < T.nd; row += nwarp) {
      const double* __restrict__ a = T.Ainv + row * T.nd;
      double acc = 0.0;
      for (int c = lane; c < T.nd; c += 32) acc += a[c] * (double)Cl.b[(c % 3) * g.n + slot_of(c)];
      acc = warp_sum(acc);
      if (lane == 0) Cl.res[((int)row % 3) * g.n + slot_of((int)row)] = (float)acc;
    }
    tail_barrier(T.bar, T.err);
  }
  // ---- up
  for (int l = T.L - 1; l >= T.L0; --l) {
    const TailLevel<TS>& V = T.lv[l - T.L0];
    const TailLevel<TS>& C = T.lv[l + 1 - T.L0];
    const Geo& g = V.g;
    const Geo& gc = C.g;
    const float w = (float)(om * V.ws);
    for (long long t = tid; t < (long long)gc.nz * gc.nx * gc.ny; t += nthr) {
      const int ck = (int)(t % gc.nz), ci = (int)((t / gc.nz) % gc.nx), cj = (int)(t / ((long long)gc.nz * gc.nx));
      tail_prolong(g, gc, C.res, V.ea, ci, cj, ck);
    }
    tail_barrier(T.bar, T.err);
    float* e = V.ea;
    float* f = V.eb;
    for (int sw = 1; sw < V.nsm; ++sw) {  // sweeps on the correction: f = e + w Dinv (r - A e)
      for (long long s = tid; s < g.n; s += nthr) {
        const int k = (int)(s % g.pz), i = (int)((s / g.pz) % g.nx), j = (int)(s / g.plane);
        if (k >= g.nz) continue;
        float Au[3];
        tail_stencil(g, V.S, e, s, i, j, k, Au);
        for (int c = 0; c < 3; ++c) {
          const long long q = c * g.n + s;
          f[q] = e[q] + w * V.dinv[q] * (V.r[q] - Au[c]);
        }
      }
      tail_barrier(T.bar, T.err);
      float* t = e;
      e = f;
      f = t;
    }
    // res = x + (e + w Dinv (r - A e))
    const float* x = xcur[l - T.L0];
    for (long long s = tid; s < g.n; s += nthr) {
      const int k = (int)(s % g.pz), i = (int)((s / g.pz) % g.nx), j = (int)(s / g.plane);
      if (k >= g.nz) continue;
      float Au[3];
      tail_stencil(g, V.S, e, s, i, j, k, Au);
      for (int c = 0; c < 3; ++c) {
        const long long q = c * g.n + s;
        const float en = e[q] + w * V.dinv[q] * (V.r[q] - Au[c]);
        V.res[q] = x[q] + en;
      }
    }
    if (l > T.L0) tail_barrier(T.bar, T.err);
  }
}

}  // namespace edge
