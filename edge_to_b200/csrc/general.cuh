// Unstructured meshes (any mix of element kinds): the stiffness operator K(rho) u, its
// diagonal, the element sensitivities and a CSR density filter, FP64, sm_100a.
//
// Replaces the reference's GPU kernels for general meshes (UniformStiffnessKernel /
// GeneralStiffnessKernel, kernels/_cuda.py:305-815, node-basis CUDA kernels of
// core/_templated_cuda.cu) and CuGeneralFilter (geom/_filters.py:278-298).  Semantics
// (mat_vec_node_basis_parallel_full, core/_ops.py): the product is node-centric,
//   out[i*dof + k] = sum over the elements e of node i of rho_e * sum over the
//                    unconstrained DOFs l of e of K_e[rel*dof + k, l] u[l],
// a constrained DOF's row is the identity and its column is dropped; the diagonal is 1 on
// constrained DOFs; dk_e = -u_e^T K_e u_e without masking (process_dk_full).
//
// Layout: element matrices row-major back to back (K_ptr[e] = offset of element e), the
// connectivity flat with element offsets, and a node -> (element, local corner) adjacency
// sorted by node and then element, built on the host at creation, so every sum has a fixed
// order (no atomics; results are reproducible run to run).  One thread per DOF row; the
// element's matrix row is read contiguously.
#pragma once
#include "common.cuh"

namespace edge {

struct GenGeo {
  int dof;
  long long n_nodes, n_el;
  const int* elem_ptr;        // n_el + 1
  const int* elem_flat;       // node ids of every element
  const long long* K_ptr;     // n_el + 1, offsets into K
  const double* K;            // row-major nk x nk per element, nk = size * dof
  const long long* adj_ptr;   // n_nodes + 1
  const int* adj_el;          // element of each adjacency entry
  const unsigned char* adj_loc;  // local corner of the node in that element
};

// out = K(rho) u (identity rows/columns on constrained DOFs); with dot != null also
// acc += u . out, reduced into *dot (deterministic).
__global__ void k_gen_matvec(const GenGeo G, const double* __restrict__ rho, const uint8_t* __restrict__ cons,
                             const double* __restrict__ u, double* __restrict__ out, double* part, unsigned* ticket,
                             double* dot) {
  EDGE_PDL_ENTRY();
  const int dof = G.dof;
  const long long n = G.n_nodes * dof;
  double acc = 0.0;
  for (long long row = blockIdx.x * (long long)blockDim.x + threadIdx.x; row < n;
       row += (long long)gridDim.x * blockDim.x) {
    const long long i = row / dof;
    const int k = (int)(row - i * dof);
    double v;
    if (cons[row]) {
      v = u[row];
    } else {
      v = 0.0;
      for (long long a = G.adj_ptr[i]; a < G.adj_ptr[i + 1]; ++a) {
        const int e = G.adj_el[a];
        const int base = G.elem_ptr[e];
        const int nk = (G.elem_ptr[e + 1] - base) * dof;
        const double* Kr = G.K + G.K_ptr[e] + (long long)(G.adj_loc[a] * dof + k) * nk;
        double s = 0.0;
        for (int l = 0; l < nk; ++l) {
          const long long kk = (long long)G.elem_flat[base + l / dof] * dof + l % dof;
          if (!cons[kk]) s += Kr[l] * u[kk];
        }
        v += s * rho[e];
      }
    }
    out[row] = v;
    acc += u[row] * v;
  }
  if (dot) {
    __shared__ double sh[32];
    const double bt = block_sum(acc, sh);
    struct Fin {
      double* d;
      EDGE_D void operator()(double t) const { *d = t; }
    };
    grid_reduce_finish(bt, part, ticket, Fin{dot});
  }
}

// diag(K(rho)), 1 on constrained DOFs (get_diagonal_node_basis_full).
__global__ void k_gen_diagonal(const GenGeo G, const double* __restrict__ rho, const uint8_t* __restrict__ cons,
                               double* __restrict__ out) {
  EDGE_PDL_ENTRY();
  const int dof = G.dof;
  const long long n = G.n_nodes * dof;
  for (long long row = blockIdx.x * (long long)blockDim.x + threadIdx.x; row < n;
       row += (long long)gridDim.x * blockDim.x) {
    const long long i = row / dof;
    const int k = (int)(row - i * dof);
    double v = 0.0;
    if (cons[row]) {
      v = 1.0;
    } else {
      for (long long a = G.adj_ptr[i]; a < G.adj_ptr[i + 1]; ++a) {
        const int e = G.adj_el[a];
        const int nk = (G.elem_ptr[e + 1] - G.elem_ptr[e]) * dof;
        const int r = G.adj_loc[a] * dof + k;
        v += G.K[G.K_ptr[e] + (long long)r * nk + r] * rho[e];
      }
    }
    out[row] = v;
  }
}

// dk_e = -u_e^T K_e u_e (process_dk_full): one thread per element.
__global__ void k_gen_dk(const GenGeo G, const double* __restrict__ U, double* __restrict__ dk) {
  EDGE_PDL_ENTRY();
  const int dof = G.dof;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < G.n_el;
       e += (long long)gridDim.x * blockDim.x) {
    const int base = G.elem_ptr[e];
    const int nk = (G.elem_ptr[e + 1] - base) * dof;
    const double* Ke = G.K + G.K_ptr[e];
    double s = 0.0;
    for (int a = 0; a < nk; ++a) {
      const double ua = U[(long long)G.elem_flat[base + a / dof] * dof + a % dof];
      double t = 0.0;
      for (int b = 0; b < nk; ++b) t += Ke[(long long)a * nk + b] * U[(long long)G.elem_flat[base + b / dof] * dof + b % dof];
      s += ua * t;
    }
    dk[e] = -s;
  }
}

// y = A x for a CSR matrix, one thread per row, entries in stored order.
__global__ void k_csr_spmv(long long n, const long long* __restrict__ ptr, const int* __restrict__ idx,
                           const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y) {
  EDGE_PDL_ENTRY();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (long long a = ptr[i]; a < ptr[i + 1]; ++a) s += val[a] * x[idx[a]];
    y[i] = s;
  }
}

// y = a x + b y
__global__ void k_axpby(long long n, double a, const double* __restrict__ x, double b, double* __restrict__ y) {
  EDGE_PDL_ENTRY();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = a * x[i] + b * y[i];
}

}  // namespace edge
