// Shared definitions for the SIMP / GMG-PCG kernels (sm_100a).
//
// Internal data layout ("slot layout"), used for every vector and element array
// inside the solver:
//   3-D level with nodes (nx, ny, nz):  slot(i, j, k) = j*plane + i*pz + k,
//        pz = nz rounded up to a multiple of 4 (16-byte rows for fp32 tiles),
//        plane = nx*pz; the reference's node order (j slowest, then i, k fastest,
//        core/_geom.py:48-57) is kept, with zero padding at the end of each z-row.
//   2-D level with nodes (nx, ny):      slot(i, j) = j*pz + i, pz = nx rounded up to 4.
// Vectors are stored structure-of-arrays: component c of slot s lives at v[c*n + s],
// n = ny*plane.  Element arrays are "node aligned": element (i,j,k) is stored at the
// slot of its lower corner node; slots without an element (last row/column/plane and
// padding) hold zero, so every node has 2^d surrounding elements and a zero-stiffness
// ghost element stands in where the grid ends.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#define EDGE_HD __host__ __device__ __forceinline__
#define EDGE_D __device__ __forceinline__

namespace edge {

struct Geo {
  int dim;          // 2 or 3
  int nx, ny, nz;   // nodes per axis (nz = 1 in 2-D)
  int pz;           // padded length of the fastest axis (z in 3-D, x in 2-D)
  long long plane;  // slots per y-plane (3-D) or per row (2-D)
  long long n;      // slots per component
  int dof;          // components per node (= dim)

  EDGE_HD long long slot3(int i, int j, int k) const { return (long long)j * plane + (long long)i * pz + k; }
  EDGE_HD long long slot2(int i, int j) const { return (long long)j * pz + i; }
};

// zalign: the fastest axis is padded to a multiple of this many nodes (4 keeps FP32 rows on
// 16-byte boundaries; 8 does the same for 2-byte rows).
inline Geo make_geo(int dim, int nelx, int nely, int nelz, int zalign = 4) {
  Geo g;
  g.dim = dim;
  g.dof = dim;
  g.nx = nelx + 1;
  g.ny = nely + 1;
  if (dim == 3) {
    g.nz = nelz + 1;
    g.pz = (g.nz + zalign - 1) / zalign * zalign;
    g.plane = (long long)g.nx * g.pz;
  } else {
    g.nz = 1;
    g.pz = (g.nx + 3) & ~3;
    g.plane = g.pz;
  }
  g.n = (long long)g.ny * g.plane;
  return g;
}

// Programmatic dependent launch.  Inside the captured solve graph kernels are launched with
// programmatic stream serialization, so a kernel's blocks may be scheduled while the kernel
// before it is still finishing.  Every kernel therefore waits for that grid to complete (and
// its memory to be visible) before its first memory access, and then lets its own dependents
// start launching.  Both instructions are no-ops for a kernel launched without the attribute.
#define EDGE_PDL_ENTRY() asm volatile("griddepcontrol.wait;\n\tgriddepcontrol.launch_dependents;" ::: "memory")

// ------------------------------------------------------------------ type helpers
template <typename T> EDGE_D T ld(const T* p) { return __ldg(p); }
EDGE_D double to_d(double x) { return x; }
EDGE_D double to_d(float x) { return (double)x; }
EDGE_D double to_d(__nv_bfloat16 x) { return (double)__bfloat162float(x); }
EDGE_D float to_f(double x) { return (float)x; }
EDGE_D float to_f(float x) { return x; }
EDGE_D float to_f(__nv_bfloat16 x) { return __bfloat162float(x); }

// Two-wide vector types (pair loads in the PCG vector kernels and the paired stencil; every
// vector is 16-byte aligned and holds dof * n entries with n a multiple of 4).
template <typename T> struct V2;
template <> struct V2<double> {
  using type = double2;
};
template <> struct V2<float> {
  using type = float2;
};

template <typename T> struct Conv;
template <> struct Conv<double> {
  EDGE_D static double from(double x) { return x; }
  EDGE_D static double from(float x) { return (double)x; }
  EDGE_D static double from(__nv_bfloat16 x) { return (double)__bfloat162float(x); }
};
template <> struct Conv<float> {
  EDGE_D static float from(double x) { return (float)x; }
  EDGE_D static float from(float x) { return x; }
  EDGE_D static float from(__nv_bfloat16 x) { return __bfloat162float(x); }
};
template <> struct Conv<__nv_bfloat16> {
  EDGE_D static __nv_bfloat16 from(double x) { return __float2bfloat16_rn((float)x); }
  EDGE_D static __nv_bfloat16 from(float x) { return __float2bfloat16_rn(x); }
};

// ------------------------------------------------------------------ reductions
EDGE_D double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide fp64 sum in a fixed order (deterministic).  `sh` needs 32 doubles.
EDGE_D double block_sum(double v, double* sh) {
  const int lane = (threadIdx.x + threadIdx.y * blockDim.x) & 31;
  const int wid = (threadIdx.x + threadIdx.y * blockDim.x) >> 5;
  const int nw = (blockDim.x * blockDim.y + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (wid == 0) {
    r = lane < nw ? sh[lane] : 0.0;
    r = warp_sum(r);
  }
  return r;  // valid in thread 0 of the block
}

// Grid-wide deterministic reduction: every block writes its partial to part[block];
// the last block to arrive sums the partials in block order and calls fin(total).
// `ticket` must be zero on entry; the last block resets it.
template <class Fin>
EDGE_D void grid_reduce_finish(double block_total, double* part, unsigned int* ticket, Fin fin) {
  __shared__ bool am_last;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  const unsigned int nblk = gridDim.x * gridDim.y * gridDim.z;
  const unsigned int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  if (tid == 0) {
    part[bid] = block_total;
    __threadfence();
    unsigned int t = atomicAdd(ticket, 1u);
    am_last = (t == nblk - 1);
  }
  __syncthreads();
  if (am_last) {
    __threadfence();
    __shared__ double sh[32];
    double acc = 0.0;
    const int nthr = blockDim.x * blockDim.y;
    // fixed assignment of partials to threads, fixed tree: deterministic
    for (unsigned int b = tid; b < nblk; b += nthr) acc += ((volatile double*)part)[b];
    double tot = block_sum(acc, sh);
    if (tid == 0) {
      fin(tot);
      *ticket = 0u;
    }
  }
}

}  // namespace edge
