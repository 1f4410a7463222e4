// Element operator of the structured stiffness matrix, in the Walsh-Hadamard basis.
//
// For an axis-aligned box element (Q4 / hex8 with full Gauss integration, which is
// exact for these shape functions), the element stiffness K0 of the reference
// (physics/_linelas.py:195-309, 338-447) is a sum of Kronecker products of 1-D
// matrices that are all diagonalised, or mapped between the two basis vectors
// (1,1) and (1,-1), by the 2-point transform F = [[1,1],[1,-1]] on every axis.  With
// T = F (x) F (x) F acting on the corner index, Khat = T K0 T^-1 has 45 non-zeros
// out of 576 (hex8) and 10 out of 64 (Q4):
//   * a diagonal term for every (transform index h != 0, component c), and
//   * a coupling (h, c) <- (h ^ e_c ^ e_d, d) for d != c where bits c and d of h
//     differ.
// K u_e = T^-1 Khat T u_e = (1/2^d) T Khat (T u_e), so one element costs two
// 2^d-point fast transforms plus the sparse Khat, about 230 flops instead of the
// 1152 of a dense 24x24 product.  The host builds Khat from the actual K0 and checks
// that nothing falls outside this pattern; if something does, the dense kernels run.
//
// Corner numbering here is by bits: corner b has offset (b&1, (b>>1)&1, (b>>2)&1)
// along (x, y, z); component c (0=x, 1=y, 2=z) is the axis with bit (1<<c).
#pragma once
#include "common.cuh"

namespace edge {

template <typename T> struct KHat3 {
  T dg[3][8];      // dg[c][h] : coefficient of (h,c) <- (h,c), already divided by 8
  T of[3][3][8];   // of[c][d][h]: coefficient of (h,c) <- (h^(1<<c)^(1<<d), d), divided by 8
};
template <typename T> struct KHat2 {
  T dg[2][4];
  T of[2][2][4];
};

template <typename T> EDGE_D void fwht8(T x[8]) {
#pragma unroll
  for (int bit = 1; bit < 8; bit <<= 1) {
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      if (!(a & bit)) {
        T p = x[a], q = x[a | bit];
        x[a] = p + q;
        x[a | bit] = p - q;
      }
    }
  }
}

template <typename T> EDGE_D void fwht4(T x[4]) {
#pragma unroll
  for (int bit = 1; bit < 4; bit <<= 1) {
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      if (!(a & bit)) {
        T p = x[a], q = x[a | bit];
        x[a] = p + q;
        x[a | bit] = p - q;
      }
    }
  }
}

// f[b][c] = E * (K0 u)[b][c] for one hex8 element.  u and f are indexed [corner][comp].
template <typename T>
EDGE_D void elem3_apply(const KHat3<T>& K, T E, const T u[8][3], T f[8][3]) {
  T uh[3][8];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int b = 0; b < 8; ++b) uh[c][b] = u[b][c];
    fwht8(uh[c]);
#pragma unroll
    for (int h = 1; h < 8; ++h) uh[c][h] *= E;
  }
  T vh[3][8];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    vh[c][0] = T(0);
#pragma unroll
    for (int h = 1; h < 8; ++h) {
      T acc = K.dg[c][h] * uh[c][h];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if (d != c && (((h >> c) & 1) != ((h >> d) & 1))) {
          acc += K.of[c][d][h] * uh[d][h ^ (1 << c) ^ (1 << d)];
        }
      }
      vh[c][h] = acc;
    }
    fwht8(vh[c]);
#pragma unroll
    for (int b = 0; b < 8; ++b) f[b][c] = vh[c][b];
  }
}

// u_e^T K0 u_e for one hex8 element (no E): (1/8) uh^T Khat uh.
template <typename T>
EDGE_D T elem3_energy(const KHat3<T>& K, const T u[8][3]) {
  T uh[3][8];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int b = 0; b < 8; ++b) uh[c][b] = u[b][c];
    fwht8(uh[c]);
  }
  T e = T(0);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int h = 1; h < 8; ++h) {
      T acc = K.dg[c][h] * uh[c][h];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if (d != c && (((h >> c) & 1) != ((h >> d) & 1))) acc += K.of[c][d][h] * uh[d][h ^ (1 << c) ^ (1 << d)];
      }
      e += uh[c][h] * acc;
    }
  }
  return e;
}

template <typename T>
EDGE_D void elem2_apply(const KHat2<T>& K, T E, const T u[4][2], T f[4][2]) {
  T uh[2][4];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
#pragma unroll
    for (int b = 0; b < 4; ++b) uh[c][b] = u[b][c];
    fwht4(uh[c]);
#pragma unroll
    for (int h = 1; h < 4; ++h) uh[c][h] *= E;
  }
  T vh[2][4];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    vh[c][0] = T(0);
#pragma unroll
    for (int h = 1; h < 4; ++h) {
      T acc = K.dg[c][h] * uh[c][h];
      const int d = 1 - c;
      if (((h >> c) & 1) != ((h >> d) & 1)) acc += K.of[c][d][h] * uh[d][h ^ 3];
      vh[c][h] = acc;
    }
    fwht4(vh[c]);
#pragma unroll
    for (int b = 0; b < 4; ++b) f[b][c] = vh[c][b];
  }
}

template <typename T>
EDGE_D T elem2_energy(const KHat2<T>& K, const T u[4][2]) {
  T uh[2][4];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
#pragma unroll
    for (int b = 0; b < 4; ++b) uh[c][b] = u[b][c];
    fwht4(uh[c]);
  }
  T e = T(0);
#pragma unroll
  for (int c = 0; c < 2; ++c) {
#pragma unroll
    for (int h = 1; h < 4; ++h) {
      T acc = K.dg[c][h] * uh[c][h];
      const int d = 1 - c;
      if (((h >> c) & 1) != ((h >> d) & 1)) acc += K.of[c][d][h] * uh[d][h ^ 3];
      e += uh[c][h] * acc;
    }
  }
  return e;
}

}  // namespace edge
