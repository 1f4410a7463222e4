// Packed-pair fine-level operator for cube elements (3-D, FP32), sm_100a.
//
// The tiling, TMA staging and node-combination scheme are those of k_fine3_pk (two
// neighbouring element columns per thread in float2 registers, y-marching blocks, a ring
// of cp.async.bulk.tensor stages, transform-domain carry of the upper-face part).  Three
// things differ:
//
//  * The transformed element operator is applied in its block form.  For a cube element
//    (equal edge lengths) of an isotropic material, Khat (element_op.cuh) splits into
//      - a 3x3 block {(1,x),(2,y),(4,z)} with equal diagonals and equal off-diagonals
//        (normal strains): v = nd*u + no*(u1+u2+u3),
//      - three rank-1 2x2 blocks {(1,y),(2,x)}, {(1,z),(4,x)}, {(2,z),(4,y)} with all
//        four entries equal (shear strains): v1 = v2 = sh*(u1+u2),
//      - three 2x2 blocks {(3,x),(6,z)}, {(3,y),(5,z)}, {(5,x),(6,y)} with equal diagonals
//        (bending modes): v1 = bd*u1 + bo*u2, v2 = bo*u1 + bd*u2,
//      - a 3x3 block {(3,z),(5,y),(6,x)} like the first (twist): v = td*u + to*(sum),
//      - a diagonal for h = 7 (the hourglass mode): v = h7*u,
//    so eight coefficients describe it.  They are scaled by E once per element (8 packed
//    multiplies) and the block products take 33 more, against 66 for the general sparse
//    form, and the coefficients stay in registers for the whole kernel.  The host checks
//    every one of the 576 entries of Khat against this model before choosing the kernel.
//  * The y loop is unrolled by two so that the lower and upper planes swap roles without
//    register copies.
//  * The h = 0 transform coefficient (rigid translation) is never formed: its output is
//    zero, and the carry for (hx, hz) = (0, 0) is kept with the opposite sign so that the
//    y stage needs no negation.
//
//  * The epilogue's per-node inputs (right-hand side, Jacobi diagonal, correction base)
//    travel through the same TMA ring as u, one box per array and plane,
//    so the epilogue reads shared memory instead of waiting on global loads; this keeps
//    the smoother sweep close to the plain product although the kernel runs few warps.
//    A stage is refilled at the barrier of the layer after the one that used it, so the
//    epilogue reads its inputs after the barrier and holds no registers across it.
//
//  * The operator's input u may be computed from one or two staged arrays as the tile is
//    read (IN): u itself (InU); the first damped-Jacobi sweep from zero, u = w Dinv b
//    (InWDB: b FP32 and the BF16 Dinv, so a V-cycle's first fine sweep is never stored);
//    or the PCG search direction u = z + beta p_old (InPDir), the new p written out by the
//    epilogue into the other buffer of a ping-pong pair (blocks read p_old in their halos,
//    so it cannot be overwritten in place).  The epilogue recomputes each output node's
//    input value from the stage it was read from (no registers held across the layer).
//
// TMA boxes, strides and alignments are those of k_fine3_pk, plus the staged arrays: FP32
// and FP64 boxes start at z0-1 rounded down to 4 nodes (16 / 32 bytes), BF16 boxes at z0-1
// rounded down to 8 nodes (16 bytes; the 3-D fine level pads z to a multiple of 8 so that
// BF16 rows are 16-byte strided).  Every mbarrier wait is bounded (fast try first, then
// the clocked wait of fine_tma.cuh).  No multicast.
#pragma once
#include "fine_pk.cuh"
#include "misc.cuh"  // PcgState (the search-direction input reads beta from it)

namespace edge {

// Block-form coefficients of a cube element's Khat (already divided by 8 like KHat3).
struct KCube {
  float nd, no, sh, bd, bo, td, to, h7;
};

EDGE_D bool mbar_wait_fast(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  if (ok) return true;
  return mbar_wait(bar, parity);
}

// Optional members of the input transforms (IN) and epilogues (SE), detected at compile time:
// IN::parity0() selects the alternative map of input array 0 (a ping-pong pair), IN::kT2 the
// type of a third input array; SE::kParS names the staged array with an alternative map
// (chosen by SE::parity()), SE::fin() a custom finisher of the launch's reduction.
template <class T, class = void> struct HasPar0 : std::false_type {};
template <class T> struct HasPar0<T, std::void_t<decltype(std::declval<const T&>().parity0())>> : std::true_type {};
template <class T, class = void> struct HasParS : std::false_type {};
template <class T> struct HasParS<T, std::void_t<decltype(T::kParS)>> : std::true_type {};
template <class T, class = void> struct HasFin : std::false_type {};
template <class T> struct HasFin<T, std::void_t<decltype(std::declval<const T&>().fin())>> : std::true_type {};
template <class IN> EDGE_HD constexpr int in_t2() {
  if constexpr (IN::kN == 3) return IN::kT2;
  else return 0;
}
template <class SE> EDGE_HD constexpr int se_pars() {
  if constexpr (HasParS<SE>::value) return SE::kParS;
  else return -1;
}

// v = E * Khat u in block form; uh / vh indexed [h][c], h = hx | hy<<1 | hz<<2; h = 0 is
// neither read nor written.
EDGE_D void khat_cube(const P2 kc[8], P2 E, const P2 uh[8][3], P2 vh[8][3]) {
  P2 k[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) k[i] = kc[i] * E;
  {  // normal strains
    const P2 t = k[1] * (uh[1][0] + uh[2][1] + uh[4][2]);
    vh[1][0] = pfma(k[0], uh[1][0], t);
    vh[2][1] = pfma(k[0], uh[2][1], t);
    vh[4][2] = pfma(k[0], uh[4][2], t);
  }
  {  // shear strains
    const P2 a = k[2] * (uh[1][1] + uh[2][0]);
    vh[1][1] = a;
    vh[2][0] = a;
    const P2 b = k[2] * (uh[1][2] + uh[4][0]);
    vh[1][2] = b;
    vh[4][0] = b;
    const P2 c = k[2] * (uh[2][2] + uh[4][1]);
    vh[2][2] = c;
    vh[4][1] = c;
  }
  // bending pairs
  auto pair = [&](int h1, int c1, int h2, int c2) {
    const P2 a = uh[h1][c1], b = uh[h2][c2];
    vh[h1][c1] = pfma(k[4], b, k[3] * a);
    vh[h2][c2] = pfma(k[4], a, k[3] * b);
  };
  pair(3, 0, 6, 2);
  pair(3, 1, 5, 2);
  pair(5, 0, 6, 1);
  {  // twist
    const P2 t = k[6] * (uh[3][2] + uh[5][1] + uh[6][0]);
    vh[3][2] = pfma(k[5], uh[3][2], t);
    vh[5][1] = pfma(k[5], uh[5][1], t);
    vh[6][0] = pfma(k[5], uh[6][0], t);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) vh[7][c] = k[7] * uh[7][c];
}

// ------------------------------------------------------------------ staged epilogues
// Each epilogue names the arrays it reads per output node (kN of them, element types kT),
// loads its inputs from the stage of the output plane (load, before the stage is recycled)
// and finishes the node (apply).  sp[i] points at component 0 of array i for this node;
// cs4 / cs2 are the component strides (elements) of 4/8-byte and 2-byte boxes.
enum : int { ST_F32 = 0, ST_BF16 = 1, ST_F64 = 2 };
EDGE_HD constexpr int st_width(int t) { return t == ST_BF16 ? 32 : 24; }
EDGE_HD constexpr int st_esize(int t) { return t == ST_BF16 ? 2 : (t == ST_F64 ? 8 : 4); }

struct SEStore {  // out = A u
  float* out;
  long long n;
  static constexpr int kN = 0;
  static constexpr bool kDot = false;
  EDGE_HD static constexpr int kT(int i) { return i == 0 ? 0 : i == 1 ? 0 : i == 2 ? 0 : 0; }
  struct In {};
  EDGE_D void init() {}
  EDGE_D In load(const unsigned char* const*, int, int, const float*, const float*, int) const { return {}; }
  EDGE_D void apply(long long s, const float*, const float* Au, const In&, double&) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) out[c * n + s] = Au[c];
  }
};

struct SEStoreDot {  // out = A u, acc += u . A u
  float* out;
  long long n;
  static constexpr int kN = 0;
  static constexpr bool kDot = true;
  EDGE_HD static constexpr int kT(int i) { return i == 0 ? 0 : i == 1 ? 0 : i == 2 ? 0 : 0; }
  struct In {};
  EDGE_D void init() {}
  EDGE_D In load(const unsigned char* const*, int, int, const float*, const float*, int) const { return {}; }
  EDGE_D void apply(long long s, const float* own, const float* Au, const In&, double& acc) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      out[c * n + s] = Au[c];
      acc += (double)own[c] * (double)Au[c];
    }
  }
};

struct SEResid {  // r = b - A u
  float* r;
  long long n;
  static constexpr int kN = 1;
  static constexpr bool kDot = false;
  EDGE_HD static constexpr int kT(int i) { return i == 0 ? ST_F32 : i == 1 ? 0 : i == 2 ? 0 : 0; }
  struct In {
    float b[3];
  };
  EDGE_D void init() {}
  EDGE_D In load(const unsigned char* const* sp, int cs4, int, const float*, const float*, int) const {
    In v;
#pragma unroll
    for (int c = 0; c < 3; ++c) v.b[c] = reinterpret_cast<const float*>(sp[0])[c * cs4];
    return v;
  }
  EDGE_D void apply(long long s, const float*, const float* Au, const In& v, double&) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) r[c * n + s] = v.b[c] - Au[c];
  }
};

struct SEJacobi {  // xo = u + w Dinv (b - A u)
  float* xo;
  const double* omega;
  double wscale;
  long long n;
  float w;
  static constexpr int kN = 2;
  static constexpr bool kDot = false;
  EDGE_HD static constexpr int kT(int i) { return i == 0 ? ST_F32 : i == 1 ? ST_BF16 : i == 2 ? 0 : 0; }
  struct In {
    float b[3], d[3];
  };
  EDGE_D void init() { w = (float)(__ldg(omega) * wscale); }
  EDGE_D In load(const unsigned char* const* sp, int cs4, int cs2, const float*, const float*, int) const {
    In v;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      v.b[c] = reinterpret_cast<const float*>(sp[0])[c * cs4];
      v.d[c] = __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(sp[1])[c * cs2]);
    }
    return v;
  }
  EDGE_D void apply(long long s, const float* own, const float* Au, const In& v, double&) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) xo[c * n + s] = own[c] + w * v.d[c] * (v.b[c] - Au[c]);
  }
};

// last post-smoothing sweep with the correction: xo = xbase + e + w Dinv (b - A e), e = u;
// with DOT, acc += dotv . xo accumulated in FP64, dotv an FP32 array staged like the others
// (the PCG's r.z with the FP32 copy of the residual)
template <bool DOT> struct SEJacobiAdd {
  float* xo;
  const double* omega;
  double wscale;
  long long n;
  float w;
  static constexpr int kN = DOT ? 4 : 3;
  static constexpr bool kDot = DOT;
  EDGE_HD static constexpr int kT(int i) { return i == 0 ? ST_F32 : i == 1 ? ST_BF16 : ST_F32; }
  struct In {
    float b[3], d[3], xb[3];
    float dv[DOT ? 3 : 1];
  };
  EDGE_D void init() { w = (float)(__ldg(omega) * wscale); }
  EDGE_D In load(const unsigned char* const* sp, int cs4, int cs2, const float*, const float*, int) const {
    In v;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      v.b[c] = reinterpret_cast<const float*>(sp[0])[c * cs4];
      v.d[c] = __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(sp[1])[c * cs2]);
      v.xb[c] = reinterpret_cast<const float*>(sp[2])[c * cs4];
      if constexpr (DOT) v.dv[c] = reinterpret_cast<const float*>(sp[3])[c * cs4];
    }
    return v;
  }
  EDGE_D void apply(long long s, const float* own, const float* Au, const In& v, double& acc) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float x = v.xb[c] + (own[c] + w * v.d[c] * (v.b[c] - Au[c]));
      xo[c * n + s] = x;
      if constexpr (DOT) acc += (double)v.dv[c] * (double)x;
    }
  }
};


// r = b - A u with b the operator's input array 0 (the V-cycle's first fine step: u = w Dinv
// b computed from the staged b and Dinv, so b is already in the stage)
struct SEResidIn {
  float* r;
  long long n;
  static constexpr int kN = 0;
  static constexpr bool kDot = false;
  EDGE_HD static constexpr int kT(int) { return 0; }
  struct In {
    float b[3];
  };
  EDGE_D void init() {}
  EDGE_D In load(const unsigned char* const*, int, int, const float* in0, const float*, int uc4) const {
    In v;
#pragma unroll
    for (int c = 0; c < 3; ++c) v.b[c] = in0[c * uc4];
    return v;
  }
  EDGE_D void apply(long long s, const float*, const float* Au, const In& v, double&) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) r[c * n + s] = v.b[c] - Au[c];
  }
};

// Last post-smoothing sweep of a one-sweep fine level with the correction, where the
// pre-smoothed iterate was never stored: xo = w Dinv b + (e + w Dinv (r - A e)), e = u, r the
// level's residual (the correction equation's right-hand side) and b the V-cycle's right-hand
// side; with DOT, acc += b . xo (the PCG's r.z: b is the FP32 residual).  The same arithmetic,
// in the same order, as the stored-iterate path (k_jacobi0 followed by SEJacobiAdd).
template <bool DOT> struct SEJacobiAdd0 {
  float* xo;
  const double* omega;
  double wscale;
  long long n;
  float w;
  // with st: b is the residual of a ping-pong pair, in the buffer of the iteration's parity
  // (staged array 2 from the alternative map when st->iter is odd)
  const PcgState* st;
  static constexpr int kN = 3;
  static constexpr bool kDot = DOT;
  static constexpr int kParS = 2;
  EDGE_D int parity() const { return st ? (st->iter & 1) : 0; }
  EDGE_HD static constexpr int kT(int i) { return i == 1 ? ST_BF16 : ST_F32; }  // r, Dinv, b
  struct In {
    float r[3], d[3], b[3];
  };
  EDGE_D void init() { w = (float)(__ldg(omega) * wscale); }
  EDGE_D In load(const unsigned char* const* sp, int cs4, int cs2, const float*, const float*, int) const {
    In v;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      v.r[c] = reinterpret_cast<const float*>(sp[0])[c * cs4];
      v.d[c] = __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(sp[1])[c * cs2]);
      v.b[c] = reinterpret_cast<const float*>(sp[2])[c * cs4];
    }
    return v;
  }
  EDGE_D void apply(long long s, const float* own, const float* Au, const In& v, double& acc) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float xb = (w * v.d[c]) * v.b[c];
      const float x = xb + (own[c] + w * v.d[c] * (v.r[c] - Au[c]));
      xo[c * n + s] = x;
      if constexpr (DOT) acc += (double)v.b[c] * (double)x;
    }
  }
};

// q = A p, p written out, acc += p . A p, with p = z + beta p_old computed by the input
// transform (InPDir); p_new goes to the buffer the iteration's parity selects.
struct SEStorePDot {
  float* q;
  float* pa;  // p buffers: iteration parity 0 reads pa and writes pb, parity 1 the reverse
  float* pb;
  const PcgState* st;
  long long n;
  float* pout;
  static constexpr int kN = 0;
  static constexpr bool kDot = true;
  EDGE_HD static constexpr int kT(int) { return 0; }
  struct In {};
  EDGE_D void init() { pout = (st->iter & 1) ? pa : pb; }
  EDGE_D In load(const unsigned char* const*, int, int, const float*, const float*, int) const { return {}; }
  EDGE_D void apply(long long s, const float* own, const float* Au, const In&, double& acc) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      q[c * n + s] = Au[c];
      pout[c * n + s] = own[c];
      acc += (double)own[c] * (double)Au[c];
    }
  }
};

// Finisher of the residual-update launch: the state of k_pcg_xr32's finisher (alpha, rz,
// rr, residual, iteration count, stop reason, next omega), and the pending solution update
// x32 += alpha p that the next search-direction launch applies (st->xa).
struct PcgXrFinX {
  PcgState* st;
  bool upd;
  double alpha;
  EDGE_D void operator()(double t) const {
    if (!upd) return;
    PcgXrFin{st, alpha}(t);
    st->xa = alpha;
  }
};

// Epilogue of the fused first launch (InWDBQ): r = b - A u into the level-0 residual, and,
// with an update pending, the updated PCG residual b into the other buffer of the ping-pong
// pair and r.r (FP64 sum of the FP32 squares) for the finisher.
struct SEResidInX {
  float* r;
  float* R0;
  float* R1;
  PcgState* st;
  long long n;
  float af;
  bool upd;
  double alpha;
  float* rout;
  static constexpr int kN = 0;
  static constexpr bool kDot = true;
  EDGE_HD static constexpr int kT(int) { return 0; }
  struct In {
    float b[3];
  };
  EDGE_D void init() {
    upd = st->pend != 0;
    alpha = upd ? st->rz_new / st->pq : 0.0;
    af = (float)alpha;
    rout = (st->iter & 1) ? R0 : R1;
  }
  EDGE_D In load(const unsigned char* const*, int, int, const float* in0, const float* in1, int uc4) const {
    In v;
#pragma unroll
    for (int c = 0; c < 3; ++c) v.b[c] = upd ? fmaf(-af, in1[c * uc4], in0[c * uc4]) : in0[c * uc4];
    return v;
  }
  EDGE_D void apply(long long s, const float*, const float* Au, const In& v, double& acc) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      r[c * n + s] = v.b[c] - Au[c];
      if (upd) {
        rout[c * n + s] = v.b[c];
        acc += (double)(v.b[c] * v.b[c]);
      }
    }
  }
  EDGE_D PcgXrFinX fin() const { return PcgXrFinX{st, upd, alpha}; }
};

// Finisher of the search-direction launch: p.q, and from now on a residual update is pending.
struct PqFin {
  PcgState* st;
  EDGE_D void operator()(double t) const {
    st->pq = t;
    st->pend = 1;
  }
};

// SEStorePDot with the pending solution update: x32 += xa p_old at the owner nodes (FP32,
// k_pcg_xr32's arithmetic; p_old is the input transform's array 1, x32 staged), xa the alpha
// of the previous iteration (0: nothing pending).
struct SEStorePDotX {
  float* q;
  float* pa;
  float* pb;
  PcgState* st;
  long long n;
  float* x32;
  float* pout;
  float xa;
  static constexpr int kN = 1;
  static constexpr bool kDot = true;
  EDGE_HD static constexpr int kT(int) { return ST_F32; }
  struct In {
    float x[3], po[3];
  };
  EDGE_D void init() {
    pout = (st->iter & 1) ? pa : pb;
    xa = (float)st->xa;
  }
  EDGE_D In load(const unsigned char* const* sp, int cs4, int, const float*, const float* in1, int uc4) const {
    In v;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      v.x[c] = reinterpret_cast<const float*>(sp[0])[c * cs4];
      v.po[c] = in1[c * uc4];
    }
    return v;
  }
  EDGE_D void apply(long long s, const float* own, const float* Au, const In& v, double& acc) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      q[c * n + s] = Au[c];
      pout[c * n + s] = own[c];
      acc += (double)own[c] * (double)Au[c];
      if (xa != 0.f) x32[c * n + s] = fmaf(xa, v.po[c], v.x[c]);
    }
  }
  EDGE_D PqFin fin() const { return PqFin{st}; }
};

// ------------------------------------------------------------------ operator inputs
// value(a0, a1, i4, i2): the input at one node and component of the stage, from array 0
// (FP32, element index i4) and array 1 (kT1: FP32 index i4 or BF16 index i2).
struct InU {  // u itself
  static constexpr int kN = 1;
  static constexpr int kT1 = ST_F32;
  EDGE_D void init() {}
  EDGE_D int parity() const { return 0; }
  EDGE_D float value(const float* a0, const void*, const void*, int i4, int) const { return a0[i4]; }
};
struct InWDB {  // u = (w Dinv) b: the first damped-Jacobi sweep from zero (k_jacobi0)
  const double* omega;
  double wscale;
  float w;
  static constexpr int kN = 2;
  static constexpr int kT1 = ST_BF16;
  EDGE_D void init() { w = (float)(__ldg(omega) * wscale); }
  EDGE_D int parity() const { return 0; }
  EDGE_D float value(const float* a0, const void* a1, const void*, int i4, int i2) const {
    return (w * __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(a1)[i2])) * a0[i4];
  }
};
struct InPDir {  // u = z + beta p_old (the first PCG iteration: u = z)
  const PcgState* st;
  float beta;
  int par;
  bool first;
  static constexpr int kN = 2;
  static constexpr int kT1 = ST_F32;
  EDGE_D void init() {
    first = st->iter == 0;
    par = st->iter & 1;
    beta = first ? 0.f : (float)(st->rz_new / st->rz);
  }
  EDGE_D int parity() const { return par; }
  EDGE_D float value(const float* a0, const void* a1, const void*, int i4, int) const {
    return first ? a0[i4] : fmaf(beta, reinterpret_cast<const float*>(a1)[i4], a0[i4]);
  }
};

// The PCG's residual update folded into the V-cycle's first fine launch: b = r_old - alpha q
// (alpha = rz / pq of the previous iteration; FP32 arithmetic of k_pcg_xr32), then
// u = (w Dinv) b, the first damped-Jacobi sweep from zero.  r_old is the residual of a
// ping-pong pair (array 0: the map of the buffer of st->iter's parity), q FP32 (array 1),
// Dinv BF16 (array 2).  No update is pending before the first product (st->pend == 0) or with
// `plain` (the residual was just replaced): b = r_old.
struct InWDBQ {
  const PcgState* st;
  const double* omega;
  double wscale;
  bool plain;
  float w, af;
  bool upd;
  int par;
  static constexpr int kN = 3;
  static constexpr int kT1 = ST_F32;
  static constexpr int kT2 = ST_BF16;
  EDGE_D void init() {
    w = (float)(__ldg(omega) * wscale);
    upd = !plain && st->pend;
    af = upd ? (float)(st->rz_new / st->pq) : 0.f;
    par = st->iter & 1;
  }
  EDGE_D int parity() const { return 0; }
  EDGE_D int parity0() const { return par; }
  EDGE_D float value(const float* a0, const void* a1, const void* a2, int i4, int i2) const {
    const float b = upd ? fmaf(-af, reinterpret_cast<const float*>(a1)[i4], a0[i4]) : a0[i4];
    return (w * __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(a2)[i2])) * b;
  }
};

// Stage layout of the cube kernel: the operator's input array(s) with the k_fine3_pk u-box
// geometry (array 1, when there is one, right after array 0), the element flags and E, then
// the epilogue's staged arrays.
template <int BX, class SE, class IN = InU> struct CubeTile {
  using B = PkTile<BX>;
  static constexpr int ROWS = 4 * BX;  // staged rows: the block's output node rows
  static constexpr int NR = B::NR;     // input rows (with the halo row)
  static constexpr int up(int b) { return (b + 127) & ~127; }
  static constexpr int sbytes(int t) { return 3 * ROWS * st_width(t) * st_esize(t); }
  static constexpr int U0_BYTES = B::U_BYTES;
  static constexpr int U1_BYTES = IN::kN >= 2 ? 3 * NR * st_width(IN::kT1) * st_esize(IN::kT1) : 0;
  static constexpr int U2_BYTES = IN::kN == 3 ? 3 * NR * st_width(in_t2<IN>()) * st_esize(in_t2<IN>()) : 0;
  static constexpr int U1_OFF = up(U0_BYTES);
  static constexpr int U2_OFF = U1_OFF + up(U1_BYTES);
  static constexpr int F_OFF = U2_OFF + up(U2_BYTES);
  static constexpr int E_OFF = F_OFF + up(B::F_BYTES);
  static constexpr int BASE = E_OFF + up(B::E_BYTES);
  static constexpr int s_off(int i) {
    int o = BASE;
    for (int j = 0; j < i; ++j) o += up(sbytes(SE::kT(j)));
    return o;
  }
  static constexpr int tx_bytes() {
    int t = B::TX_BYTES + U1_BYTES + U2_BYTES;
    for (int j = 0; j < SE::kN; ++j) t += sbytes(SE::kT(j));
    return t;
  }
  static constexpr int STAGE = s_off(SE::kN);
  static constexpr int TX_BYTES = tx_bytes();
  static constexpr int X_BYTES = B::X_BYTES;
  static constexpr int UC4 = NR * PK_ZB;               // component stride of an FP32 input array
  static constexpr int UC2 = NR * st_width(ST_BF16);   // ... of a BF16 input array
};

template <int BX, int NS, class SE, class IN = InU>
constexpr int cube_smem_bytes() {
  return NS * CubeTile<BX, SE, IN>::STAGE + CubeTile<BX, SE, IN>::X_BYTES + 128 + 16 * NS;
}

template <class SE, int BX, int NS, int MINB, class IN = InU>
__global__ void __launch_bounds__(32 * BX, MINB)
k_fine3_cube(const Geo g, const __grid_constant__ CUtensorMap mapU, const __grid_constant__ CUtensorMap mapUb,
             const __grid_constant__ CUtensorMap mapU1, const __grid_constant__ CUtensorMap mapU1b,
             const __grid_constant__ CUtensorMap mapU2, const __grid_constant__ CUtensorMap mapF,
             const __grid_constant__ CUtensorMap mapE, const uint8_t* __restrict__ mask,
             const __grid_constant__ CUtensorMap mapS0, const __grid_constant__ CUtensorMap mapS1,
             const __grid_constant__ CUtensorMap mapS2, const __grid_constant__ CUtensorMap mapS3,
             const __grid_constant__ CUtensorMap mapSb, const KCube KC, const int ly, IN in, SE epi, double* part,
             unsigned* ticket, double* dot_dst, int* err) {
  EDGE_PDL_ENTRY();
  static_assert(NS >= 3, "a stage is refilled one layer after its last use");
  using Tile = CubeTile<BX, SE, IN>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  typedef float XArr[2][BX][16][3];
  XArr& sX = *reinterpret_cast<XArr*>(smem + NS * Tile::STAGE);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + NS * Tile::STAGE + Tile::X_BYTES);

  const int lane = threadIdx.x & 31, w = threadIdx.y, tid = threadIdx.x + 32 * w;
  const int zl = lane & 15, xh = lane >> 4;
  const int c0 = 2 * (2 * w + xh);  // first element column of the pair
  const int z0 = blockIdx.x * 15, x0 = blockIdx.y * (4 * BX - 1);
  const int y0 = blockIdx.z * ly;
  const int y1 = min(y0 + ly, g.ny);
  const int ez = z0 - 1 + zl, exa = x0 - 1 + c0;
  const int zs4 = (z0 >= 1) ? ((z0 - 1) & ~3) : -4;
  const int zo4 = (z0 - 1) - zs4;
  const int zs16 = (z0 >= 1) ? ((z0 - 1) & ~15) : -16;
  const int zo16 = (z0 - 1) - zs16;
  const int zs8 = (z0 >= 1) ? ((z0 - 1) & ~7) : -8;
  const int zo8 = (z0 - 1) - zs8;
  const int p0 = y0 - 1;
  const int np = y1 - p0 + 1;
  const bool zok = (zl >= 1) && (ez < g.nz);
  const bool writerA = zok && (c0 >= 1) && (exa < g.nx);
  const bool writerB = zok && (exa + 1 < g.nx);
  in.init();
  epi.init();
  // the array 1 map: the second buffer of a ping-pong pair on odd iterations (InPDir); array 0
  // and the staged array SE::kParS likewise when the input transform / epilogue says so
  const CUtensorMap* map1 = in.parity() ? &mapU1b : &mapU1;
  const CUtensorMap* map0 = &mapU;
  if constexpr (HasPar0<IN>::value) map0 = in.parity0() ? &mapUb : &mapU;
  int spar = 0;
  if constexpr (se_pars<SE>() >= 0) spar = epi.parity();
  bool ok = true;
  P2 kc[8];
  kc[0] = pk(KC.nd, KC.nd);
  kc[1] = pk(KC.no, KC.no);
  kc[2] = pk(KC.sh, KC.sh);
  kc[3] = pk(KC.bd, KC.bd);
  kc[4] = pk(KC.bo, KC.bo);
  kc[5] = pk(KC.td, KC.td);
  kc[6] = pk(KC.to, KC.to);
  kc[7] = pk(KC.h7, KC.h7);

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
    tma_load_4d(st, map0, zs4, x0 - 1, p, 0, &bar[s]);
    if constexpr (IN::kN >= 2)
      tma_load_4d(st + Tile::U1_OFF, map1, IN::kT1 == ST_BF16 ? zs8 : zs4, x0 - 1, p, 0, &bar[s]);
    if constexpr (IN::kN == 3)
      tma_load_4d(st + Tile::U2_OFF, &mapU2, in_t2<IN>() == ST_BF16 ? zs8 : zs4, x0 - 1, p, 0, &bar[s]);
    tma_load_3d(st + Tile::F_OFF, &mapF, zs16, x0 - 1, p, &bar[s]);
    tma_load_3d(st + Tile::E_OFF, &mapE, zs4, x0 - 1, p, &bar[s]);
    const CUtensorMap* ms[4] = {&mapS0, &mapS1, &mapS2, &mapS3};
#pragma unroll
    for (int i = 0; i < SE::kN; ++i)
      tma_load_4d(st + Tile::s_off(i), (i == se_pars<SE>() && spar) ? &mapSb : ms[i],
                  SE::kT(i) == ST_BF16 ? zs8 : zs4, x0 - 1, p, 0, &bar[s]);
  };
  if (tid == 0)
    for (int k = 0; k < NS && k < np; ++k) issue(k);

  constexpr int UC4 = Tile::UC4, UC2 = Tile::UC2;
  const int i4 = c0 * PK_ZB + zo4 + zl;                 // this thread's (row c0, z) in an FP32 input array
  const int i2 = c0 * st_width(ST_BF16) + zo8 + zl;     // ... in a BF16 input array
  const int foff = c0 * PK_FB + zo16 + zl;
  auto a0_of = [&](int k) { return reinterpret_cast<const float*>(smem + (k % NS) * Tile::STAGE); };
  auto a1_of = [&](int k) { return (const void*)(smem + (k % NS) * Tile::STAGE + Tile::U1_OFF); };
  auto a2_of = [&](int k) { return (const void*)(smem + (k % NS) * Tile::STAGE + Tile::U2_OFF); };
  // input value of component c at row offset r (0..2) and z offset dz (0, 1) of plane k; the
  // transform indexes FP32 arrays with the first index and BF16 arrays with the second
  auto input = [&](int k, int c, int r, int dz) {
    return in.value(a0_of(k), a1_of(k), a2_of(k), c * UC4 + r * PK_ZB + dz + i4,
                    c * UC2 + r * st_width(ST_BF16) + dz + i2);
  };

  // The 3 node rows x 2 z of plane p (stage k), masked on constrained DOFs when `fl` says
  // some corner of the pair may be constrained; x-z transformed into t.
  auto load_plane = [&](int k, int p, uint8_t fl, P2 t[2][2][3]) {
    float s[3][2][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int c = 0; c < 3; ++c) s[r][dz][c] = input(k, c, r, dz);
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
    // x stage (scalar, written straight into the pair registers), then z stage (packed)
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        t[0][dz][c] = pk(s[0][dz][c] + s[1][dz][c], s[1][dz][c] + s[2][dz][c]);
        t[1][dz][c] = pk(s[0][dz][c] - s[1][dz][c], s[1][dz][c] - s[2][dz][c]);
      }
#pragma unroll
    for (int hx = 0; hx < 2; ++hx)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const P2 a = t[hx][0][c], b = t[hx][1][c];
        t[hx][0][c] = a + b;
        t[hx][1][c] = a - b;
      }
  };
  auto flags_of = [&](int k, uint8_t& fa, uint8_t& fb) {
    const uint8_t* sf = smem + (k % NS) * Tile::STAGE + Tile::F_OFF + foff;
    fa = sf[0];
    fb = sf[PK_FB];
  };

  P2 pa[2][2][3], pb[2][2][3];  // x-z transforms of two consecutive planes (roles alternate)
  P2 car[2][2][3];              // carry to the next plane; car[0][0] holds the negated value
  if (ok) ok = mbar_wait_fast(&bar[0], 0);
  {
    uint8_t fa, fb;
    flags_of(0, fa, fb);
    load_plane(0, p0, fa | fb, pa);
  }
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c) car[a][b][c] = pk(0.f, 0.f);
  double dacc = 0.0;
  const long long sA_base = g.slot3(max(exa, 0), 0, max(ez, 0));
  const long long sB_base = g.slot3(exa + 1, 0, max(ez, 0));

  // One layer: element row ey = p0 + k between plane k (lo, already transformed) and plane
  // k+1 (loaded into hi); writes the outputs of plane ey.
  auto layer = [&](int k, P2 (&lo)[2][2][3], P2 (&hi)[2][2][3]) {
    const int ey = p0 + k;
    const long long sA = sA_base + (long long)ey * g.plane;
    const long long sB = sB_base + (long long)ey * g.plane;
    const bool wrA = (ey >= y0) && writerA, wrB = (ey >= y0) && writerB;
    if (ok) ok = mbar_wait_fast(&bar[(k + 1) % NS], ((k + 1) / NS) & 1);
    uint8_t fa, fb, fa1, fb1;
    flags_of(k, fa, fb);
    flags_of(k + 1, fa1, fb1);
    const float* sE = reinterpret_cast<const float*>(smem + (k % NS) * Tile::STAGE + Tile::E_OFF) + i4;
    const P2 Ee = pk(sE[0], sE[PK_ZB]);
    load_plane(k + 1, ey + 1, fa | fb | fa1 | fb1, hi);
    P2 uh[8][3];
#pragma unroll
    for (int hx = 0; hx < 2; ++hx)
#pragma unroll
      for (int hz = 0; hz < 2; ++hz)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (hx | hz) uh[hx | (hz << 2)][c] = lo[hx][hz][c] + hi[hx][hz][c];
          uh[hx | 2 | (hz << 2)][c] = lo[hx][hz][c] - hi[hx][hz][c];
        }
    P2 vh[8][3];
    khat_cube(kc, Ee, uh, vh);
    P2 cur[2][2][3];
#pragma unroll
    for (int hx = 0; hx < 2; ++hx)
#pragma unroll
      for (int hz = 0; hz < 2; ++hz)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const P2 b = vh[hx | 2 | (hz << 2)][c];
          if (hx | hz) {
            const P2 a = vh[hx | (hz << 2)][c];
            cur[hx][hz][c] = car[hx][hz][c] + (a + b);
            car[hx][hz][c] = a - b;
          } else {  // a = 0: carry kept as +b, subtracted next layer
            cur[0][0][c] = b - car[0][0][c];
            car[0][0][c] = b;
          }
        }
    wht_xz(cur);  // cur[ax][az][c]: contributions of the pair's two elements to plane ey
    P2 gx[2][3];
#pragma unroll
    for (int ax = 0; ax < 2; ++ax)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float2 up = cur[ax][1][c].v;
        const P2 sh = pk(__shfl_up_sync(0xffffffffu, up.x, 1, 16), __shfl_up_sync(0xffffffffu, up.y, 1, 16));
        gx[ax][c] = cur[ax][0][c] + sh;
      }
    float AuA[3], AuB[3], fromL[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      AuB[c] = gx[1][c].v.x + gx[0][c].v.y;
      fromL[c] = __shfl_up_sync(0xffffffffu, gx[1][c].v.y, 16);
    }
    const int xb = k & 1;
    if (xh == 1)
#pragma unroll
      for (int c = 0; c < 3; ++c) sX[xb][w][zl][c] = gx[1][c].v.y;
    __syncthreads();
    // every thread has finished layer k-1, whose epilogue was the last reader of stage k-1:
    // refill it (with NS >= 3 it is neither stage k nor stage k+1, both still in use)
    if (tid == 0 && k >= 1 && k - 1 + NS < np) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(k - 1 + NS);
    }
    // the output plane's staged epilogue inputs (stage k stays valid until layer k+1)
    typename SE::In inA, inB;
    {
      const unsigned char* st = smem + (k % NS) * Tile::STAGE;
      const unsigned char* spA[4];
      const unsigned char* spB[4];
#pragma unroll
      for (int i = 0; i < SE::kN; ++i) {
        const int t = SE::kT(i);
        const int e = c0 * st_width(t) + (t == ST_BF16 ? zo8 : zo4) + zl;
        spA[i] = st + Tile::s_off(i) + e * st_esize(t);
        spB[i] = spA[i] + st_width(t) * st_esize(t);
      }
      constexpr int cs4 = Tile::ROWS * st_width(ST_F32), cs2 = Tile::ROWS * st_width(ST_BF16);
      const float* in0 = a0_of(k) + i4;
      // array 1 at the node when it is FP32 (the previous search direction, the product q)
      const float* in1 = reinterpret_cast<const float*>(a1_of(k)) + i4;
      if (wrA) inA = epi.load(spA, cs4, cs2, in0, in1, UC4);
      if (wrB) inB = epi.load(spB, cs4, cs2, in0 + PK_ZB, in1 + PK_ZB, UC4);
    }
    if (xh == 0) {
#pragma unroll
      for (int c = 0; c < 3; ++c) fromL[c] = (w > 0) ? sX[xb][w - 1][zl][c] : 0.f;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) AuA[c] = gx[0][c].v.x + fromL[c];
    // each output node's input value, again from stage k (rows c0 and c0 + 1, z = ez);
    // on a constrained DOF the row is the identity: (A u)_c = u_c
    if (wrA) {
      float own[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) own[c] = input(k, c, 0, 0);
      if (fa) {
        const uint8_t m = __ldg(mask + sA);
#pragma unroll
        for (int c = 0; c < 3; ++c)
          if ((m >> c) & 1) AuA[c] = own[c];
      }
      epi.apply(sA, own, AuA, inA, dacc);
    }
    if (wrB) {
      float own[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) own[c] = input(k, c, 1, 0);
      if (fb) {
        const uint8_t m = __ldg(mask + sB);
#pragma unroll
        for (int c = 0; c < 3; ++c)
          if ((m >> c) & 1) AuB[c] = own[c];
      }
      epi.apply(sB, own, AuB, inB, dacc);
    }
  };

  int k = 0;
  for (; k + 2 < np; k += 2) {
    layer(k, pa, pb);
    layer(k + 1, pb, pa);
  }
  if (k + 1 < np) layer(k, pa, pb);
  if (!ok) atomicOr(err, 1);
  if constexpr (HasFin<SE>::value) {
    __shared__ double shf[32];
    const double bt = block_sum(dacc, shf);
    grid_reduce_finish(bt, part, ticket, epi.fin());
  } else {
    finish_dot(epi, dacc, part, ticket, dot_dst);
  }
}

}  // namespace edge
