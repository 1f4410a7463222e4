// Host orchestration and the C ABI (include/edge_b200.h).
//
// Problem = one structured Q4/hex8 mesh with its stiffness operator, BC mask, density,
// multigrid hierarchy and PCG workspace, all allocated at create/config time.
// The solve path (edge_mg_solve / edge_simp_solve_and_process) only launches kernels on
// the problem's stream; the host reads back the PCG state once per iteration to decide
// convergence, exactly where the reference syncs (solvers/_multigrid_cuda.py:223-226).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <cmath>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/edge_b200.h"
#include "coarse.cuh"
#include "common.cuh"
#include "element_op.cuh"
#include "fine_apply.cuh"
#include "fine_tma.cuh"
#include "fine_pk.cuh"
#include "fine_cube.cuh"
#include "general.cuh"
#include "misc.cuh"
#include "tail.cuh"
#include "batch.cuh"

namespace edge {

static thread_local std::string g_err;

struct EdgeError {
  int code;
  std::string msg;
};

#define CK(call)                                                                                  \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess) throw EdgeError{EDGE_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
  } while (0)
#define KCHECK() CK(cudaGetLastError())

static void fail(int code, const std::string& m) { throw EdgeError{code, m}; }

static inline unsigned cdiv(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

// ------------------------------------------------------------------ element matrix analysis
struct ElemInfo {
  int dim = 0, nc = 0, nk = 0;  // corners, matrix size
  double K0b[576];              // bit-order corners
  double kdiag[24];
  bool wht = false;
  KHat3<double> k3{};
  KHat2<double> k2{};
  std::vector<double> Q;  // Galerkin parity tables
};

static const int REF_CORNER3[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                      {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
static const int REF_CORNER2[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};

static double pw_h(int s, int a, int c) {
  return s == 0 ? (a == 0 ? (c == 0 ? 1.0 : 0.0) : 0.5) : (a == 0 ? 0.5 : (c == 1 ? 1.0 : 0.0));
}

static void analyse_element(int dim, const double* K0ref, ElemInfo& ei) {
  ei.dim = dim;
  ei.nc = 1 << dim;
  ei.nk = ei.nc * dim;
  const int nc = ei.nc, nk = ei.nk, d = dim;
  std::vector<int> bit(nc);
  for (int L = 0; L < nc; ++L)
    bit[L] = dim == 3 ? (REF_CORNER3[L][0] | (REF_CORNER3[L][1] << 1) | (REF_CORNER3[L][2] << 2))
                      : (REF_CORNER2[L][0] | (REF_CORNER2[L][1] << 1));
  for (int L1 = 0; L1 < nc; ++L1)
    for (int c1 = 0; c1 < d; ++c1)
      for (int L2 = 0; L2 < nc; ++L2)
        for (int c2 = 0; c2 < d; ++c2)
          ei.K0b[(bit[L1] * d + c1) * nk + bit[L2] * d + c2] = K0ref[(L1 * d + c1) * nk + L2 * d + c2];
  for (int b = 0; b < nc; ++b)
    for (int c = 0; c < d; ++c) ei.kdiag[b * d + c] = ei.K0b[(b * d + c) * nk + b * d + c];
  // transform: Ks = T K0b T / 4^d with T[(h,c),(b,c)] = (-1)^popcount(h&b)
  std::vector<double> tmp(nk * nk, 0.0), Ks(nk * nk, 0.0);
  auto sgn = [](int h, int b) { return (__builtin_popcount(h & b) & 1) ? -1.0 : 1.0; };
  for (int h = 0; h < nc; ++h)
    for (int c = 0; c < d; ++c)
      for (int col = 0; col < nk; ++col) {
        double s = 0;
        for (int b = 0; b < nc; ++b) s += sgn(h, b) * ei.K0b[(b * d + c) * nk + col];
        tmp[(h * d + c) * nk + col] = s;
      }
  const double scale = 1.0 / double(nc * nc);
  double mx = 0.0;
  for (int row = 0; row < nk; ++row)
    for (int h = 0; h < nc; ++h)
      for (int c = 0; c < d; ++c) {
        double s = 0;
        for (int b = 0; b < nc; ++b) s += tmp[row * nk + b * d + c] * sgn(h, b);
        Ks[row * nk + h * d + c] = s * scale;
        mx = std::max(mx, std::fabs(s * scale));
      }
  // pattern check
  bool ok = mx > 0.0;
  double outside = 0.0;
  for (int h = 0; h < nc; ++h)
    for (int c = 0; c < d; ++c)
      for (int h2 = 0; h2 < nc; ++h2)
        for (int c2 = 0; c2 < d; ++c2) {
          bool in = false;
          if (h != 0 && h2 == h && c2 == c) in = true;
          if (h != 0 && c2 != c && (((h >> c) & 1) != ((h >> c2) & 1)) && h2 == (h ^ (1 << c) ^ (1 << c2))) in = true;
          if (!in) outside = std::max(outside, std::fabs(Ks[(h * d + c) * nk + h2 * d + c2]));
        }
  if (outside > 1e-12 * mx) ok = false;
  ei.wht = ok;
  if (dim == 3) {
    for (int c = 0; c < 3; ++c)
      for (int h = 0; h < 8; ++h) {
        ei.k3.dg[c][h] = Ks[(h * 3 + c) * 24 + h * 3 + c];
        for (int c2 = 0; c2 < 3; ++c2) {
          const int h2 = h ^ (1 << c) ^ (1 << c2);
          ei.k3.of[c][c2][h] = (c2 != c) ? Ks[(h * 3 + c) * 24 + h2 * 3 + c2] : 0.0;
        }
      }
  } else {
    for (int c = 0; c < 2; ++c)
      for (int h = 0; h < 4; ++h) {
        ei.k2.dg[c][h] = Ks[(h * 2 + c) * 8 + h * 2 + c];
        for (int c2 = 0; c2 < 2; ++c2) {
          const int h2 = h ^ 3;
          ei.k2.of[c][c2][h] = (c2 != c) ? Ks[(h * 2 + c) * 8 + h2 * 2 + c2] : 0.0;
        }
      }
  }
  // Galerkin parity tables Q_s = P_s^T K0b P_s
  const int npar = nc;
  ei.Q.assign((size_t)npar * nk * nk, 0.0);
  for (int s = 0; s < npar; ++s) {
    std::vector<double> P(nc * nc);
    for (int a = 0; a < nc; ++a)
      for (int cI = 0; cI < nc; ++cI) {
        double w = 1.0;
        for (int q = 0; q < d; ++q) w *= pw_h((s >> q) & 1, (a >> q) & 1, (cI >> q) & 1);
        P[a * nc + cI] = w;
      }
    for (int cI = 0; cI < nc; ++cI)
      for (int c = 0; c < d; ++c)
        for (int cJ = 0; cJ < nc; ++cJ)
          for (int e = 0; e < d; ++e) {
            double v = 0.0;
            for (int a = 0; a < nc; ++a) {
              if (P[a * nc + cI] == 0.0) continue;
              for (int b = 0; b < nc; ++b) {
                if (P[b * nc + cJ] == 0.0) continue;
                v += P[a * nc + cI] * ei.K0b[(a * d + c) * nk + b * d + e] * P[b * nc + cJ];
              }
            }
            ei.Q[(size_t)s * nk * nk + (cI * d + c) * nk + cJ * d + e] = v;
          }
  }
}

template <typename T> static KHat3<T> cast3(const KHat3<double>& k) {
  KHat3<T> o;
  for (int c = 0; c < 3; ++c)
    for (int h = 0; h < 8; ++h) {
      o.dg[c][h] = (T)k.dg[c][h];
      for (int d = 0; d < 3; ++d) o.of[c][d][h] = (T)k.of[c][d][h];
    }
  return o;
}
template <typename T> static KHat2<T> cast2(const KHat2<double>& k) {
  KHat2<T> o;
  for (int c = 0; c < 2; ++c)
    for (int h = 0; h < 4; ++h) {
      o.dg[c][h] = (T)k.dg[c][h];
      for (int d = 0; d < 2; ++d) o.of[c][d][h] = (T)k.of[c][d][h];
    }
  return o;
}

// ------------------------------------------------------------------ problem
struct Level {
  Geo g;
  void *b = nullptr, *xa = nullptr, *xb = nullptr, *r = nullptr, *ea = nullptr, *eb = nullptr, *res = nullptr;
  void* S = nullptr;     // stencil (l >= 1)
  void* S16 = nullptr;   // BF16 copy of the FP32 stencil, applied when Prob::st_bf16 is set
  void* S16t = nullptr;  // tile-major BF16 pair copy for k_st3_apply2t (3-D levels of at least st_tile_min slots)
  void* dinv = nullptr;  // Jacobi inverse diagonal
};

struct Prob {
  int dim = 0, nel[3] = {1, 1, 1}, prec = EDGE_FP64;
  Geo g0;
  long long n_el = 0, n_dof = 0;
  ElemInfo ei;
  cudaStream_t stream = 0;
  std::vector<void*> allocs;
  // element / operator data
  double* dK0b = nullptr;
  double* dK0ref = nullptr;  // element matrix in the reference's corner order
  float* dK0bf = nullptr;
  double* dK0diag = nullptr;
  double* dQ = nullptr;
  uint8_t* mask = nullptr;
  uint8_t* eflag16 = nullptr;  // element flags with rows padded to 16 bytes (TMA source)
  int mpz = 0;
  uint8_t* eflag = nullptr;
  int* err = nullptr;          // set by kernels whose bounded waits expired
  bool use_tma = true;
  int tile_variant = 0;    // k_fine3_tma (BX, NS): 0 (8,4) 1 (8,3) 2 (8,2) 3 (4,4) 4 (4,3);
                           // FP32 only, k_fine3_pk (BX, NS, min blocks/SM): 5 (4,3,1) 6 (4,3,4)
                           // 7 (2,3,8) 8 (4,4,4); FP32 cube elements only, k_fine3_cube:
                           // 9 (4,3,2) 10 (4,4,2) 11 (2,3,4) 12 (8,3,1) 13 (4,3,4) 14 (4,4,4)
  KHat3P k3p;              // packed transformed element operator (FP32 pairs)
  KCube kcube;             // block form of the same operator (cube elements)
  bool cube = false;       // kcube reproduces every entry of the transformed operator
  int blocks_per_sm = 4;   // y-chunking target of the fine kernel
  // per kind of fused cube launch (0: first sweep + residual, 1: last sweep + correction,
  // 2: search direction + product), the tile variant and y-chunking target chosen for that
  // launch alone; -1: tile_variant / blocks_per_sm
  int kind_variant[3] = {-1, -1, -1};
  int kind_bps[3] = {0, 0, 0};
  bool kind_tune = true;  // edge_autotune_fine also picks the per-kind tiles
  long long st_quad_max = 40000;   // 3-D stencil levels with at most this many slots use k_st3_apply_q
  bool st_bf16 = true;             // mixed precision: apply the coarse stencils from BF16 copies
  // mixed precision: the residual recurrence between FP64 replacements is stored in FP32
  // (arithmetic and r.r in FP64); false keeps an FP64 recurrence with an FP32 copy
  bool res32 = true;
  // solve graph: kernels launched with programmatic stream serialization (each kernel's
  // blocks may be scheduled while its predecessor drains; every kernel waits on entry).
  // Off by default: at 12.8M DOF the SIMP loop ran 1.5 % slower with it.
  bool pdl = false;
  bool capturing = false;  // set while capture_solve records the solve graph
  // FP32 3-D levels with at least st_pair_min slots: two nodes per thread (k_st3_apply2;
  // 21 % faster than one node per thread at 570 k slots, slower at 75 k and in FP64)
  bool st_pair = true;
  long long st_pair_min = 200000;
  // mixed precision, 3-D, two nodes per thread: levels with at least st_tile_min slots at
  // hierarchy allocation keep a tile-major BF16 pair copy and are applied by k_st3_apply2t
  // (st_tile_min < 0: off).  At 570 k slots (level 1 of 12.8M DOF) the SIMP step ran 1.7 %
  // faster than with k_st3_apply2 on the linear copy (167.5 against 170.4 ms, same PCG counts).
  long long st_tile_min = 200000;
  // CUDA graph of one solve (hierarchy set-up + the whole PCG loop under a while node)
  bool use_graph = true;
  cudaGraph_t sg_graph = nullptr;
  cudaGraphExec_t sg_exec = nullptr;
  // one SIMP iteration (OC update + analysis) as one graph over owned buffers
  cudaGraph_t it_graph = nullptr;
  cudaGraphExec_t it_exec = nullptr;
  std::vector<double> it_key;
  long long it_fixed = 0, it_oc_body = 0, it_body = 0, it_rep = 0;
  double *it_rho = nullptr, *it_dr = nullptr, *it_rho_new = nullptr, *it_dr_new = nullptr;
  std::vector<double> sg_key;
  long long sg_pro = 0, sg_body = 0, sg_if = 0;  // launches per section, for the launch tally
  cudaStream_t cap[3] = {nullptr, nullptr, nullptr};
  std::string graph_error;
  // grounded point springs (slot-layout flat index, user DOF index, stiffness)
  static constexpr int MAX_SPRINGS = 64;
  int n_springs = 0;
  long long* spr_flat = nullptr;
  long long* spr_user = nullptr;
  double* spr_k = nullptr;
  std::map<std::pair<const void*, int>, CUtensorMap> tmaps;
  double* E64 = nullptr;
  float* E32 = nullptr;
  bool has_rho = false, has_cons = false;
  // MG configuration
  int n_level = -1, n_smooth = 3;
  std::vector<int> level_sweeps;  // per-level sweep counts (pre = post); levels past its end use n_smooth
  int sweeps(int l) const { return l < (int)level_sweeps.size() ? level_sweeps[l] : n_smooth; }
  double omega = 0.5, min_omega = 0.4;
  // smoother weight across solves: false = reset every solve (the GPU solver), true = carried
  // over from the previous solve (the CPU solver); omega_started: a solve has run since set
  bool omega_carry = false, omega_started = false;
  // mixed path: fused fine launches (first sweep + residual in one launch, the last sweep
  // without a stored pre-smoothed iterate, the search direction formed inside the product)
  bool fuse = true;
  // mixed path with a fixed smoother weight and the fused fine launches: the PCG's x/r update
  // folded into the next iteration's first fine launch (residual) and search-direction launch
  // (solution); r32b is the second buffer of the FP32 residual's ping-pong pair.  Off by
  // default: at 12.8M DOF the two launches grew by 50 and 31 us (their third staged array and
  // the extra registers cost occupancy), more than the 50 us update launch they replace.
  bool fuse_xr = false;
  float* r32b = nullptr;
  // mixed path, 3-D: the V-cycle from level tail_l0 down (sweeps, residuals, transfers and
  // the coarsest solve) as one persistent cooperative launch; 0 = off (the default: at 12.8M
  // DOF the launch took longer than the per-step launches it replaces)
  int tail_l0 = 0;
  unsigned* tail_bar = nullptr;  // grid barrier of that launch (count, generation)
  int tail_blocks = 0;
  bool cycle_w = false;
  std::vector<int> w_levels;
  std::vector<Level> lv;
  int nd = 0;
  double *Adense = nullptr, *Ainv = nullptr, *Ut = nullptr;
  // 3-D Galerkin products of the stencil levels as three one-axis passes (k_galerkin3_axis)
  // through two FP64 intermediates sized for the level 1 -> 2 product; false: k_galerkin3_st
  bool gal_axis = true;
  double *gal_t1 = nullptr, *gal_t2 = nullptr;
  int* chol_status = nullptr;
  // PCG (level 0) vectors, FP64 slots
  double *b64 = nullptr, *x64 = nullptr, *r64 = nullptr;
  void *p = nullptr, *q = nullptr;  // type T of the precision mode
  float* r32 = nullptr;
  float* x32 = nullptr;  // mixed path: FP32 solution increment since the last replacement
  // user-layout scratch for the fused SIMP step
  double *rho_f = nullptr, *gsens = nullptr;
  // reductions
  double* part = nullptr;
  unsigned* ticket = nullptr;
  PcgState* st = nullptr;
  PcgState* st_h = nullptr;  // pinned
  OcState* oc = nullptr;
  OcState* oc_h = nullptr;
  double* ocp = nullptr;
  double* scal = nullptr;    // device scalars
  double* scal_h = nullptr;  // pinned
  int* zero_int = nullptr;
  // stats
  cudaEvent_t ev[4];
  double last_setup_ms = 0, last_solve_ms = 0;
  int last_iters = 0, last_true_res = 0;
  size_t part_cap = 0;
  long long nlaunch = 0;
  // fine-operator profiling (CUDA events around each launch + algorithmic bytes)
  bool prof = false;
  std::vector<cudaEvent_t> pev;
  std::vector<double> pbytes;
  size_t pev_used = 0;
  // per-category time breakdown of every launch (benchmark instrumentation)
  bool bd = false;
  int cur_cat = 0;
  std::vector<cudaEvent_t> bev;
  std::vector<int> bcat;
  size_t bev_used = 0;

  template <typename T> T* alloc(size_t n) {
    void* ptr = nullptr;
    CK(cudaMalloc(&ptr, std::max<size_t>(n, 1) * sizeof(T)));
    CK(cudaMemset(ptr, 0, std::max<size_t>(n, 1) * sizeof(T)));
    allocs.push_back(ptr);
    return (T*)ptr;
  }
  ~Prob() {
    if (sg_exec) cudaGraphExecDestroy(sg_exec);
    if (sg_graph) cudaGraphDestroy(sg_graph);
    if (it_exec) cudaGraphExecDestroy(it_exec);
    if (it_graph) cudaGraphDestroy(it_graph);
    for (int i = 0; i < 3; ++i)
      if (cap[i]) cudaStreamDestroy(cap[i]);
    for (void* a : allocs) cudaFree(a);
    if (st_h) cudaFreeHost(st_h);
    if (oc_h) cudaFreeHost(oc_h);
    if (scal_h) cudaFreeHost(scal_h);
    for (int i = 0; i < 4; ++i) cudaEventDestroy(ev[i]);
    for (auto e : pev) cudaEventDestroy(e);
    for (auto e : bev) cudaEventDestroy(e);
  }
};


// Every kernel launch of the solve path goes through here: counted for the benchmark's
// launch tally and checked immediately.
template <typename... KArgs, typename... Args>
static void launch(Prob& P, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, Args... args) {
  const bool rec = P.bd && P.bev_used + 2 <= P.bev.size();
  if (rec) CK(cudaEventRecord(P.bev[P.bev_used], P.stream));
  if (P.pdl && P.capturing) {  // only on the library's own capture streams
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = P.stream;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...));
  } else {
    kern<<<grid, block, smem, P.stream>>>(static_cast<KArgs>(args)...);
  }
  ++P.nlaunch;
  KCHECK();
  if (rec) {
    CK(cudaEventRecord(P.bev[P.bev_used + 1], P.stream));
    P.bev_used += 2;
    P.bcat.push_back(P.cur_cat);
  }
}

// Launch categories of the breakdown instrumentation.
enum { CAT_OTHER = 0, CAT_FINE, CAT_STENCIL, CAT_TRANSFER, CAT_VECTOR, CAT_SETUP, CAT_COARSE, CAT_OC, CAT_SENS,
       CAT_COUNT };
struct CatScope {
  Prob& P;
  int old;
  CatScope(Prob& p, int c) : P(p), old(p.cur_cat) { P.cur_cat = c; }
  ~CatScope() { P.cur_cat = old; }
};

// The 3-D fine level pads z to 8 nodes so that its BF16 rows (the Jacobi diagonal) are
// 16-byte aligned TMA sources; coarser levels and 2-D pad to 4.
static int fine_zalign(int dim, int level) { return (dim == 3 && level == 0) ? 8 : 4; }

// Grids between the one-axis Galerkin passes from gf to gc: x coarsened (g1), then x and y (g2);
// both keep the fine z padding.
static void gal_axis_geos(const Geo& gf, const Geo& gc, Geo& g1, Geo& g2) {
  g1 = gf;
  g1.nx = gc.nx;
  g1.plane = (long long)g1.nx * g1.pz;
  g1.n = (long long)g1.ny * g1.plane;
  g2 = g1;
  g2.ny = gc.ny;
  g2.n = (long long)g2.ny * g2.plane;
}

static Geo level_geo(const Prob& P, int l) {
  int ne[3] = {P.nel[0], P.nel[1], P.nel[2]};
  for (int i = 0; i < l; ++i)
    for (int d = 0; d < 3; ++d) ne[d] /= 2;
  return make_geo(P.dim, ne[0], ne[1], P.dim == 3 ? ne[2] : 0, fine_zalign(P.dim, l));
}

// ------------------------------------------------------------------ TMA tensor maps
static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

// Queried once per process (problems may live on different host threads).
static void get_encode() {
  static std::once_flag once;
  std::call_once(once, []() {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess && fn)
      g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  });
  if (!g_encode) fail(EDGE_ECUDA, "cuTensorMapEncodeTiled not available");
}

static CUtensorMap encode_map(const void* base, CUtensorMapDataType dt, int rank, const uint64_t* dims,
                              const uint64_t* strides, const uint32_t* box) {
  get_encode();
  CUtensorMap m;
  uint32_t es[5] = {1, 1, 1, 1, 1};
  CUresult r = g_encode(&m, dt, rank, const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(EDGE_ECUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return m;
}

template <typename T> static CUtensorMapDataType tma_dt() {
  return sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
}

// kind 0: 3-component fine vector (box 48 x (BX+1) x 1 x 3); 1: fine element array (48 x BX x 1)
template <typename T, int BX>
static const CUtensorMap& fine_map(Prob& P, const T* base, int kind) {
  auto key = std::make_pair((const void*)base, kind * 16 + (int)sizeof(T) + 100 * BX);
  auto it = P.tmaps.find(key);
  if (it != P.tmaps.end()) return it->second;
  const Geo& g = P.g0;
  const uint64_t sz = sizeof(T);
  CUtensorMap m;
  if (kind == 0) {
    uint64_t dims[4] = {(uint64_t)g.pz, (uint64_t)g.nx, (uint64_t)g.ny, 3};
    uint64_t str[3] = {g.pz * sz, g.plane * sz, g.n * sz};
    uint32_t box[4] = {TMA_ZB, 2 * BX + 1, 1, 3};
    m = encode_map(base, tma_dt<T>(), 4, dims, str, box);
  } else {
    uint64_t dims[3] = {(uint64_t)g.pz, (uint64_t)g.nx, (uint64_t)g.ny};
    uint64_t str[2] = {g.pz * sz, g.plane * sz};
    uint32_t box[3] = {TMA_ZB, 2 * BX, 1};
    m = encode_map(base, tma_dt<T>(), 3, dims, str, box);
  }
  return P.tmaps.emplace(key, m).first->second;
}

template <int BX>
static const CUtensorMap& flag_map(Prob& P) {
  auto key = std::make_pair((const void*)P.eflag16, 1000 + BX);
  auto it = P.tmaps.find(key);
  if (it != P.tmaps.end()) return it->second;
  const Geo& g = P.g0;
  uint64_t dims[3] = {(uint64_t)P.mpz, (uint64_t)g.nx, (uint64_t)g.ny};
  uint64_t str[2] = {(uint64_t)P.mpz, (uint64_t)P.mpz * g.nx};
  uint32_t box[3] = {TMA_ZB, 2 * BX, 1};
  return P.tmaps.emplace(key, encode_map(P.eflag16, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, dims, str, box)).first->second;
}

// Maps of the packed-pair kernel (FP32): u box 24 x (4BX+1) x 1 x 3, E box 24 x 4BX x 1,
// flags 48 x 4BX x 1.
template <int BX>
static const CUtensorMap& pk_map(Prob& P, const float* base, int kind) {
  auto key = std::make_pair((const void*)base, 2000 + kind * 16 + BX);
  auto it = P.tmaps.find(key);
  if (it != P.tmaps.end()) return it->second;
  const Geo& g = P.g0;
  const uint64_t sz = sizeof(float);
  CUtensorMap m;
  if (kind == 0) {
    uint64_t dims[4] = {(uint64_t)g.pz, (uint64_t)g.nx, (uint64_t)g.ny, 3};
    uint64_t str[3] = {g.pz * sz, g.plane * sz, g.n * sz};
    uint32_t box[4] = {PK_ZB, 4 * BX + 1, 1, 3};
    m = encode_map(base, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, dims, str, box);
  } else {
    uint64_t dims[3] = {(uint64_t)g.pz, (uint64_t)g.nx, (uint64_t)g.ny};
    uint64_t str[2] = {g.pz * sz, g.plane * sz};
    uint32_t box[3] = {PK_ZB, 4 * BX, 1};
    m = encode_map(base, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, dims, str, box);
  }
  return P.tmaps.emplace(key, m).first->second;
}

template <int BX>
static const CUtensorMap& pk_flag_map(Prob& P) {
  auto key = std::make_pair((const void*)P.eflag16, 3000 + BX);
  auto it = P.tmaps.find(key);
  if (it != P.tmaps.end()) return it->second;
  const Geo& g = P.g0;
  uint64_t dims[3] = {(uint64_t)P.mpz, (uint64_t)g.nx, (uint64_t)g.ny};
  uint64_t str[2] = {(uint64_t)P.mpz, (uint64_t)P.mpz * g.nx};
  uint32_t box[3] = {PK_FB, 4 * BX, 1};
  return P.tmaps.emplace(key, encode_map(P.eflag16, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, dims, str, box)).first->second;
}

static KHat3P pack3(const KHat3<double>& k) {
  KHat3P o;
  for (int c = 0; c < 3; ++c)
    for (int h = 0; h < 8; ++h) {
      const float a = (float)k.dg[c][h];
      o.dg[c][h].v = make_float2(a, a);
      for (int d = 0; d < 3; ++d) {
        const float b = (float)k.of[c][d][h];
        o.of[c][d][h].v = make_float2(b, b);
      }
    }
  return o;
}

// Block form of a cube element's transformed operator (fine_cube.cuh): read the eight
// coefficients off KHat3 and accept them only if the model reproduces all 576 entries.
static bool cube_form(const KHat3<double>& k, KCube& out) {
  const double nd = k.dg[0][1], no = k.of[0][1][1], sh = k.dg[1][1], bd = k.dg[0][3], bo = k.of[0][2][3],
               td = k.dg[2][3], to = k.of[2][1][3], h7 = k.dg[0][7];
  // model entries: M[(h,c)][(h2,c2)]
  double M[8][3][8][3] = {};
  auto set_sym = [&](int h1, int c1, int h2, int c2, double v) {
    M[h1][c1][h2][c2] = v;
    M[h2][c2][h1][c1] = v;
  };
  const int N[3][2] = {{1, 0}, {2, 1}, {4, 2}}, TW[3][2] = {{3, 2}, {5, 1}, {6, 0}};
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      M[N[a][0]][N[a][1]][N[b][0]][N[b][1]] = a == b ? nd : no;
      M[TW[a][0]][TW[a][1]][TW[b][0]][TW[b][1]] = a == b ? td : to;
    }
  const int SH[3][4] = {{1, 1, 2, 0}, {1, 2, 4, 0}, {2, 2, 4, 1}}, BE[3][4] = {{3, 0, 6, 2}, {3, 1, 5, 2}, {5, 0, 6, 1}};
  for (int i = 0; i < 3; ++i) {
    M[SH[i][0]][SH[i][1]][SH[i][0]][SH[i][1]] = sh;
    M[SH[i][2]][SH[i][3]][SH[i][2]][SH[i][3]] = sh;
    set_sym(SH[i][0], SH[i][1], SH[i][2], SH[i][3], sh);
    M[BE[i][0]][BE[i][1]][BE[i][0]][BE[i][1]] = bd;
    M[BE[i][2]][BE[i][3]][BE[i][2]][BE[i][3]] = bd;
    set_sym(BE[i][0], BE[i][1], BE[i][2], BE[i][3], bo);
  }
  for (int c = 0; c < 3; ++c) M[7][c][7][c] = h7;
  // actual entries from KHat3 (diagonal + the coupling pattern), zero elsewhere
  double mx = 0.0, dev = 0.0;
  for (int h = 0; h < 8; ++h)
    for (int c = 0; c < 3; ++c)
      for (int h2 = 0; h2 < 8; ++h2)
        for (int c2 = 0; c2 < 3; ++c2) {
          double a = 0.0;
          if (h2 == h && c2 == c) a = k.dg[c][h];
          else if (c2 != c && h2 == (h ^ (1 << c) ^ (1 << c2)) && (((h >> c) & 1) != ((h >> c2) & 1))) a = k.of[c][c2][h];
          mx = std::max(mx, std::fabs(a));
          dev = std::max(dev, std::fabs(a - M[h][c][h2][c2]));
        }
  if (!(mx > 0.0) || dev > 1e-12 * mx) return false;
  out = KCube{(float)(nd - no), (float)no, (float)sh, (float)bd, (float)bo, (float)(td - to), (float)to, (float)h7};
  return true;
}

static size_t vbytes(int prec) { return prec == EDGE_FP64 ? sizeof(double) : sizeof(float); }

// ------------------------------------------------------------------ launch helpers
static const int FINE_BX = 8;
static const int FINE2_NW = 4;

static dim3 fine3_grid(const Geo& g, int& ly) {
  const unsigned tz = cdiv(g.nz, 31), tx = cdiv(g.nx, FINE_BX - 1);
  const long long want = 148LL * 4;
  long long chunks = std::max<long long>(1, (want + (long long)tz * tx - 1) / ((long long)tz * tx));
  chunks = std::min<long long>(chunks, g.ny);
  ly = (int)cdiv(g.ny, chunks);
  return dim3(tz, tx, cdiv(g.ny, ly));
}
static dim3 fine3_grid_v3(const Geo& g, int bx, int& ly) {
  const unsigned tz = cdiv(g.nz, 15), tx = cdiv(g.nx, 2 * bx - 1);
  const long long want = 148LL * 4;
  long long chunks = std::max<long long>(1, (want + (long long)tz * tx - 1) / ((long long)tz * tx));
  chunks = std::min<long long>(chunks, g.ny);
  ly = (int)cdiv(g.ny, chunks);
  return dim3(tz, tx, cdiv(g.ny, ly));
}
static dim3 fine2_grid(const Geo& g, int& ly) {
  const unsigned tx = cdiv(g.nx, 32 * FINE2_NW - 1);
  const long long want = 148LL * 8;
  long long chunks = std::max<long long>(1, (want + tx - 1) / tx);
  chunks = std::min<long long>(chunks, g.ny);
  ly = (int)cdiv(g.ny, chunks);
  return dim3(tx, cdiv(g.ny, ly));
}

template <typename T> struct TypeOps;
template <> struct TypeOps<double> {
  static const double* E(const Prob& P) { return P.E64; }
  static const double* K0b(const Prob& P) { return P.dK0b; }
};
template <> struct TypeOps<float> {
  static const float* E(const Prob& P) { return P.E32; }
  static const float* K0b(const Prob& P) { return P.dK0bf; }
};

// One launch of the TMA fine kernel with BX warps and NS stages per block; the number of
// y-chunks follows P.blocks_per_sm (the grid aims at that many resident blocks per SM).
template <typename T, class Epi, int BX, int NS>
static void fine3_tma_launch(Prob& P, const T* u, const T* E, Epi epi, double* dot_dst) {
  const Geo& g = P.g0;
  constexpr int smem = tma_smem_bytes<T, BX, NS>();
  static std::atomic<bool> attr{false};  // setting the attribute twice is harmless
  if (!attr.load()) {
    CK(cudaFuncSetAttribute(k_fine3_tma<T, Epi, BX, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr = true;
  }
  const unsigned tz = cdiv(g.nz, 15), tx = cdiv(g.nx, 2 * BX - 1);
  const long long want = 148LL * P.blocks_per_sm;
  long long chunks = std::max<long long>(1, (want + (long long)tz * tx - 1) / ((long long)tz * tx));
  chunks = std::min<long long>(chunks, g.ny);
  const int ly = (int)cdiv(g.ny, chunks);
  launch(P, k_fine3_tma<T, Epi, BX, NS>, dim3(tz, tx, cdiv(g.ny, ly)), dim3(32, BX), smem, g,
         fine_map<T, BX>(P, u, 0), flag_map<BX>(P), fine_map<T, BX>(P, E, 1), u, (const uint8_t*)P.mask,
         cast3<T>(P.ei.k3), ly, epi, P.part, P.ticket, dot_dst, P.err);
}

// One launch of the packed-pair FP32 kernel (BX warps, NS stages).
template <class Epi, int BX, int NS, int MINB>
static void fine3_pk_launch(Prob& P, const float* u, const float* E, Epi epi, double* dot_dst) {
  const Geo& g = P.g0;
  constexpr int smem = pk_smem_bytes<BX, NS>();
  static std::atomic<bool> attr{false};  // setting the attribute twice is harmless
  if (!attr.load()) {
    CK(cudaFuncSetAttribute(k_fine3_pk<Epi, BX, NS, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr = true;
  }
  const unsigned tz = cdiv(g.nz, 15), tx = cdiv(g.nx, 4 * BX - 1);
  const long long want = 148LL * P.blocks_per_sm;
  long long chunks = std::max<long long>(1, (want + (long long)tz * tx - 1) / ((long long)tz * tx));
  chunks = std::min<long long>(chunks, g.ny);
  const int ly = (int)cdiv(g.ny, chunks);
  launch(P, k_fine3_pk<Epi, BX, NS, MINB>, dim3(tz, tx, cdiv(g.ny, ly)), dim3(32, BX), smem, g, pk_map<BX>(P, u, 0),
         pk_flag_map<BX>(P), pk_map<BX>(P, E, 1), u, (const uint8_t*)P.mask, P.k3p, ly, epi, P.part, P.ticket,
         dot_dst, P.err);
}

// Staged form (fine_cube.cuh) of the solver's FP32 fine-level epilogues; `arr` receives the
// arrays the kernel stages through TMA, in the order of SE::kT.
template <class Epi> struct StagedOf {
  static constexpr bool ok = false;
};
template <class Epi> static bool staged_usable(const Epi& e) {
  if constexpr (StagedOf<Epi>::ok) {
    if constexpr (std::is_same<typename StagedOf<Epi>::SE, SEJacobiAdd<true>>::value ||
                  std::is_same<typename StagedOf<Epi>::SE, SEJacobiAdd<false>>::value)
      return StagedOf<Epi>::usable(e);
    return true;
  }
  return false;
}
template <> struct StagedOf<EpiStore<float, float>> {
  static constexpr bool ok = true;
  using SE = SEStore;
  static SE make(const EpiStore<float, float>& e, const void**) { return SE{e.out, e.n}; }
};
template <> struct StagedOf<EpiStoreDot<float>> {
  static constexpr bool ok = true;
  using SE = SEStoreDot;
  static SE make(const EpiStoreDot<float>& e, const void**) { return SE{e.out, e.n}; }
};
template <> struct StagedOf<EpiResid<float, float, float>> {
  static constexpr bool ok = true;
  using SE = SEResid;
  static SE make(const EpiResid<float, float, float>& e, const void** arr) {
    arr[0] = e.b;
    return SE{e.r, e.n};
  }
};
template <> struct StagedOf<EpiJacobi<float, float, __nv_bfloat16>> {
  static constexpr bool ok = true;
  using SE = SEJacobi;
  static SE make(const EpiJacobi<float, float, __nv_bfloat16>& e, const void** arr) {
    arr[0] = e.b;
    arr[1] = e.dinv;
    return SE{e.xo, e.omega, e.wscale, e.n, 0.f};
  }
};
template <bool DOT, typename TV> struct StagedOf<EpiJacobiAdd<float, float, __nv_bfloat16, float, DOT, TV>> {
  static constexpr bool ok = true;
  using SE = SEJacobiAdd<DOT>;
  using Epi = EpiJacobiAdd<float, float, __nv_bfloat16, float, DOT, TV>;
  // the staged form stages an FP32 dot vector
  static bool usable(const Epi&) { return !DOT || std::is_same<TV, float>::value; }
  static SE make(const Epi& e, const void** arr) {
    arr[0] = e.b;
    arr[1] = e.dinv;
    arr[2] = e.xbase;
    if constexpr (DOT) arr[3] = e.dotv;
    return SE{e.xo, e.omega, e.wscale, e.n, 0.f};
  }
};

// Tensor map of a staged epilogue array [3][n] (slot layout) of element type t: boxes of
// st_width(t) z-nodes x 4*BX node rows x 1 plane x 3 components.
template <int BX>
static const CUtensorMap& stage_map(Prob& P, const void* base, int t) {
  auto key = std::make_pair(base, 4000 + t * 16 + BX);
  auto it = P.tmaps.find(key);
  if (it != P.tmaps.end()) return it->second;
  const Geo& g = P.g0;
  const uint64_t sz = (uint64_t)st_esize(t);
  const CUtensorMapDataType dt = t == ST_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                 : t == ST_F64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                               : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  uint64_t dims[4] = {(uint64_t)g.pz, (uint64_t)g.nx, (uint64_t)g.ny, 3};
  uint64_t str[3] = {g.pz * sz, g.plane * sz, g.n * sz};
  uint32_t box[4] = {(uint32_t)st_width(t), 4 * BX, 1, 3};
  return P.tmaps.emplace(key, encode_map(base, dt, 4, dims, str, box)).first->second;
}

// Map of an operator-input array of the cube kernel (u-box geometry, with the halo row):
// FP32 24 x (4BX+1) x 1 x 3 (the packed-pair u map), BF16 32 x (4BX+1) x 1 x 3.
template <int BX>
static const CUtensorMap& in_map(Prob& P, const void* base, int t) {
  if (t != ST_BF16) return pk_map<BX>(P, (const float*)base, 0);
  auto key = std::make_pair(base, 5000 + BX);
  auto it = P.tmaps.find(key);
  if (it != P.tmaps.end()) return it->second;
  const Geo& g = P.g0;
  uint64_t dims[4] = {(uint64_t)g.pz, (uint64_t)g.nx, (uint64_t)g.ny, 3};
  uint64_t str[3] = {(uint64_t)g.pz * 2, (uint64_t)g.plane * 2, (uint64_t)g.n * 2};
  uint32_t box[4] = {(uint32_t)st_width(ST_BF16), 4 * BX + 1, 1, 3};
  return P.tmaps.emplace(key, encode_map(base, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, dims, str, box)).first->second;
}

// One launch of the cube kernel: input transform IN over arrays in0 (FP32) and in1 (IN::kT1;
// in1b its second ping-pong buffer, or null), staged epilogue arrays arr[0..SE::kN).
// Alternative and third arrays of a cube launch: in0b, the other buffer of input array 0's
// ping-pong pair (IN::parity0); in2, input array 2 (IN::kN == 3); sb, the other buffer of the
// staged array SE::kParS.
struct CubeExtra {
  const float* in0b = nullptr;
  const void* in2 = nullptr;
  const void* sb = nullptr;
};

template <class SE, class IN, int BX, int NS, int MINB>
static void fine3_cube_go(Prob& P, const float* in0, const void* in1, const void* in1b, const float* E, IN in,
                          SE epi, const void* const* arr, double* dot_dst, const CubeExtra& xa = {}) {
  const Geo& g = P.g0;
  constexpr int smem = cube_smem_bytes<BX, NS, SE, IN>();
  static_assert(smem <= 227 * 1024, "cube kernel stage ring exceeds shared memory");
  static std::atomic<bool> attr{false};  // setting the attribute twice is harmless
  if (!attr.load()) {
    CK(cudaFuncSetAttribute(k_fine3_cube<SE, BX, NS, MINB, IN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr = true;
  }
  const CUtensorMap& m0 = pk_map<BX>(P, in0, 0);
  const CUtensorMap& m0b = xa.in0b ? pk_map<BX>(P, xa.in0b, 0) : m0;
  const CUtensorMap& m1 = IN::kN >= 2 ? in_map<BX>(P, in1, IN::kT1) : m0;
  const CUtensorMap& m1b = (IN::kN >= 2 && in1b) ? in_map<BX>(P, in1b, IN::kT1) : m1;
  const CUtensorMap& m2 = IN::kN == 3 ? in_map<BX>(P, xa.in2, in_t2<IN>()) : m0;
  const CUtensorMap* ms[4];
  for (int i = 0; i < 4; ++i) ms[i] = i < SE::kN ? &stage_map<BX>(P, arr[i], SE::kT(i)) : &m0;
  constexpr int ps = se_pars<SE>();
  const CUtensorMap* msb = &m0;
  if constexpr (ps >= 0 && ps < SE::kN) msb = xa.sb ? &stage_map<BX>(P, xa.sb, SE::kT(ps)) : ms[ps];
  const unsigned tz = cdiv(g.nz, 15), tx = cdiv(g.nx, 4 * BX - 1);
  const long long want = 148LL * P.blocks_per_sm;
  long long chunks = std::max<long long>(1, (want + (long long)tz * tx - 1) / ((long long)tz * tx));
  chunks = std::min<long long>(chunks, g.ny);
  const int ly = (int)cdiv(g.ny, chunks);
  launch(P, k_fine3_cube<SE, BX, NS, MINB, IN>, dim3(tz, tx, cdiv(g.ny, ly)), dim3(32, BX), smem, g, m0, m0b, m1,
         m1b, m2, pk_flag_map<BX>(P), pk_map<BX>(P, E, 1), (const uint8_t*)P.mask, *ms[0], *ms[1], *ms[2], *ms[3],
         *msb, P.kcube, ly, in, epi, P.part, P.ticket, dot_dst, P.err);
}

template <class Epi, int BX, int NS, int MINB>
static void fine3_cube_launch(Prob& P, const float* u, const float* E, Epi epi0, double* dot_dst) {
  using ST = StagedOf<Epi>;
  using SE = typename ST::SE;
  const void* arr[4] = {nullptr, nullptr, nullptr, nullptr};
  SE epi = ST::make(epi0, arr);
  fine3_cube_go<SE, InU, BX, NS, MINB>(P, u, nullptr, nullptr, E, InU{}, epi, arr, dot_dst);
}

// Whether the fused cube launches (operator input computed from staged arrays) can run.
static bool cube_fusable(const Prob& P) {
  return P.fuse && P.dim == 3 && P.use_tma && P.tile_variant >= 9 && P.cube && P.ei.wht;
}

// A cube-kernel launch with an input transform, on the problem's tile variant; profiled like
// fine_apply with io_bytes algorithmic bytes per DOF besides E.
// Kind of a fused cube launch for the per-kind tile choice (Prob::kind_variant), -1 for others.
template <class SE, class IN> constexpr int cube_kind() {
  if constexpr (std::is_same<SE, SEResidIn>::value && std::is_same<IN, InWDB>::value) return 0;
  else if constexpr (std::is_same<SE, SEJacobiAdd0<true>>::value || std::is_same<SE, SEJacobiAdd0<false>>::value)
    return 1;
  else if constexpr (std::is_same<SE, SEStorePDot>::value) return 2;
  else return -1;
}

template <class SE, class IN>
static void fine3_cube_fused(Prob& P, const float* in0, const void* in1, const void* in1b, IN in, SE epi,
                             const void* const* arr, double* dot_dst, double io_bytes, const CubeExtra& xa = {}) {
  CatScope cat(P, CAT_FINE);
  const bool rec = P.prof && P.pev_used + 2 <= P.pev.size();
  if (rec) CK(cudaEventRecord(P.pev[P.pev_used], P.stream));
  constexpr int kind = cube_kind<SE, IN>();
  int variant = P.tile_variant;
  const int bps0 = P.blocks_per_sm;
  if constexpr (kind >= 0) {
    if (P.kind_variant[kind] >= 9) {
      variant = P.kind_variant[kind];
      P.blocks_per_sm = P.kind_bps[kind];
    }
  }
  struct Restore {
    Prob& P;
    int b;
    ~Restore() { P.blocks_per_sm = b; }
  } restore{P, bps0};
  switch (variant) {
    case 9: fine3_cube_go<SE, IN, 4, 3, 2>(P, in0, in1, in1b, P.E32, in, epi, arr, dot_dst, xa); break;
    case 10: fine3_cube_go<SE, IN, 4, 4, 2>(P, in0, in1, in1b, P.E32, in, epi, arr, dot_dst, xa); break;
    case 11: fine3_cube_go<SE, IN, 2, 3, 4>(P, in0, in1, in1b, P.E32, in, epi, arr, dot_dst, xa); break;
    case 12: fine3_cube_go<SE, IN, 8, 3, 1>(P, in0, in1, in1b, P.E32, in, epi, arr, dot_dst, xa); break;
    case 13: fine3_cube_go<SE, IN, 4, 3, 4>(P, in0, in1, in1b, P.E32, in, epi, arr, dot_dst, xa); break;
    case 15: fine3_cube_go<SE, IN, 4, 3, 3>(P, in0, in1, in1b, P.E32, in, epi, arr, dot_dst, xa); break;
    default: fine3_cube_go<SE, IN, 4, 4, 4>(P, in0, in1, in1b, P.E32, in, epi, arr, dot_dst, xa); break;
  }
  if (rec) {
    CK(cudaEventRecord(P.pev[P.pev_used + 1], P.stream));
    P.pev_used += 2;
    P.pbytes.push_back((double)P.n_dof * io_bytes + (double)P.n_el * sizeof(float));
  }
}

// Fine-level operator with epilogue.  u, E in type T.  When profiling is on, each launch is
// bracketed by CUDA events on the problem's stream and its algorithmic bytes recorded:
// input vector + E + the epilogue's per-DOF traffic (BC mask excluded).
template <typename T, class Epi>
static void fine_apply(Prob& P, const T* u, Epi epi, double* dot_dst) {
  CatScope cat(P, CAT_FINE);
  const Geo& g = P.g0;
  const T* E = TypeOps<T>::E(P);
  const bool rec = P.prof && P.pev_used + 2 <= P.pev.size();
  if (rec) CK(cudaEventRecord(P.pev[P.pev_used], P.stream));
  if (P.ei.wht) {
    bool packed = false;
    if constexpr (std::is_same<T, float>::value) {
      if constexpr (StagedOf<Epi>::ok) {
        if (P.dim == 3 && P.use_tma && P.tile_variant >= 9 && P.cube && staged_usable(epi)) {
          switch (P.tile_variant) {
            case 9: fine3_cube_launch<Epi, 4, 3, 2>(P, u, E, epi, dot_dst); break;
            case 10: fine3_cube_launch<Epi, 4, 4, 2>(P, u, E, epi, dot_dst); break;
            case 11: fine3_cube_launch<Epi, 2, 3, 4>(P, u, E, epi, dot_dst); break;
            case 12: fine3_cube_launch<Epi, 8, 3, 1>(P, u, E, epi, dot_dst); break;
            case 13: fine3_cube_launch<Epi, 4, 3, 4>(P, u, E, epi, dot_dst); break;
            case 15: fine3_cube_launch<Epi, 4, 3, 3>(P, u, E, epi, dot_dst); break;
            default: fine3_cube_launch<Epi, 4, 4, 4>(P, u, E, epi, dot_dst); break;
          }
          packed = true;
        }
      }
      if (packed) {
      } else if (P.dim == 3 && P.use_tma && P.tile_variant >= 5) {
        switch (P.tile_variant) {
          case 5: fine3_pk_launch<Epi, 4, 3, 1>(P, u, E, epi, dot_dst); break;
          case 6: fine3_pk_launch<Epi, 4, 3, 4>(P, u, E, epi, dot_dst); break;
          case 7: fine3_pk_launch<Epi, 2, 3, 8>(P, u, E, epi, dot_dst); break;
          default: fine3_pk_launch<Epi, 4, 4, 4>(P, u, E, epi, dot_dst); break;
        }
        packed = true;
      }
    }
    if (packed) {
    } else if (P.dim == 3 && P.use_tma) {
      switch (P.tile_variant) {
        case 0: fine3_tma_launch<T, Epi, 8, 4>(P, u, E, epi, dot_dst); break;
        case 1: fine3_tma_launch<T, Epi, 8, 3>(P, u, E, epi, dot_dst); break;
        case 2: fine3_tma_launch<T, Epi, 8, 2>(P, u, E, epi, dot_dst); break;
        case 3: fine3_tma_launch<T, Epi, 4, 4>(P, u, E, epi, dot_dst); break;
        default: fine3_tma_launch<T, Epi, 4, 3>(P, u, E, epi, dot_dst); break;
      }
    } else if (P.dim == 3) {
      int ly;
      dim3 grid = fine3_grid(g, ly);
      launch(P, k_fine3_wht<T, T, Epi, FINE_BX>, grid, dim3(32, FINE_BX), 0, g, u, E, (const uint8_t*)P.mask,
             cast3<T>(P.ei.k3), ly, epi, P.part, P.ticket, dot_dst);
    } else {
      int ly;
      dim3 grid = fine2_grid(g, ly);
      launch(P, k_fine2_wht<T, T, Epi, FINE2_NW>, grid, dim3(32 * FINE2_NW), 0, g, u, E, (const uint8_t*)P.mask,
             cast2<T>(P.ei.k2), ly, epi, P.part, P.ticket, dot_dst);
    }
  } else {
    if (P.dim == 3)
      launch(P, k_fine3_dense<T, T, Epi>, dim3(cdiv(g.nz, 128), g.nx, g.ny), dim3(128), 0, g, u, E,
             (const uint8_t*)P.mask, TypeOps<T>::K0b(P), epi, P.part, P.ticket, dot_dst);
    else
      launch(P, k_fine2_dense<T, T, Epi>, dim3(cdiv(g.nx, 128), g.ny), dim3(128), 0, g, u, E, (const uint8_t*)P.mask,
             TypeOps<T>::K0b(P), epi, P.part, P.ticket, dot_dst);
  }
  if (rec) {
    CK(cudaEventRecord(P.pev[P.pev_used + 1], P.stream));
    P.pev_used += 2;
    P.pbytes.push_back((double)P.n_dof * (sizeof(T) + Epi::kIoBytes) + (double)P.n_el * sizeof(T));
  }
}

// Same operator, forcing the dense path (cross-checks).
template <typename T, class Epi>
static void fine_apply_dense(Prob& P, const T* u, Epi epi, double* dot_dst) {
  const Geo& g = P.g0;
  const T* E = TypeOps<T>::E(P);
  if (P.dim == 3)
    launch(P, k_fine3_dense<T, T, Epi>, dim3(cdiv(g.nz, 128), g.nx, g.ny), 128, 0, 
        g, u, E, P.mask, TypeOps<T>::K0b(P), epi, P.part, P.ticket, dot_dst);
  else
    launch(P, k_fine2_dense<T, T, Epi>, dim3(cdiv(g.nx, 128), g.ny), 128, 0, 
        g, u, E, P.mask, TypeOps<T>::K0b(P), epi, P.part, P.ticket, dot_dst);
  KCHECK();
}

template <typename T, class Epi, typename TS = T>
static void st_apply(Prob& P, const Geo& g, const T* u, const TS* S, Epi epi, double* dot_dst) {
  CatScope cat(P, CAT_STENCIL);
  if (g.dim == 3 && g.n <= P.st_quad_max)
    launch(P, k_st3_apply_q<T, TS, Epi>, dim3(cdiv(g.n * 4, 128)), dim3(128), 0, g, u, S, epi, P.part, P.ticket,
           dot_dst);
  else if (g.dim == 3 && P.st_pair && std::is_same<T, float>::value && g.n >= P.st_pair_min)
    launch(P, k_st3_apply2<T, TS, Epi>, dim3(cdiv(g.n / 2, 128)), dim3(128), 0, g, u, S, epi, P.part, P.ticket,
           dot_dst);
  else if (g.dim == 3)
    launch(P, k_st3_apply<T, TS, Epi>, dim3(cdiv(g.n, 128)), dim3(128), 0, g, u, S, epi, P.part, P.ticket, dot_dst);
  else
    launch(P, k_st2_apply<T, TS, Epi>, dim3(cdiv(g.n, 128)), dim3(128), 0, g, u, S, epi, P.part, P.ticket, dot_dst);
}

template <typename T, class Epi>
static void level_apply(Prob& P, int l, const T* u, Epi epi, double* dot_dst = nullptr) {
  if (l == 0) {
    fine_apply<T>(P, u, epi, dot_dst);
    return;
  }
  if constexpr (std::is_same<T, float>::value) {
    if (P.st_bf16 && P.st_pair && P.lv[l].S16t && P.st_tile_min >= 0 && P.lv[l].g.n >= P.st_tile_min &&
        P.lv[l].g.n > P.st_quad_max) {
      CatScope cat(P, CAT_STENCIL);
      const Geo& g = P.lv[l].g;
      launch(P, k_st3_apply2t<Epi>, dim3(cdiv(g.n / 2, 128)), dim3(128), 0, g, u, (const unsigned*)P.lv[l].S16t, epi,
             P.part, P.ticket, dot_dst);
      return;
    }
    if (P.st_bf16 && P.lv[l].S16) {
      st_apply<T, Epi, __nv_bfloat16>(P, P.lv[l].g, u, (const __nv_bfloat16*)P.lv[l].S16, epi, dot_dst);
      return;
    }
  }
  st_apply<T>(P, P.lv[l].g, u, (const T*)P.lv[l].S, epi, dot_dst);
}

static unsigned ew_blocks(long long n) { return (unsigned)std::min<long long>(cdiv(n, 256), 148LL * 16); }

// out += sign * S x for the point springs (slot layout), and *dot += x^T S x when given.
template <typename TX, typename TO>
static void springs_apply(Prob& P, const TX* x, TO* out, double sign, double* dot) {
  if (P.n_springs == 0) return;
  launch(P, k_springs<TX, TO>, 1, 64, 0, P.n_springs, (const long long*)P.spr_flat, (const double*)P.spr_k,
         P.g0.n, (const uint8_t*)P.mask, x, out, sign, dot);
}

// ------------------------------------------------------------------ small kernels
template <typename TB, typename TD, typename TO>
__global__ void k_jacobi0(long long n, const TB* __restrict__ b, const TD* __restrict__ dinv, TO* __restrict__ x,
                          const double* omega, double wscale) {
  EDGE_PDL_ENTRY();
  const double w = (*omega) * wscale;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    using Tc = TO;
    const Tc wt = Conv<Tc>::from(w);
    x[i] = wt * Conv<Tc>::from(dinv[i]) * Conv<Tc>::from(b[i]);
  }
}
template <typename TA, typename TB, typename TO>
__global__ void k_add(long long n, const TA* __restrict__ a, const TB* __restrict__ b, TO* __restrict__ o) {
  EDGE_PDL_ENTRY();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    o[i] = Conv<TO>::from((double)Conv<double>::from(a[i]) + (double)Conv<double>::from(b[i]));
}
template <typename TI, typename TO>
__global__ void k_copy(long long n, const TI* __restrict__ a, TO* __restrict__ o) {
  EDGE_PDL_ENTRY();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    o[i] = Conv<TO>::from(a[i]);
}
// Start of a solve.  keep_omega = 0: the smoother weight starts at omega0 (the GPU solver
// resets it to min_omega every solve, solvers/_multigrid_cuda.py:210; the CPU solver starts
// its first solve at the constructor's omega); 1: it keeps the value the previous solve
// ended with (the CPU solver never resets it, solvers/_multigrid.py:178-225).
__global__ void k_pcg_init(PcgState* st, double tol, int maxiter, double min_omega, double d_omega, double omega0,
                           int keep_omega) {
  EDGE_PDL_ENTRY();
  st->tol = tol;
  st->maxiter = maxiter;
  st->min_omega = min_omega;
  st->d_omega = d_omega;
  if (!keep_omega) st->omega = omega0;
  st->iter = 0;
  st->done = 0;
  st->rz = st->rz_new = st->pq = st->rr = st->alpha = st->beta = 0.0;
  st->res = 0.0;
  st->last_replace = 1.0;
  st->n_true = 0;
  st->pend = 0;
  st->xa = 0.0;
}
__global__ void k_pcg_check_bb(PcgState* st, const int* chol_status) {
  EDGE_PDL_ENTRY();
  // ||f|| == 0: nothing to solve, report residual 0 like a converged solve
  if (st->bb == 0.0) {
    st->done = 1;
    st->res = 0.0;
  }
  // the coarsest factorisation failed (only reachable inside a graph, where the host
  // checks the status after the solve): stop before iterating on a broken preconditioner
  if (*chol_status) st->done = 3;
}

// ------------------------------------------------------------------ multigrid setup
template <typename T, typename TD0>
static void mg_setup(Prob& P) {
  CatScope cat(P, CAT_SETUP);
  const int L = P.n_level;
  const Geo& g0 = P.g0;
  const T* E = TypeOps<T>::E(P);
  // fine Jacobi diagonal
  launch(P, k_fine_dinv<T, TD0>, cdiv(g0.n, 256), 256, 0, g0, E, P.mask, P.dK0diag, (TD0*)P.lv[0].dinv, nullptr);
  KCHECK();
  if (L == 0) return;
  // level 1 from the fine operator
  {
    const Geo& gc = P.lv[1].g;
    const int nnb = P.dim == 3 ? 14 : 5;  // centre + upper directions
    dim3 grid(cdiv(gc.n, 128), nnb);
    if (P.dim == 3)
      launch(P, k_galerkin3_l0<T, T>, grid, 128, 0, g0, gc, E, P.mask, P.eflag, P.dQ, P.dK0b, (T*)P.lv[1].S);
    else
      launch(P, k_galerkin2_l0<T, T>, grid, 128, 0, g0, gc, E, P.mask, P.eflag, P.dQ, P.dK0b, (T*)P.lv[1].S);
    KCHECK();
  }
  for (int l = 1; l < L; ++l) {
    const Geo& gf = P.lv[l].g;
    const Geo& gc = P.lv[l + 1].g;
    const int nnb = P.dim == 3 ? 14 : 5;
    dim3 grid(cdiv(gc.n, 128), nnb);
    if (P.dim == 3 && P.gal_axis && P.gal_t1) {
      Geo g1, g2;
      gal_axis_geos(gf, gc, g1, g2);
      launch(P, k_galerkin3_axis<0, T, double>, dim3(cdiv(g1.n, 128), nnb), 128, 0, gf, g1, (const T*)P.lv[l].S,
             P.gal_t1);
      launch(P, k_galerkin3_axis<1, double, double>, dim3(cdiv(g2.n, 128), nnb), 128, 0, g1, g2,
             (const double*)P.gal_t1, P.gal_t2);
      launch(P, k_galerkin3_axis<2, double, T>, grid, 128, 0, g2, gc, (const double*)P.gal_t2, (T*)P.lv[l + 1].S);
    } else if (P.dim == 3)
      launch(P, k_galerkin3_st<T>, grid, 128, 0, gf, gc, (const T*)P.lv[l].S, (T*)P.lv[l + 1].S);
    else
      launch(P, k_galerkin2_st<T>, grid, 128, 0, gf, gc, (const T*)P.lv[l].S, (T*)P.lv[l + 1].S);
    KCHECK();
  }
  for (int l = 1; l < L; ++l) {
    const Geo& g = P.lv[l].g;
    launch(P, k_st_dinv<T, T>, cdiv(g.n, 256), 256, 0, g, (const T*)P.lv[l].S, (T*)P.lv[l].dinv);
    KCHECK();
    if (P.st_bf16 && P.lv[l].S16) {  // the Jacobi diagonal above keeps the FP32 centre
      const long long ns = (long long)nst(P.dim) * g.n;
      launch(P, k_copy<T, __nv_bfloat16>, ew_blocks(ns), 256, 0, ns, (const T*)P.lv[l].S,
             (__nv_bfloat16*)P.lv[l].S16);
      if constexpr (std::is_same<T, float>::value) {
        if (P.lv[l].S16t && P.st_tile_min >= 0 && g.n >= P.st_tile_min) {
          const long long nw = stt_words(g.n);
          launch(P, k_stencil_tiled_bf16, ew_blocks(nw), 256, 0, (long long)g.n, (const float*)P.lv[l].S,
                 (unsigned*)P.lv[l].S16t, nw);
        }
      }
    }
  }
  // coarsest: dense FP64 Cholesky and explicit inverse
  const Geo& gL = P.lv[L].g;
  const int nd = P.nd;
  CK(cudaMemsetAsync(P.Adense, 0, (size_t)nd * nd * sizeof(double), P.stream));
  launch(P, k_st_to_dense<T>, cdiv(gL.n, 256), 256, 0, gL, (const T*)P.lv[L].S, P.Adense, nd);
  KCHECK();
  CK(cudaMemsetAsync(P.chol_status, 0, sizeof(int), P.stream));
  const int nt = (nd + CB - 1) / CB;
  for (int K = 0; K < nt; ++K) {
    launch(P, k_chol_diag, 1, CB * CB / 4, 0, P.Adense, nd, K, P.chol_status);
    if (K + 1 < nt) {
      launch(P, k_chol_panel, nt - K - 1, CB * CB / 4, 0, P.Adense, nd, K);
      const int m = nt - K - 1;
      launch(P, k_chol_update, m * (m + 1) / 2, CB * CB / 4, 0, P.Adense, nd, K, nt);
    }
  }
  KCHECK();
  launch(P, k_transpose_lower, cdiv((long long)nd * nd, 256), 256, 0, P.Adense, P.Ut, nd);
  if (nd * sizeof(double) > 48 * 1024)
    CK(cudaFuncSetAttribute(k_chol_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(nd * sizeof(double))));
  launch(P, k_chol_inverse, nd, 256, nd * sizeof(double), P.Adense, P.Ut, P.Ainv, nd);
  KCHECK();
}

// ------------------------------------------------------------------ V-cycle
// Whether the mixed path runs the V-cycle from level l down as one persistent launch.
static bool tail_usable(const Prob& P, int l) {
  if (P.tail_l0 < 1 || l != P.tail_l0 || P.dim != 3 || P.prec == EDGE_FP64 || l >= P.n_level) return false;
  if (P.n_level - l + 1 > TAIL_MAX) return false;
  if (P.cycle_w)
    for (int w : P.w_levels)
      if (w >= l) return false;
  return true;
}

template <typename TS>
static void launch_tail(Prob& P, int l0) {
  TailParams<TS> T{};
  T.L0 = l0;
  T.L = P.n_level;
  for (int l = l0; l <= P.n_level; ++l) {
    Level& Lv = P.lv[l];
    TailLevel<TS>& V = T.lv[l - l0];
    V.g = Lv.g;
    V.S = (l < P.n_level) ? (const TS*)((std::is_same<TS, __nv_bfloat16>::value) ? Lv.S16 : Lv.S) : nullptr;
    V.dinv = (const float*)Lv.dinv;
    V.b = (float*)Lv.b;
    V.xa = (float*)Lv.xa;
    V.xb = (float*)Lv.xb;
    V.r = (float*)Lv.r;
    V.ea = (float*)Lv.ea;
    V.eb = (float*)Lv.eb;
    V.res = (float*)Lv.res;
    V.ws = std::pow(1.06, l);
    V.nsm = std::max(1, P.sweeps(l));
  }
  T.Ainv = P.Ainv;
  T.nd = P.nd;
  T.omega = &P.st->omega;
  T.bar = P.tail_bar;
  T.err = P.err;
  if (P.tail_blocks == 0) {
    int dev = 0, sms = 0, per = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_vcycle_tail<TS>, 256, 0));
    if (per < 1) fail(EDGE_ECUDA, "persistent V-cycle kernel cannot be resident");
    P.tail_blocks = sms * std::min(per, 2);
  }
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(P.tail_blocks);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = P.stream;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  const bool rec = P.bd && P.bev_used + 2 <= P.bev.size();
  if (rec) CK(cudaEventRecord(P.bev[P.bev_used], P.stream));
  CK(cudaLaunchKernelEx(&cfg, k_vcycle_tail<TS>, T));
  ++P.nlaunch;
  KCHECK();
  if (rec) {
    CK(cudaEventRecord(P.bev[P.bev_used + 1], P.stream));
    P.bev_used += 2;
    P.bcat.push_back(CAT_STENCIL);
  }
}

// Result in `out`; b and out have type T.  With dot_dst, the last fine sweep also
// computes dotv . out (FP64 accumulation).
// Whether the restriction from level l also runs level l+1's first sweep (mixed path, 3-D,
// level l+1 smoothed with the per-launch kernels).
static bool restrict_j0(const Prob& P, int l) {
  const int c = l + 1;
  return P.fuse && P.prec != EDGE_FP64 && P.dim == 3 && c < P.n_level && P.sweeps(c) >= 1 && !tail_usable(P, c);
}

// Restriction of level l's residual r into level l+1's right-hand side (with level l+1's
// first Jacobi sweep when restrict_j0).
template <typename T>
static void restrict_to(Prob& P, int l, const T* r) {
  Level& Lc = P.lv[l + 1];
  const Geo& g = P.lv[l].g;
  P.cur_cat = CAT_TRANSFER;
  if (P.dim == 3 && restrict_j0(P, l))
    launch(P, k_restrict3_j0<T>, dim3(cdiv((long long)Lc.g.nz * Lc.g.nx, 256), Lc.g.ny), 256, 0, g, Lc.g, r,
           (T*)Lc.b, (const T*)Lc.dinv, (T*)Lc.xa, (const double*)&P.st->omega, std::pow(1.06, l + 1));
  else if (P.dim == 3)
    launch(P, k_restrict3<T, T>, dim3(cdiv((long long)Lc.g.nz * Lc.g.nx, 256), Lc.g.ny), 256, 0, g, Lc.g, r,
           (T*)Lc.b);
  else
    launch(P, k_restrict2<T, T>, dim3(cdiv(Lc.g.nx, 64), Lc.g.ny), 64, 0, g, Lc.g, r, (T*)Lc.b);
  KCHECK();
  P.cur_cat = CAT_VECTOR;
}

// xr (level 0 of the fused x/r path): the first fine launch already ran (pcgmx_l1x) and b is
// the FP32 residual of the ping-pong pair (P.r32 / P.r32b by the iteration's parity).
template <typename T, typename TD0, typename TV>
static void vcycle(Prob& P, int l, const T* b, T* out, const TV* dotv, double* dot_dst, bool pre_done = false,
                   bool xr = false) {
  Level& Lv = P.lv[l];
  const Geo& g = Lv.g;
  const long long nv = (long long)g.dof * g.n;
  if (l == P.n_level) {
    CatScope cat(P, CAT_COARSE);
    launch(P, k_coarse_solve<T, T>, cdiv((long long)P.nd * 32, 256), 256, (size_t)P.nd * sizeof(T), g, P.Ainv, P.nd,
           b, out);
    KCHECK();
    return;
  }
  const double ws = std::pow(1.06, l);
  const double* om = &P.st->omega;
  T* x = (T*)Lv.xa;
  T* y = (T*)Lv.xb;
  T* r = (T*)Lv.r;
  const int nsm = P.sweeps(l);
  if constexpr (std::is_same<T, float>::value) {
    if (tail_usable(P, l) && (const void*)b == Lv.b && (const void*)out == Lv.res) {
      if (P.st_bf16 && P.lv[l].S16)
        launch_tail<__nv_bfloat16>(P, l);
      else
        launch_tail<float>(P, l);
      return;
    }
  }
  const int visits0 =
      (P.cycle_w && std::find(P.w_levels.begin(), P.w_levels.end(), l) != P.w_levels.end()) ? 2 : 1;
  if constexpr (std::is_same<T, float>::value && std::is_same<TD0, __nv_bfloat16>::value) {
    // one sweep on the fine level of the mixed path: the pre-smoothed iterate w Dinv b is
    // computed inside the two fine launches that need it instead of being stored
    if (l == 0 && nsm == 1 && visits0 == 1 && cube_fusable(P) && (!dot_dst || (const void*)dotv == (const void*)b)) {
      if (!xr) {  // r = b - A (w Dinv b)
        InWDB in{om, ws, 0.f};
        SEResidIn e{r, g.n};
        fine3_cube_fused(P, b, Lv.dinv, nullptr, in, e, nullptr, nullptr, 4 + 2 + 4);
      }
      Level& Lc = P.lv[1];
      restrict_to<T>(P, l, r);
      vcycle<T, TD0, T>(P, l + 1, (const T*)Lc.b, (T*)Lc.res, (const T*)nullptr, nullptr, restrict_j0(P, l));
      T* e1 = (T*)Lv.ea;
      P.cur_cat = CAT_TRANSFER;
      launch(P, k_prolong3<T, T>, dim3(cdiv((long long)Lc.g.nz * Lc.g.nx, 256), Lc.g.ny), 256, 0, g, Lc.g,
             (const T*)Lc.res, e1);
      KCHECK();
      P.cur_cat = CAT_VECTOR;
      const void* arr[3] = {r, Lv.dinv, b};  // out = w Dinv b + (e + w Dinv (r - A e)) [, b . out]
      CubeExtra xb;
      if (xr) xb.sb = P.r32b;
      const PcgState* pst = xr ? (const PcgState*)P.st : nullptr;
      if (dot_dst) {
        SEJacobiAdd0<true> e{out, om, ws, g.n, 0.f, pst};
        fine3_cube_fused(P, e1, nullptr, nullptr, InU{}, e, arr, dot_dst, 4 + 4 + 2 + 4 + 4, xb);
      } else {
        SEJacobiAdd0<false> e{out, om, ws, g.n, 0.f, pst};
        fine3_cube_fused(P, e1, nullptr, nullptr, InU{}, e, arr, nullptr, 4 + 4 + 2 + 4 + 4, xb);
      }
      KCHECK();
      return;
    }
  }
  auto sweep = [&](const T* bb, T* in, T* outv) {
    if (l == 0) {
      EpiJacobi<T, T, TD0> e{bb, (const TD0*)Lv.dinv, outv, om, ws, g.n};
      level_apply<T>(P, l, in, e);
    } else {
      EpiJacobi<T, T, T> e{bb, (const T*)Lv.dinv, outv, om, ws, g.n};
      level_apply<T>(P, l, in, e);
    }
  };
  // pre-smoothing from x = 0 (the first sweep already done by the restriction when pre_done)
  if (nsm >= 1) {
    if (pre_done) {
    } else if (l == 0)
      launch(P, k_jacobi0<T, TD0, T>, ew_blocks(nv), 256, 0, nv, b, (const TD0*)Lv.dinv, x, om, ws);
    else
      launch(P, k_jacobi0<T, T, T>, ew_blocks(nv), 256, 0, nv, b, (const T*)Lv.dinv, x, om, ws);
    KCHECK();
    for (int s = 1; s < nsm; ++s) {
      sweep(b, x, y);
      std::swap(x, y);
    }
  } else {
    CK(cudaMemsetAsync(x, 0, nv * sizeof(T), P.stream));
  }
  bool first = true;
  const int visits = (P.cycle_w && std::find(P.w_levels.begin(), P.w_levels.end(), l) != P.w_levels.end()) ? 2 : 1;
  for (int vis = 0; vis < visits; ++vis) {
    // residual on this level
    {
      EpiResid<T, T, T> e{b, r, g.n};
      level_apply<T>(P, l, first ? x : out, e);
    }
    const T* xcur = first ? x : out;
    Level& Lc = P.lv[l + 1];
    restrict_to<T>(P, l, r);
    vcycle<T, TD0, T>(P, l + 1, (const T*)Lc.b, (T*)Lc.res, (const T*)nullptr, nullptr, restrict_j0(P, l));
    T* e1 = (T*)Lv.ea;
    T* e2 = (T*)Lv.eb;
    P.cur_cat = CAT_TRANSFER;
    if (P.dim == 3)
      launch(P, k_prolong3<T, T>, dim3(cdiv((long long)Lc.g.nz * Lc.g.nx, 256), Lc.g.ny), 256, 0, g, Lc.g,
             (const T*)Lc.res, e1);
    else
      launch(P, k_prolong2<T, T>, dim3(cdiv(g.nx, 64), g.ny), 64, 0, g, Lc.g, (const T*)Lc.res, e1);
    KCHECK();
    P.cur_cat = CAT_VECTOR;
    const bool last_visit = (vis == visits - 1);
    if (nsm >= 1) {
      for (int s = 0; s < nsm - 1; ++s) {
        sweep(r, e1, e2);
        std::swap(e1, e2);
      }
      const bool dot = last_visit && dot_dst != nullptr;
      if (l == 0) {
        if (dot) {
          EpiJacobiAdd<T, T, TD0, T, true, TV> e{r, (const TD0*)Lv.dinv, xcur, out, dotv, om, ws, g.n};
          level_apply<T>(P, l, e1, e, dot_dst);
        } else {
          EpiJacobiAdd<T, T, TD0, T, false> e{r, (const TD0*)Lv.dinv, xcur, out, (const T*)nullptr, om, ws, g.n};
          level_apply<T>(P, l, e1, e);
        }
      } else {
        EpiJacobiAdd<T, T, T, T, false> e{r, (const T*)Lv.dinv, xcur, out, (const T*)nullptr, om, ws, g.n};
        level_apply<T>(P, l, e1, e);
      }
    } else {
      launch(P, k_add<T, T, T>, ew_blocks(nv), 256, 0, nv, xcur, e1, out);
      KCHECK();
      if (last_visit && dot_dst) {
        launch(P, k_dot<TV, T>, std::min<unsigned>(ew_blocks(nv), 1024), 256, 0, nv, dotv, out, P.part, P.ticket,
                                                                                   dot_dst);
        KCHECK();
      }
    }
    first = false;
  }
}

// ------------------------------------------------------------------ allocation of the hierarchy
static void mg_allocate(Prob& P) {
  const int L = P.n_level;
  P.gal_t1 = P.gal_t2 = nullptr;
  const size_t vb = vbytes(P.prec);
  P.lv.clear();
  P.lv.resize(L + 1);
  for (int l = 0; l <= L; ++l) {
    Level& Lv = P.lv[l];
    Lv.g = level_geo(P, l);
    const size_t nv = (size_t)Lv.g.dof * Lv.g.n;
    auto vec = [&]() -> void* { return vb == 8 ? (void*)P.alloc<double>(nv) : (void*)P.alloc<float>(nv); };
    if (l > 0) Lv.b = vec();
    Lv.res = vec();
    if (l < L) {
      Lv.xa = vec();
      Lv.xb = vec();
      Lv.r = vec();
      Lv.ea = vec();
      Lv.eb = vec();
      if (l == 0)
        Lv.dinv = (P.prec == EDGE_FP64) ? (void*)P.alloc<double>(nv) : (void*)P.alloc<__nv_bfloat16>(nv);
      else
        Lv.dinv = vec();
    }
    if (l > 0) {
      const size_t ns = (size_t)nst(P.dim) * Lv.g.n;
      Lv.S = vb == 8 ? (void*)P.alloc<double>(ns) : (void*)P.alloc<float>(ns);
      if (vb == 4 && l < L) Lv.S16 = (void*)P.alloc<__nv_bfloat16>(ns);
      if (vb == 4 && l < L && P.dim == 3 && P.st_tile_min >= 0 && Lv.g.n >= P.st_tile_min)
        Lv.S16t = (void*)P.alloc<unsigned>(stt_words(Lv.g.n));
    }
  }
  const Geo& gL = P.lv[L].g;
  P.nd = gL.nx * gL.ny * gL.nz * gL.dof;
  if (P.nd > 8192) fail(EDGE_EINVAL, "coarsest level has " + std::to_string(P.nd) + " DOFs; use more levels (<= 8192)");
  // k_coarse_solve stages b in shared memory: up to 64 KB for 8192 FP64 values (one constant
  // limit for every problem, so concurrent set-ups do not race on it)
  CK(cudaFuncSetAttribute(k_coarse_solve<float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          8192 * (int)sizeof(double)));
  CK(cudaFuncSetAttribute(k_coarse_solve<double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          8192 * (int)sizeof(double)));
  if (!P.tail_bar) {
    P.tail_bar = P.alloc<unsigned>(2);
    CK(cudaMemset(P.tail_bar, 0, 2 * sizeof(unsigned)));
  }
  P.Adense = P.alloc<double>((size_t)P.nd * P.nd);
  P.Ainv = P.alloc<double>((size_t)P.nd * P.nd);
  P.Ut = P.alloc<double>((size_t)P.nd * P.nd);
  if (P.dim == 3 && L >= 2) {  // the largest stencil product, level 1 -> 2
    Geo g1, g2;
    gal_axis_geos(P.lv[1].g, P.lv[2].g, g1, g2);
    P.gal_t1 = P.alloc<double>((size_t)NST3 * g1.n);
    P.gal_t2 = P.alloc<double>((size_t)NST3 * g2.n);
  }
}

// ------------------------------------------------------------------ PCG
// The solve is built from four pieces (prologue, iteration body, and for mixed precision the
// true-residual replacement) that run either from a host loop (one status read per
// iteration) or inside one CUDA graph (solve_graph below) whose while node repeats the body
// and whose if node runs the replacement, so the two drivers execute the same launches.
//
// PCG state at the start of a multigrid solve, with the smoother weight of the GPU solver
// (reset to min_omega) or, with omega_carry, of the CPU solver (omega at the first solve,
// then whatever the previous solve ended with).
static void pcg_init(Prob& P, double tol, int maxiter) {
  const int keep = (P.omega_carry && P.omega_started) ? 1 : 0;
  const double omega0 = P.omega_carry ? P.omega : P.min_omega;
  launch(P, k_pcg_init, 1, 1, 0, P.st, tol, maxiter, P.min_omega, P.omega - P.min_omega, omega0, keep);
}

// FP64: every level, vector and operator in FP64 (solvers/_multigrid_cuda.py:188-241).
static void pcg64_prologue(Prob& P, double tol, int maxiter) {
  CatScope cat(P, CAT_VECTOR);
  const Geo& g = P.g0;
  const long long nv = (long long)g.dof * g.n;
  pcg_init(P, tol, maxiter);
  {  // r = b - A x
    EpiResid<double, double, double> e{P.b64, P.r64, g.n};
    fine_apply<double>(P, (const double*)P.x64, e, nullptr);
    springs_apply(P, (const double*)P.x64, P.r64, -1.0, nullptr);
  }
  launch(P, k_dot<double, double>, std::min<unsigned>(ew_blocks(nv), 1024), 256, 0, nv, (const double*)P.b64,
         (const double*)P.b64, P.part, P.ticket, &P.st->bb);
  launch(P, k_pcg_check_bb, 1, 1, 0, P.st, (const int*)P.chol_status);
}
static void pcg64_body(Prob& P) {
  CatScope cat(P, CAT_VECTOR);
  const Geo& g = P.g0;
  const long long nv = (long long)g.dof * g.n;
  double* p = (double*)P.p;
  double* q = (double*)P.q;
  double* z = (double*)P.lv[0].res;
  vcycle<double, double, double>(P, 0, P.r64, z, P.r64, &P.st->rz_new);
  launch(P, k_pcg_p<double>, ew_blocks(nv), 256, 0, nv, p, (const double*)z, (const PcgState*)P.st);
  {
    EpiStoreDot<double> e{q, g.n};
    fine_apply<double>(P, (const double*)p, e, &P.st->pq);
    springs_apply(P, (const double*)p, q, 1.0, &P.st->pq);
  }
  launch(P, k_pcg_xr<double, double>, std::min<unsigned>(ew_blocks(nv), 1024), 256, 0, nv, P.x64, (const double*)p,
         P.r64, (const double*)q, P.st, P.part, P.ticket, (float*)nullptr);
}

// Plain CG (no preconditioner), the reference's CG solver (solvers/_gpu.py:11-58, cupyx cg
// with M = None): the FP64 PCG pieces with z = r.
static void cg_prologue(Prob& P, double tol, int maxiter) {
  CatScope cat(P, CAT_VECTOR);
  const Geo& g = P.g0;
  const long long nv = (long long)g.dof * g.n;
  const unsigned nb = std::min<unsigned>(ew_blocks(nv), 1024);
  launch(P, k_pcg_init, 1, 1, 0, P.st, tol, maxiter, 0.0, 0.0, 0.0, 0);
  {
    EpiResid<double, double, double> e{P.b64, P.r64, g.n};
    fine_apply<double>(P, (const double*)P.x64, e, nullptr);
    springs_apply(P, (const double*)P.x64, P.r64, -1.0, nullptr);
  }
  launch(P, k_dot<double, double>, nb, 256, 0, nv, (const double*)P.b64, (const double*)P.b64, P.part, P.ticket,
         &P.st->bb);
  launch(P, k_dot<double, double>, nb, 256, 0, nv, (const double*)P.r64, (const double*)P.r64, P.part, P.ticket,
         &P.st->rr);
  launch(P, k_pcg_check_bb, 1, 1, 0, P.st, (const int*)P.zero_int);
}
static void cg_body(Prob& P) {
  CatScope cat(P, CAT_VECTOR);
  const Geo& g = P.g0;
  const long long nv = (long long)g.dof * g.n;
  double* p = (double*)P.p;
  double* q = (double*)P.q;
  launch(P, k_cg_rz, 1, 1, 0, P.st);
  launch(P, k_pcg_p<double>, ew_blocks(nv), 256, 0, nv, p, (const double*)P.r64, (const PcgState*)P.st);
  {
    EpiStoreDot<double> e{q, g.n};
    fine_apply<double>(P, (const double*)p, e, &P.st->pq);
    springs_apply(P, (const double*)p, q, 1.0, &P.st->pq);
  }
  launch(P, k_pcg_xr<double, double>, std::min<unsigned>(ew_blocks(nv), 1024), 256, 0, nv, P.x64, (const double*)p,
         P.r64, (const double*)q, P.st, P.part, P.ticket, (float*)nullptr);
}
// True residual after the loop (the reference recomputes ||f - K x|| / ||f||); r64 is
// scratch at that point.
static void cg_epilogue(Prob& P) {
  CatScope cat(P, CAT_VECTOR);
  const Geo& g = P.g0;
  const long long nv = (long long)g.dof * g.n;
  EpiResid<double, double, double> e{P.b64, P.r64, g.n};
  fine_apply<double>(P, (const double*)P.x64, e, nullptr);
  springs_apply(P, (const double*)P.x64, P.r64, -1.0, nullptr);
  launch(P, k_dot<double, double>, std::min<unsigned>(ew_blocks(nv), 1024), 256, 0, nv, (const double*)P.r64,
         (const double*)P.r64, P.part, P.ticket, &P.st->rr);
  launch(P, k_final_res, 1, 1, 0, P.st);
}

// Mixed precision: FP32 operator, V-cycle and search directions; FP64 solution (kept as an
// FP32 increment between replacements), dot products, coarse solve, and true residuals
// r = b - A x (FP64 operator with FP64 E) that replace the residual recurrence every time it
// has dropped by REPLACE_DROP and before convergence is declared.  The recurrence itself is
// stored in FP32 (Prob::res32, default) or FP64.
static const double REPLACE_DROP = 1e-2;

static void pcgmx_true_residual(Prob& P) {
  const Geo& g = P.g0;
  const long long nv = (long long)g.dof * g.n;
  const unsigned nb = std::min<unsigned>(ew_blocks(nv), 1024);
  EpiResid<double, double, double> e{P.b64, P.r64, g.n};
  fine_apply<double>(P, (const double*)P.x64, e, nullptr);
  springs_apply(P, (const double*)P.x64, P.r64, -1.0, nullptr);
  launch(P, k_dot<double, double>, nb, 256, 0, nv, (const double*)P.r64, (const double*)P.r64, P.part, P.ticket,
         &P.st->rr);
  launch(P, k_copy<double, float>, ew_blocks(nv), 256, 0, nv, (const double*)P.r64, P.r32);
}
static void pcgmx_prologue(Prob& P, double tol, int maxiter) {
  CatScope cat(P, CAT_VECTOR);
  const Geo& g = P.g0;
  const long long nv = (long long)g.dof * g.n;
  const unsigned nb = std::min<unsigned>(ew_blocks(nv), 1024);
  pcg_init(P, tol, maxiter);
  CK(cudaMemsetAsync(P.x32, 0, nv * sizeof(float), P.stream));
  launch(P, k_dot<double, double>, nb, 256, 0, nv, (const double*)P.b64, (const double*)P.b64, P.part, P.ticket,
         &P.st->bb);
  pcgmx_true_residual(P);
  launch(P, k_pcg_check_bb, 1, 1, 0, P.st, (const int*)P.chol_status);
}
static void pcgmx_body(Prob& P) {
  CatScope cat(P, CAT_VECTOR);
  const Geo& g = P.g0;
  const long long nv = (long long)g.dof * g.n;
  const unsigned nb = std::min<unsigned>(ew_blocks(nv), 1024);
  float* p = (float*)P.p;
  float* q = (float*)P.q;
  float* z = (float*)P.lv[0].res;
  // r.z with the FP32 copy of the residual (the V-cycle's right-hand side), FP64 accumulation
  vcycle<float, __nv_bfloat16, float>(P, 0, P.r32, z, P.r32, &P.st->rz_new);
  if (P.res32 && P.n_springs == 0 && cube_fusable(P)) {
    // p = z + beta p_old inside the product (q = A p, p.q); p ping-pongs between the two
    // FP32 halves of the FP64-sized p buffer by iteration parity, and the x/r update reads
    // the half the product wrote
    float* p1 = p + nv;
    InPDir in{(const PcgState*)P.st, 0.f, 0, false};
    SEStorePDot e{q, p, p1, (const PcgState*)P.st, g.n, nullptr};
    fine3_cube_fused(P, (const float*)z, p, p1, in, e, nullptr, &P.st->pq, 4 + 4 + 4 + 4);
    launch(P, k_pcg_xr32, nb, 256, 0, nv, P.x32, (const float*)p, (const float*)p1, P.r32, (const float*)q, P.st,
           P.part, P.ticket);
    return;
  }
  launch(P, k_pcg_p<float>, ew_blocks(nv), 256, 0, nv, p, (const float*)z, (const PcgState*)P.st);
  {
    EpiStoreDot<float> e{q, g.n};
    fine_apply<float>(P, (const float*)p, e, &P.st->pq);
    springs_apply(P, (const float*)p, q, 1.0, &P.st->pq);
  }
  if (P.res32)  // x32 += alpha p, r32 -= alpha q in FP32
    launch(P, k_pcg_xr32, nb, 256, 0, nv, P.x32, (const float*)p, (const float*)nullptr, P.r32, (const float*)q,
           P.st, P.part, P.ticket);
  else
    launch(P, k_pcg_xr_lag, nb, 256, 0, nv, P.x32, (const float*)p, P.r64, (const float*)q, P.st, P.part, P.ticket,
           P.r32);
}
// ---- mixed path, x/r update fused (xr_usable).  One iteration:
//   head: the first fine launch applies the previous iteration's residual update
//         r = r_old - alpha q on the fly (InWDBQ), writes it into the other buffer of the
//         residual's ping-pong pair with r.r for the convergence test (SEResidInX), and starts
//         the V-cycle from it (u = w Dinv r, level-0 residual r - A u);
//   replace (when due): the pending solution update, fold into FP64, true residual, and the
//         head's V-cycle start again from the replaced residual;
//   rest (while not done): the V-cycle below the head, p = z + beta p_old with q = A p and the
//         previous iteration's solution update x32 += alpha p_old (SEStorePDotX).
// The smoother weight must not depend on the residual of the same iteration (it is fixed):
// the head's V-cycle start runs before that residual's norm is known.
static bool xr_usable(const Prob& P) {
  if (P.prec == EDGE_FP64 || !P.fuse || !P.fuse_xr || !P.res32 || P.n_springs || !cube_fusable(P)) return false;
  if (P.omega != P.min_omega || P.sweeps(0) != 1 || P.n_level < 1) return false;
  return !(P.cycle_w && std::find(P.w_levels.begin(), P.w_levels.end(), 0) != P.w_levels.end());
}
static void pcgmx_l1x(Prob& P, bool plain) {
  const Level& L0 = P.lv[0];
  const Geo& g = P.g0;
  InWDBQ in{(const PcgState*)P.st, &P.st->omega, 1.0, plain, 0.f, 0.f, false, 0};
  CubeExtra xa;
  xa.in0b = P.r32b;
  xa.in2 = L0.dinv;
  const float* q = (const float*)P.q;
  if (plain) {
    SEResidIn e{(float*)L0.r, g.n};
    fine3_cube_fused(P, P.r32, q, q, in, e, nullptr, nullptr, 4 + 4 + 2 + 4, xa);
  } else {
    SEResidInX e{(float*)L0.r, P.r32, P.r32b, P.st, g.n, 0.f, false, 0.0, nullptr};
    fine3_cube_fused(P, P.r32, q, q, in, e, nullptr, nullptr, 4 + 4 + 2 + 4 + 4, xa);
  }
}
static void pcgmx_pending_x(Prob& P) {
  const long long nv = (long long)P.g0.dof * P.g0.n;
  float* p = (float*)P.p;
  launch(P, k_x32_pend, ew_blocks(nv), 256, 0, nv, P.x32, (const float*)p, (const float*)(p + nv),
         (const PcgState*)P.st);
}
static void pcgmx_replace_xr(Prob& P) {
  CatScope cat(P, CAT_VECTOR);
  const Geo& g = P.g0;
  const long long nv = (long long)g.dof * g.n;
  const unsigned nb = std::min<unsigned>(ew_blocks(nv), 1024);
  pcgmx_pending_x(P);
  launch(P, k_fold_x, ew_blocks(nv), 256, 0, nv, P.x64, P.x32);
  EpiResid<double, double, double> e{P.b64, P.r64, g.n};
  fine_apply<double>(P, (const double*)P.x64, e, nullptr);
  launch(P, k_dot<double, double>, nb, 256, 0, nv, (const double*)P.r64, (const double*)P.r64, P.part, P.ticket,
         &P.st->rr);
  launch(P, k_r32_par, ew_blocks(nv), 256, 0, nv, (const double*)P.r64, P.r32, P.r32b, (const PcgState*)P.st);
  launch(P, k_pcg_true_res, 1, 1, 0, P.st);
  pcgmx_l1x(P, true);
}
static void pcgmx_rest_xr(Prob& P) {
  CatScope cat(P, CAT_VECTOR);
  const Geo& g = P.g0;
  const long long nv = (long long)g.dof * g.n;
  float* p = (float*)P.p;
  float* q = (float*)P.q;
  float* z = (float*)P.lv[0].res;
  vcycle<float, __nv_bfloat16, float>(P, 0, P.r32, z, P.r32, &P.st->rz_new, false, true);
  float* p1 = p + nv;
  InPDir in{(const PcgState*)P.st, 0.f, 0, false};
  SEStorePDotX e{q, p, p1, P.st, g.n, P.x32, nullptr, 0.f};
  const void* arr[1] = {P.x32};
  fine3_cube_fused(P, (const float*)z, p, p1, in, e, arr, nullptr, 4 + 4 + 4 + 4 + 8);
}

// x64 += x32 (the FP32 increment of the solution since the last replacement), x32 = 0
static void pcgmx_fold(Prob& P) {
  CatScope cat(P, CAT_VECTOR);
  const long long nv = (long long)P.g0.dof * P.g0.n;
  launch(P, k_fold_x, ew_blocks(nv), 256, 0, nv, P.x64, P.x32);
}
static void pcgmx_replace(Prob& P) {
  CatScope cat(P, CAT_VECTOR);
  pcgmx_fold(P);
  pcgmx_true_residual(P);
  launch(P, k_pcg_true_res, 1, 1, 0, P.st);
}

static void read_state(Prob& P) {
  CK(cudaMemcpyAsync(P.st_h, P.st, sizeof(PcgState), cudaMemcpyDeviceToHost, P.stream));
  CK(cudaStreamSynchronize(P.stream));
}

// Host-driven loop (used while profiling with per-launch events, or with graphs disabled).
static void pcg_host(Prob& P, double tol, int maxiter) {
  const bool mixed = P.prec != EDGE_FP64;
  if (mixed)
    pcgmx_prologue(P, tol, maxiter);
  else
    pcg64_prologue(P, tol, maxiter);
  read_state(P);
  P.last_true_res = mixed ? 1 : 0;
  if (mixed && xr_usable(P)) {  // the launches of the graph's fused x/r iteration
    while (!P.st_h->done) {
      pcgmx_l1x(P, false);
      read_state(P);
      if (replace_due_xr(P.st_h, REPLACE_DROP)) {
        pcgmx_replace_xr(P);
        read_state(P);
        ++P.last_true_res;
      }
      if (!P.st_h->done) pcgmx_rest_xr(P);
    }
    pcgmx_pending_x(P);
    pcgmx_fold(P);
    P.last_iters = P.st_h->iter;
    return;
  }
  while (!P.st_h->done) {
    if (mixed) {
      pcgmx_body(P);
      read_state(P);
      if (P.st_h->done == 1 || P.st_h->res < REPLACE_DROP * P.st_h->last_replace) {
        pcgmx_replace(P);
        read_state(P);
        ++P.last_true_res;
      }
    } else {
      pcg64_body(P);
      read_state(P);
    }
  }
  if (mixed) pcgmx_fold(P);  // stopped on maxiter after the last replacement
  P.last_iters = P.st_h->iter;
}

static void check_err(Prob& P) {
  int e = 0;
  CK(cudaMemcpyAsync(&e, P.err, sizeof(int), cudaMemcpyDeviceToHost, P.stream));
  CK(cudaStreamSynchronize(P.stream));
  if (e) {
    CK(cudaMemsetAsync(P.err, 0, sizeof(int), P.stream));
    fail(EDGE_ECUDA, "a bounded wait for a TMA stage expired; results of this call are invalid");
  }
}

static void ensure_mg(Prob& P) {
  if (P.n_level < 0) fail(EDGE_ESTATE, "multigrid not configured (edge_mg_config)");
}

static void mg_setup_prec(Prob& P) {
  if (P.prec == EDGE_FP64)
    mg_setup<double, double>(P);
  else
    mg_setup<float, __nv_bfloat16>(P);
}

// Capture parameters of the solve graph: anything baked into its launches.
static std::vector<double> graph_key(const Prob& P, double tol, int maxiter, bool cg = false) {
  std::vector<double> k = {cg ? -1.0 : (double)P.prec, tol, (double)maxiter, (double)P.n_level, (double)P.n_smooth, P.omega,
                           P.min_omega, (double)P.cycle_w, (double)P.tile_variant, (double)P.blocks_per_sm,
                           (double)P.st_quad_max, (double)P.n_springs, (double)P.use_tma, (double)P.has_cons,
                           (double)P.st_bf16, (double)P.st_pair, (double)P.st_pair_min, (double)P.st_tile_min,
                           (double)P.gal_axis, (double)P.res32,
                           (double)P.pdl, (double)P.fuse, (double)P.tail_l0, (double)P.omega_carry, (double)(P.omega_carry && P.omega_started),
                           (double)P.fuse_xr, (double)P.kind_variant[0], (double)P.kind_variant[1],
                           (double)P.kind_variant[2], (double)P.kind_bps[0], (double)P.kind_bps[1], (double)P.kind_bps[2]};
  for (int l : P.w_levels) k.push_back((double)l);
  k.push_back(-1.0);
  for (int v : P.level_sweeps) k.push_back((double)v);
  return k;
}

// Records one solve (hierarchy set-up, PCG prologue, and the iteration loop as a while node
// whose body holds, for mixed precision, the replacement as an if node) into P.sg_exec.
// Captured on the library's own streams so that the caller's stream may be the legacy
// default stream; touches only buffers the problem owns.
// Launch counts of one captured solve, for the launch tally of a graph execution: prologue
// and epilogue once, the loop body per iteration, the replacement per true residual.
struct SolveCounts {
  long long pro = 0, body = 0, rep = 0;
};

// Appends one solve (hierarchy set-up, PCG prologue, the iteration loop as a while node whose
// body holds, for mixed precision, the replacement as an if node, the epilogue) to the
// capture open on P.cap[0] (P.stream == P.cap[0]).  `depth` tracks the captures open (for
// the caller's clean-up on error).
static SolveCounts capture_solve_into(Prob& P, double tol, int maxiter, bool cg, int& depth) {
  const bool mixed = !cg && P.prec != EDGE_FP64;
  const long long n0 = P.nlaunch;
  long long n1 = 0, n2 = 0, n3 = 0, n4e = 0;
  if (cg)
    cg_prologue(P, tol, maxiter);
  else {
    mg_setup_prec(P);
    if (mixed)
      pcgmx_prologue(P, tol, maxiter);
    else
      pcg64_prologue(P, tol, maxiter);
  }
  cudaStreamCaptureStatus cs;
  cudaGraph_t g;
  const cudaGraphNode_t* deps;
  size_t nd;
  CK(cudaStreamGetCaptureInfo(P.cap[0], &cs, nullptr, &g, &deps, &nd));
  cudaGraphConditionalHandle hw;
  CK(cudaGraphConditionalHandleCreate(&hw, g, 0, cudaGraphCondAssignDefault));
  launch(P, k_cond_while, 1, 1, 0, hw, (const PcgState*)P.st);
  n1 = P.nlaunch;
  CK(cudaStreamGetCaptureInfo(P.cap[0], &cs, nullptr, &g, &deps, &nd));
  cudaGraphNodeParams wp = {};
  wp.type = cudaGraphNodeTypeConditional;
  wp.conditional.handle = hw;
  wp.conditional.type = cudaGraphCondTypeWhile;
  wp.conditional.size = 1;
  cudaGraphNode_t wnode;
  CK(cudaGraphAddNode(&wnode, g, deps, nd, &wp));
  CK(cudaStreamUpdateCaptureDependencies(P.cap[0], &wnode, 1, cudaStreamSetCaptureDependencies));
  cudaGraph_t body = wp.conditional.phGraph_out[0];
  P.stream = P.cap[1];
  CK(cudaStreamBeginCaptureToGraph(P.cap[1], body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  depth = 2;
  // an if node inside the body whose graph `rec` records (on P.cap[2]); h is set by `cond`
  auto if_node = [&](auto cond, auto rec) {
    cudaGraph_t gb;
    CK(cudaStreamGetCaptureInfo(P.cap[1], &cs, nullptr, &gb, &deps, &nd));
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, gb, 0, cudaGraphCondAssignDefault));
    cond(h);
    CK(cudaStreamGetCaptureInfo(P.cap[1], &cs, nullptr, &gb, &deps, &nd));
    cudaGraphNodeParams ip = {};
    ip.type = cudaGraphNodeTypeConditional;
    ip.conditional.handle = h;
    ip.conditional.type = cudaGraphCondTypeIf;
    ip.conditional.size = 1;
    cudaGraphNode_t inode;
    CK(cudaGraphAddNode(&inode, gb, deps, nd, &ip));
    CK(cudaStreamUpdateCaptureDependencies(P.cap[1], &inode, 1, cudaStreamSetCaptureDependencies));
    P.stream = P.cap[2];
    CK(cudaStreamBeginCaptureToGraph(P.cap[2], ip.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal));
    depth = 3;
    rec();
    CK(cudaStreamEndCapture(P.cap[2], nullptr));
    depth = 2;
    P.stream = P.cap[1];
  };
  const bool xr = mixed && xr_usable(P);
  if (xr) {
    pcgmx_l1x(P, false);
    n2 = P.nlaunch;
    if_node([&](cudaGraphConditionalHandle h) {
      launch(P, k_cond_replace_xr, 1, 1, 0, h, (const PcgState*)P.st, REPLACE_DROP);
    }, [&]() { pcgmx_replace_xr(P); });
    n3 = P.nlaunch;
    if_node([&](cudaGraphConditionalHandle h) { launch(P, k_cond_rest, 1, 1, 0, h, (const PcgState*)P.st); },
            [&]() { pcgmx_rest_xr(P); });
  } else if (mixed) {
    pcgmx_body(P);
    cudaGraph_t gb;
    CK(cudaStreamGetCaptureInfo(P.cap[1], &cs, nullptr, &gb, &deps, &nd));
    cudaGraphConditionalHandle hr;
    CK(cudaGraphConditionalHandleCreate(&hr, gb, 0, cudaGraphCondAssignDefault));
    launch(P, k_cond_replace, 1, 1, 0, hr, (const PcgState*)P.st, REPLACE_DROP);
    CK(cudaStreamGetCaptureInfo(P.cap[1], &cs, nullptr, &gb, &deps, &nd));
    cudaGraphNodeParams ip = {};
    ip.type = cudaGraphNodeTypeConditional;
    ip.conditional.handle = hr;
    ip.conditional.type = cudaGraphCondTypeIf;
    ip.conditional.size = 1;
    cudaGraphNode_t inode;
    CK(cudaGraphAddNode(&inode, gb, deps, nd, &ip));
    CK(cudaStreamUpdateCaptureDependencies(P.cap[1], &inode, 1, cudaStreamSetCaptureDependencies));
    n2 = P.nlaunch;
    P.stream = P.cap[2];
    CK(cudaStreamBeginCaptureToGraph(P.cap[2], ip.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal));
    depth = 3;
    pcgmx_replace(P);
    CK(cudaStreamEndCapture(P.cap[2], nullptr));
    depth = 2;
    n3 = P.nlaunch;
    P.stream = P.cap[1];
  } else if (cg) {
    cg_body(P);
  } else {
    pcg64_body(P);
  }
  launch(P, k_cond_while, 1, 1, 0, hw, (const PcgState*)P.st);
  CK(cudaStreamEndCapture(P.cap[1], nullptr));
  depth = 1;
  P.stream = P.cap[0];
  n4e = P.nlaunch;
  if (cg) cg_epilogue(P);
  if (xr) pcgmx_pending_x(P);
  if (mixed) pcgmx_fold(P);
  const long long n5 = P.nlaunch;
  SolveCounts c;
  c.pro = (n1 - n0) + (n5 - n4e);
  if (mixed) {
    c.rep = n3 - n2;
    c.body = (n2 - n1) + (n4e - n3);
  } else {
    c.body = n4e - n1;
  }
  return c;
}

// Runs `record` inside a capture of the library's own streams (the caller's stream may be the
// legacy default stream) into a new graph; on any error every capture still open is ended
// and the state restored before the error propagates.
template <class F>
static cudaGraph_t capture_graph(Prob& P, F record) {
  for (int i = 0; i < 3; ++i)
    if (!P.cap[i]) CK(cudaStreamCreateWithFlags(&P.cap[i], cudaStreamNonBlocking));
  cudaStream_t user = P.stream;
  const long long n0 = P.nlaunch;
  int depth = 0;
  cudaGraph_t graph = nullptr;
  try {
    P.stream = P.cap[0];
    P.capturing = true;
    CK(cudaStreamBeginCapture(P.cap[0], cudaStreamCaptureModeThreadLocal));
    depth = 1;
    record(depth);
    CK(cudaStreamEndCapture(P.cap[0], &graph));
    depth = 0;
    P.capturing = false;
  } catch (...) {
    P.capturing = false;
    for (int d = depth; d >= 1; --d) {
      cudaGraph_t junk = nullptr;
      cudaStreamEndCapture(P.cap[d - 1], &junk);
      if (d == 1 && junk) cudaGraphDestroy(junk);
    }
    cudaGetLastError();
    P.stream = user;
    P.nlaunch = n0;
    throw;
  }
  P.stream = user;
  P.nlaunch = n0;
  return graph;
}

static void capture_solve(Prob& P, double tol, int maxiter, bool cg = false) {
  if (P.sg_exec) {
    CK(cudaGraphExecDestroy(P.sg_exec));
    P.sg_exec = nullptr;
  }
  if (P.sg_graph) {
    CK(cudaGraphDestroy(P.sg_graph));
    P.sg_graph = nullptr;
  }
  SolveCounts c;
  P.sg_graph = capture_graph(P, [&](int& depth) { c = capture_solve_into(P, tol, maxiter, cg, depth); });
  CK(cudaGraphInstantiate(&P.sg_exec, P.sg_graph, 0));
  P.sg_pro = c.pro;
  P.sg_body = c.body;
  P.sg_if = c.rep;
  P.sg_key = graph_key(P, tol, maxiter, cg);
}

static void solve_graph(Prob& P, double tol, int maxiter, bool cg = false) {
  if (!P.sg_exec || P.sg_key != graph_key(P, tol, maxiter, cg)) capture_solve(P, tol, maxiter, cg);
  CK(cudaEventRecord(P.ev[0], P.stream));
  CK(cudaGraphLaunch(P.sg_exec, P.stream));
  CK(cudaEventRecord(P.ev[2], P.stream));
  int status = 0;
  if (!cg) CK(cudaMemcpyAsync(&status, P.chol_status, sizeof(int), cudaMemcpyDeviceToHost, P.stream));
  read_state(P);
  if (status) fail(EDGE_ENOTPD, "coarsest Galerkin matrix is not positive definite (missing boundary conditions?)");
  P.last_iters = P.st_h->iter;
  P.last_true_res = cg ? 1 : ((P.prec != EDGE_FP64) ? 1 + P.st_h->n_true : 0);
  P.nlaunch += P.sg_pro + P.sg_body * (long long)P.st_h->iter + P.sg_if * (long long)P.st_h->n_true;
}

static void solve_internal(Prob& P, double tol, int maxiter) {
  ensure_mg(P);
  if (!P.has_rho) fail(EDGE_ESTATE, "Solver requires a density vector to be passed or set on the kernel.");
  if (P.use_graph && !P.prof && !P.bd) {
    solve_graph(P, tol, maxiter);
    P.omega_started = true;
    check_err(P);
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, P.ev[0], P.ev[2]));
    P.last_setup_ms = 0.0;  // inside the graph: counted in the solve time
    P.last_solve_ms = ms;
    return;
  }
  CK(cudaEventRecord(P.ev[0], P.stream));
  mg_setup_prec(P);
  CK(cudaEventRecord(P.ev[1], P.stream));
  // check the coarse factorisation
  int status = 0;
  CK(cudaMemcpyAsync(&status, P.chol_status, sizeof(int), cudaMemcpyDeviceToHost, P.stream));
  CK(cudaStreamSynchronize(P.stream));
  if (status) fail(EDGE_ENOTPD, "coarsest Galerkin matrix is not positive definite (missing boundary conditions?)");
  pcg_host(P, tol, maxiter);
  P.omega_started = true;
  CK(cudaEventRecord(P.ev[2], P.stream));
  CK(cudaEventSynchronize(P.ev[2]));
  check_err(P);
  float a = 0, b = 0;
  CK(cudaEventElapsedTime(&a, P.ev[0], P.ev[1]));
  CK(cudaEventElapsedTime(&b, P.ev[1], P.ev[2]));
  P.last_setup_ms = a;
  P.last_solve_ms = b;
}


}  // namespace edge

using namespace edge;

struct edge_problem {
  Prob P;
};
struct edge_filter {
  Geo g;
  Taps taps;
  double* N = nullptr;
  long long n_el = 0;
  ~edge_filter() {
    if (N) cudaFree(N);
  }
};

// One SIMP iteration as one CUDA graph: the OC update of (it_rho, it_dr) into it_rho_new
// (prep, floor, bracket init, the bisection passes as a while node whose condition a kernel
// sets from the device-side state, the final design), then the analysis of it_rho_new:
// filter + SIMP law, the solve (hierarchy set-up and PCG loop as in capture_solve),
// compliance, sensitivities and the filter transpose into it_dr_new.  Every buffer is the
// problem's own; the caller copies the user's arrays in and out around the launch.
static const int OC_MAX_STEPS = 200;  // the host loop's bound (edge_oc_update)
static void capture_iteration(Prob& P, const edge_filter& F, double A, double vol, double vf, double move,
                              double penalty, double void_, double tol, int maxiter) {
  if (P.it_exec) {
    CK(cudaGraphExecDestroy(P.it_exec));
    P.it_exec = nullptr;
  }
  if (P.it_graph) {
    CK(cudaGraphDestroy(P.it_graph));
    P.it_graph = nullptr;
  }
  const Geo& g = P.g0;
  const long long n = P.n_el;
  const unsigned nb = std::min<unsigned>(ew_blocks(n), 1024);
  const unsigned nbp = std::min<unsigned>(nb, (unsigned)(P.part_cap / OC_NODES));
  const unsigned nbe = cdiv(P.n_el, 256);
  const long long nv = (long long)g.dof * g.n;
  long long n_fixed0 = 0, n_fixed1 = 0, n_fixed2 = 0, n_ocb = 0;
  SolveCounts sc;
  P.it_graph = capture_graph(P, [&](int& depth) {
    const long long a0 = P.nlaunch;
    {
      CatScope cat(P, CAT_OC);
      launch(P, k_oc_prep, nb, 256, 0, n, (const double*)P.it_rho, (const double*)P.it_dr, A, P.ocp, P.part,
             P.ticket, P.scal);
      launch(P, k_oc_floor, nb, 256, 0, n, P.ocp, (const double*)P.scal);
      launch(P, k_oc_state_init, 1, 1, 0, P.oc, vf, vol);
      cudaStreamCaptureStatus cs;
      cudaGraph_t gg;
      const cudaGraphNode_t* deps;
      size_t nd;
      CK(cudaStreamGetCaptureInfo(P.cap[0], &cs, nullptr, &gg, &deps, &nd));
      cudaGraphConditionalHandle ho;
      CK(cudaGraphConditionalHandleCreate(&ho, gg, 0, cudaGraphCondAssignDefault));
      launch(P, k_cond_oc, 1, 1, 0, ho, (const OcState*)P.oc, OC_MAX_STEPS);
      CK(cudaStreamGetCaptureInfo(P.cap[0], &cs, nullptr, &gg, &deps, &nd));
      cudaGraphNodeParams wp = {};
      wp.type = cudaGraphNodeTypeConditional;
      wp.conditional.handle = ho;
      wp.conditional.type = cudaGraphCondTypeWhile;
      wp.conditional.size = 1;
      cudaGraphNode_t wnode;
      CK(cudaGraphAddNode(&wnode, gg, deps, nd, &wp));
      CK(cudaStreamUpdateCaptureDependencies(P.cap[0], &wnode, 1, cudaStreamSetCaptureDependencies));
      P.stream = P.cap[1];
      CK(cudaStreamBeginCaptureToGraph(P.cap[1], wp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                       cudaStreamCaptureModeThreadLocal));
      depth = 2;
      const long long b0 = P.nlaunch;
      launch(P, k_oc_pass, nbp, 256, 0, n, (const double*)P.it_rho, (const double*)P.ocp, A, move, P.oc, P.part,
             P.ticket);
      launch(P, k_cond_oc, 1, 1, 0, ho, (const OcState*)P.oc, OC_MAX_STEPS);
      n_ocb = P.nlaunch - b0;
      CK(cudaStreamEndCapture(P.cap[1], nullptr));
      depth = 1;
      P.stream = P.cap[0];
      launch(P, k_oc_final, nb, 256, 0, n, (const double*)P.it_rho, (const double*)P.ocp, move, (const OcState*)P.oc,
             P.it_rho_new, P.part, P.ticket, P.scal + 1);
    }
    {
      CatScope cat(P, CAT_SENS);
      launch(P, k_filter_material<double, float>, nbe, 256, 0, g, F.taps, (const double*)P.it_rho_new, P.rho_f,
             P.E64, P.E32, penalty, void_, 0);
    }
    n_fixed0 = P.nlaunch - a0 - n_ocb;
    sc = capture_solve_into(P, tol, maxiter, false, depth);
    const long long c0 = P.nlaunch;
    {
      CatScope cat(P, CAT_SENS);
      launch(P, k_dot<double, double>, std::min<unsigned>(ew_blocks(nv), 1024), 256, 0, nv, (const double*)P.b64,
             (const double*)P.x64, P.part, P.ticket, P.scal + 2);
      launch(P, k_dk<double>, nbe, 256, 0, g, (const double*)P.x64, P.ei.k3, P.ei.k2, (const double*)P.dK0b,
             P.ei.wht ? 1 : 0, (double*)nullptr, (const double*)P.rho_f, P.gsens, penalty, void_);
      launch(P, k_filter_T, nbe, 256, 0, F.g, F.taps, (const double*)F.N, (const double*)P.gsens, P.it_dr_new);
    }
    n_fixed1 = P.nlaunch - c0;
  });
  CK(cudaGraphInstantiate(&P.it_exec, P.it_graph, 0));
  (void)n_fixed2;
  P.it_fixed = n_fixed0 + n_fixed1 + sc.pro;
  P.it_oc_body = n_ocb;
  P.it_body = sc.body;
  P.it_rep = sc.rep;
}




// ------------------------------------------------------------------ unstructured meshes
// One general mesh with its element matrices, the node adjacency, the density, the BC mask
// and the CG workspace (all allocated at creation).
struct edge_gen {
  GenGeo G{};
  long long n_dof = 0;
  double* rho = nullptr;
  uint8_t* cons = nullptr;
  double *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *b = nullptr;
  PcgState* st = nullptr;
  PcgState* st_h = nullptr;
  double* part = nullptr;
  unsigned* ticket = nullptr;
  int* zero = nullptr;  // a device zero (the CG's "coarse factorisation ok" status)
  cudaStream_t stream = nullptr;
  bool has_rho = false;
  int last_iters = 0;
  std::vector<void*> allocs;
  template <typename T> T* alloc(size_t n) {
    void* q = nullptr;
    CK(cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)));
    allocs.push_back(q);
    return (T*)q;
  }
  template <typename T> T* upload(const T* h, size_t n) {
    T* d = alloc<T>(n);
    CK(cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice));
    return d;
  }
  ~edge_gen() {
    for (void* q : allocs) cudaFree(q);
    if (st_h) cudaFreeHost(st_h);
  }
};

static unsigned gen_blocks(long long n) { return (unsigned)std::min<long long>(cdiv(n, 256), 148LL * 8); }

template <typename... KArgs, typename... Args>
static void glaunch(edge_gen& M, void (*kern)(KArgs...), unsigned grid, unsigned block, Args... args) {
  kern<<<grid, block, 0, M.stream>>>(static_cast<KArgs>(args)...);
  KCHECK();
}

static void gen_matvec(edge_gen& M, const double* u, double* out, double* dot) {
  glaunch(M, k_gen_matvec, std::min<unsigned>(gen_blocks(M.n_dof), 1024), 256, M.G, (const double*)M.rho,
          (const uint8_t*)M.cons, u, out, M.part, M.ticket, dot);
}

// ------------------------------------------------------------------ OC update without a workspace
// edge_oc_update_static runs the OC kernels of edge_oc_update on a fixed workspace that is a
// file-scope device array, so the call allocates nothing.  One workspace per device: calls
// whose work overlaps on one device (two streams, two host threads) race on it.
constexpr long long OC_STATIC_MAX_EL = 1LL << 20;   // elements; the ocP cache is 8 MiB
constexpr unsigned OC_STATIC_MAX_BLOCKS = 1024;     // reduction partials, as edge_oc_update
struct OcStaticScratch {
  OcState st;                                  // bisection state, rewritten by k_oc_static_init
  double scal[2];                              // sum(ocP_raw), sum((rho_new - rho)^2)
  unsigned ticket;                             // grid-reduction counter: zero when a kernel starts
  double part[OC_STATIC_MAX_BLOCKS * OC_NODES];
  double ocp[OC_STATIC_MAX_EL];
};
static __device__ __align__(256) OcStaticScratch g_oc_scratch;

// Device address of g_oc_scratch on the current device, looked up on every call: the lookup
// is a cheap runtime query that allocates nothing, and an address kept from an earlier call
// would be stale after a device reset (the module, and with it the array, is loaded again).
// `stream` must belong to the current device, since the address is that device's.
static OcStaticScratch* oc_static_scratch(cudaStream_t stream) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (stream != nullptr && stream != cudaStreamLegacy && stream != cudaStreamPerThread) {
    int sdev = -1;
    CK(cudaStreamGetDevice(stream, &sdev));
    if (sdev != dev)
      fail(EDGE_EINVAL, "stream belongs to device " + std::to_string(sdev) + ", the current device is " +
                            std::to_string(dev));
  }
  void* ptr = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&ptr, g_oc_scratch);
  if (e != cudaSuccess || !ptr)
    fail(EDGE_ECUDA, std::string("cudaGetSymbolAddress(OC workspace): ") + cudaGetErrorString(e));
  return static_cast<OcStaticScratch*>(ptr);
}

// Start state of one OC update: bracket [1e-9, 1e9] (TopOpt/_cuda.py:260-261), counter zero.
__global__ void k_oc_static_init(OcStaticScratch* s, double vf, double vol) {
  EDGE_PDL_ENTRY();
  OcState init{};
  init.l1 = 1e-9;
  init.l2 = 1e9;
  init.last = 0.5 * (init.l1 + init.l2);
  init.vf = vf;
  init.vol = vol;
  s->st = init;
  s->scal[0] = 0.0;
  s->scal[1] = 0.0;
  s->ticket = 0u;
}

#define API_BEGIN try {
#define API_END                 \
  }                             \
  catch (const EdgeError& e) {  \
    g_err = e.msg;              \
    return e.code;              \
  }                             \
  catch (const std::exception& e) { \
    g_err = e.what();           \
    return EDGE_ECUDA;          \
  }                             \
  return EDGE_OK;

// Average device time of `reps` Jacobi sweeps of the stencil operator on level l >= 1, in
// the problem's precision (the hierarchy must be built).
template <typename T>
static double time_level(Prob& P, int l, int reps) {
  Level& Lv = P.lv[l];
  const Geo& g = Lv.g;
  auto run = [&]() {
    EpiJacobi<T, T, T> e{(const T*)Lv.b, (const T*)Lv.dinv, (T*)Lv.xb, &P.st->omega, 1.0, g.n};
    level_apply<T>(P, l, (const T*)Lv.xa, e);  // the stencil copy the solve uses (BF16 where set)
  };
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  run();
  CK(cudaEventRecord(a, P.stream));
  for (int r = 0; r < reps; ++r) run();
  CK(cudaEventRecord(b, P.stream));
  CK(cudaEventSynchronize(b));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return ms / reps;
}

extern "C" {

const char* edge_last_error(void) { return g_err.c_str(); }
int edge_version(void) { return 1; }

int edge_problem_create(int dim, const int* nel, const double* K0, int precision, edge_problem** out) {
  API_BEGIN
  if (!out || !nel || !K0) fail(EDGE_EINVAL, "null argument");
  if (dim != 2 && dim != 3) fail(EDGE_EINVAL, "dim must be 2 or 3");
  if (precision != EDGE_FP64 && precision != EDGE_MIXED) fail(EDGE_EINVAL, "unknown precision");
  for (int d = 0; d < dim; ++d)
    if (nel[d] < 1) fail(EDGE_EINVAL, "element counts must be >= 1");
  auto* h = new edge_problem();
  Prob& P = h->P;
  try {
    P.dim = dim;
    P.prec = precision;
    for (int d = 0; d < dim; ++d) P.nel[d] = nel[d];
    P.g0 = make_geo(dim, nel[0], nel[1], dim == 3 ? nel[2] : 0, fine_zalign(dim, 0));
    P.n_el = (long long)nel[0] * nel[1] * (dim == 3 ? nel[2] : 1);
    P.n_dof = (long long)P.g0.nx * P.g0.ny * P.g0.nz * dim;
    analyse_element(dim, K0, P.ei);
    if (dim == 3) {
      P.k3p = pack3(P.ei.k3);
      P.cube = P.ei.wht && cube_form(P.ei.k3, P.kcube);
    }
    const int nk = P.ei.nk;
    P.dK0b = P.alloc<double>(nk * nk);
    CK(cudaMemcpy(P.dK0b, P.ei.K0b, nk * nk * sizeof(double), cudaMemcpyHostToDevice));
    P.dK0ref = P.alloc<double>(nk * nk);
    CK(cudaMemcpy(P.dK0ref, K0, nk * nk * sizeof(double), cudaMemcpyHostToDevice));
    std::vector<float> kf(nk * nk);
    for (int i = 0; i < nk * nk; ++i) kf[i] = (float)P.ei.K0b[i];
    P.dK0bf = P.alloc<float>(nk * nk);
    CK(cudaMemcpy(P.dK0bf, kf.data(), nk * nk * sizeof(float), cudaMemcpyHostToDevice));
    P.dK0diag = P.alloc<double>(nk);
    CK(cudaMemcpy(P.dK0diag, P.ei.kdiag, nk * sizeof(double), cudaMemcpyHostToDevice));
    P.dQ = P.alloc<double>(P.ei.Q.size());
    CK(cudaMemcpy(P.dQ, P.ei.Q.data(), P.ei.Q.size() * sizeof(double), cudaMemcpyHostToDevice));
    const Geo& g = P.g0;
    P.mask = P.alloc<uint8_t>(g.n);
    if (dim == 3) {
      P.mpz = (g.nz + 15) & ~15;
      P.eflag16 = P.alloc<uint8_t>((size_t)g.ny * g.nx * P.mpz);
    }
    P.eflag = P.alloc<uint8_t>(g.n);
    P.err = P.alloc<int>(1);
    P.E64 = P.alloc<double>(g.n);
    P.E32 = P.alloc<float>(g.n);
    const size_t nv = (size_t)g.dof * g.n;
    P.b64 = P.alloc<double>(nv);
    P.x64 = P.alloc<double>(nv);
    P.r64 = P.alloc<double>(nv);
    P.p = P.alloc<double>(nv);  // sized for FP64; the mixed path uses the first half as FP32
    P.q = P.alloc<double>(nv);
    P.r32 = P.alloc<float>(nv);
    P.r32b = P.alloc<float>(nv);
    P.x32 = P.alloc<float>(nv);
    P.rho_f = P.alloc<double>(P.n_el);
    P.gsens = P.alloc<double>(P.n_el);
    P.ocp = P.alloc<double>(P.n_el);
    P.part_cap = 1 << 20;
    P.part = P.alloc<double>(P.part_cap);
    P.ticket = P.alloc<unsigned>(1);
    P.st = P.alloc<PcgState>(1);
    P.oc = P.alloc<OcState>(1);
    P.scal = P.alloc<double>(16);
    P.zero_int = P.alloc<int>(1);
    P.chol_status = P.alloc<int>(1);
    CK(cudaMallocHost(&P.st_h, sizeof(PcgState)));
    CK(cudaMallocHost(&P.oc_h, sizeof(OcState)));
    CK(cudaMallocHost(&P.scal_h, 16 * sizeof(double)));
    for (int i = 0; i < 4; ++i) CK(cudaEventCreate(&P.ev[i]));
  } catch (...) {
    delete h;
    throw;
  }
  *out = h;
  API_END
}

int edge_problem_destroy(edge_problem* p) {
  API_BEGIN
  if (p) {
    cudaStreamSynchronize(p->P.stream);
    delete p;
  }
  API_END
}

int edge_set_stream(edge_problem* p, void* stream) {
  API_BEGIN
  if (!p) fail(EDGE_EINVAL, "null handle");
  p->P.stream = (cudaStream_t)stream;
  API_END
}

int edge_mg_set_sweeps(edge_problem* p, const int* sweeps, int n) {
  API_BEGIN
  if (!p || n < 0 || (n > 0 && !sweeps)) fail(EDGE_EINVAL, "bad argument");
  for (int i = 0; i < n; ++i)
    if (sweeps[i] < 0 || sweeps[i] > 16) fail(EDGE_EINVAL, "sweep counts must be in 0..16");
  p->P.level_sweeps.assign(sweeps, sweeps + n);
  API_END
}

int edge_mg_set_omega_carry(edge_problem* p, int enable) {
  API_BEGIN
  if (!p) fail(EDGE_EINVAL, "null handle");
  p->P.omega_carry = enable != 0;
  p->P.omega_started = false;
  API_END
}

int edge_launch_count(const edge_problem* p, long long* n) {
  API_BEGIN
  if (!p || !n) fail(EDGE_EINVAL, "null argument");
  *n = p->P.nlaunch;
  API_END
}

int edge_set_graph(edge_problem* p, int enable) {
  API_BEGIN
  if (!p) fail(EDGE_EINVAL, "null handle");
  p->P.use_graph = enable != 0;
  API_END
}

int edge_set_stencil_pair(edge_problem* p, long long min_slots) {
  API_BEGIN
  if (!p) fail(EDGE_EINVAL, "null handle");
  p->P.st_pair = min_slots >= 0;
  p->P.st_pair_min = min_slots;
  API_END
}

int edge_set_stencil_tiled(edge_problem* p, long long min_slots) {
  API_BEGIN
  if (!p) fail(EDGE_EINVAL, "null handle");
  Prob& P = p->P;
  P.st_tile_min = min_slots < 0 ? -1 : min_slots;
  // levels allocated before this call get their tile-major copy now; every solve runs the
  // hierarchy set-up, which fills it
  if (P.st_tile_min >= 0 && P.dim == 3 && P.prec != EDGE_FP64)
    for (int l = 1; l < (int)P.lv.size() - 1; ++l) {
      Level& Lv = P.lv[l];
      if (Lv.S16 && !Lv.S16t && Lv.g.n >= P.st_tile_min) Lv.S16t = (void*)P.alloc<unsigned>(stt_words(Lv.g.n));
    }
  API_END
}

int edge_set_galerkin_axis(edge_problem* p, int enable) {
  API_BEGIN
  if (!p) fail(EDGE_EINVAL, "null handle");
  p->P.gal_axis = enable != 0;
  API_END
}

int edge_set_coarse_bf16(edge_problem* p, int enable) {
  API_BEGIN
  if (!p) fail(EDGE_EINVAL, "null handle");
  p->P.st_bf16 = enable != 0;
  API_END
}

int edge_set_pdl(edge_problem* p, int enable) {
  API_BEGIN
  if (!p) fail(EDGE_EINVAL, "null handle");
  p->P.pdl = enable != 0;
  API_END
}

int edge_set_tail(edge_problem* p, int level) {
  API_BEGIN
  if (!p) fail(EDGE_EINVAL, "null handle");
  if (level < 0) fail(EDGE_EINVAL, "level must be >= 0");
  p->P.tail_l0 = level;
  API_END
}

int edge_set_fuse(edge_problem* p, int enable) {
  API_BEGIN
  if (!p) fail(EDGE_EINVAL, "null handle");
  p->P.fuse = enable != 0;
  API_END
}

int edge_set_fuse_xr(edge_problem* p, int enable) {
  API_BEGIN
  if (!p) fail(EDGE_EINVAL, "null handle");
  p->P.fuse_xr = enable != 0;
  API_END
}

int edge_set_residual32(edge_problem* p, int enable) {
  API_BEGIN
  if (!p) fail(EDGE_EINVAL, "null handle");
  p->P.res32 = enable != 0;
  API_END
}

int edge_set_stencil_quad(edge_problem* p, long long max_slots) {
  API_BEGIN
  if (!p || max_slots < 0) fail(EDGE_EINVAL, "bad argument");
  p->P.st_quad_max = max_slots;
  API_END
}

int edge_uses_transform(const edge_problem* p) { return p && p->P.ei.wht ? 1 : 0; }
int edge_uses_cube_form(const edge_problem* p) { return p && p->P.cube ? 1 : 0; }

int edge_set_fine_tile(edge_problem* p, int variant, int blocks_per_sm) {
  API_BEGIN
  if (!p || variant < 0 || variant > 15 || blocks_per_sm < 1 || blocks_per_sm > 64) fail(EDGE_EINVAL, "bad tile");
  p->P.tile_variant = variant;
  p->P.blocks_per_sm = blocks_per_sm;
  for (int k = 0; k < 3; ++k) {  // one tile for every launch
    p->P.kind_variant[k] = -1;
    p->P.kind_bps[k] = 0;
  }
  API_END
}

// Average device time of `reps` fine-operator launches with the current tile, the smoother
// sweep epilogue (sweep = true; needs the multigrid allocated) or the plain product; buffer
// contents do not matter for timing.
static double time_fine(Prob& P, int precision, bool sweep, int reps, bool mix = false, int only_kind = -1) {
  const Geo& g = P.g0;
  auto run = [&]() {
    if (mix && cube_fusable(P)) {
      // the same three launches fused as the solver runs them on this tile: first sweep +
      // residual, last sweep + correction + r.z, search direction + product + p.q (or the
      // one of kind only_kind)
      Level& L0 = P.lv[0];
      if (only_kind < 0 || only_kind == 0) {
        InWDB i1{&P.st->omega, 1.0, 0.f};
        SEResidIn e1{(float*)L0.r, g.n};
        fine3_cube_fused(P, P.r32, L0.dinv, nullptr, i1, e1, nullptr, nullptr, 4 + 2 + 4);
      }
      if (only_kind < 0 || only_kind == 1) {
        const void* arr[3] = {L0.r, L0.dinv, P.r32};
        SEJacobiAdd0<true> e2{(float*)L0.res, &P.st->omega, 1.0, g.n, 0.f};
        fine3_cube_fused(P, (const float*)L0.ea, nullptr, nullptr, InU{}, e2, arr, &P.st->rz, 4 + 4 + 2 + 4 + 4);
      }
      if (only_kind < 0 || only_kind == 2) {
        const long long nv = (long long)g.dof * g.n;
        float* p0 = (float*)P.p;
        InPDir i3{(const PcgState*)P.st, 0.f, 0, false};
        SEStorePDot e3{(float*)P.q, p0, p0 + nv, (const PcgState*)P.st, g.n, nullptr};
        fine3_cube_fused(P, (const float*)L0.res, p0, p0 + nv, i3, e3, nullptr, &P.st->pq, 4 + 4 + 4 + 4);
      }
      return;
    }
    if (mix) {
      // the fine-level launches of one mixed-precision PCG iteration with one sweep per level:
      // residual, last sweep + correction + r.z, product + p.q
      Level& L0 = P.lv[0];
      const __nv_bfloat16* d = (const __nv_bfloat16*)L0.dinv;
      EpiResid<float, float, float> e1{P.r32, (float*)L0.r, g.n};
      fine_apply<float>(P, (const float*)L0.xa, e1, nullptr);
      EpiJacobiAdd<float, float, __nv_bfloat16, float, true, float> e2{
          P.r32, d, (const float*)L0.xa, (float*)L0.res, P.r32, &P.st->omega, 1.0, g.n};
      fine_apply<float>(P, (const float*)L0.ea, e2, &P.st->rz);
      EpiStoreDot<float> e3{(float*)P.q, g.n};
      fine_apply<float>(P, (const float*)P.p, e3, &P.st->pq);
      return;
    }
    if (precision == EDGE_FP64) {
      if (sweep) {
        EpiJacobi<double, double, double> e{P.b64, (const double*)P.lv[0].dinv, P.r64, &P.st->omega, 1.0, g.n};
        fine_apply<double>(P, P.x64, e, nullptr);
      } else {
        EpiStore<double, double> e{P.r64, g.n};
        fine_apply<double>(P, P.x64, e, nullptr);
      }
    } else {
      if (sweep) {
        EpiJacobi<float, float, __nv_bfloat16> e{P.r32, (const __nv_bfloat16*)P.lv[0].dinv, (float*)P.q,
                                                 &P.st->omega, 1.0, g.n};
        fine_apply<float>(P, (const float*)P.p, e, nullptr);
      } else {
        EpiStore<float, float> e{(float*)P.q, g.n};
        fine_apply<float>(P, (const float*)P.p, e, nullptr);
      }
    }
  };
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  run();
  CK(cudaEventRecord(a, P.stream));
  for (int r = 0; r < reps; ++r) run();
  CK(cudaEventRecord(b, P.stream));
  CK(cudaEventSynchronize(b));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return ms / reps;
}

static bool can_time_sweep(const Prob& P, int precision) {
  if (P.n_level < 0 || P.lv.empty() || !P.lv[0].dinv) return false;
  return precision == EDGE_FP64 ? P.prec == EDGE_FP64 : P.prec == EDGE_MIXED;
}

// Autotuner: times every (tile variant, y-chunking) of the fine operator on the current E and
// keeps the fastest: once the multigrid is configured, the mixed path's per-iteration mix
// of fine launches (residual, last sweep with r.z, product with p.q) or the FP64 smoother
// sweep; else the plain product.  Needs E set.
int edge_autotune_fine(edge_problem* p, int precision, int reps, double* best_ms, int* best_variant,
                       int* best_bps) {
  API_BEGIN
  if (!p) fail(EDGE_EINVAL, "null handle");
  Prob& P = p->P;
  if (!P.has_rho) fail(EDGE_ESTATE, "rho not set");
  if (P.dim != 3 || !P.ei.wht || !P.use_tma) {
    if (best_ms) *best_ms = 0;
    if (best_variant) *best_variant = P.tile_variant;
    if (best_bps) *best_bps = P.blocks_per_sm;
    return EDGE_OK;
  }
  double best = 1e30;
  int bv = P.tile_variant, bb = P.blocks_per_sm;
  // y-chunking targets: the grid's wave count against the resident blocks depends on them
  const int bps_list[8] = {2, 3, 4, 6, 8, 10, 12, 16};
  // variants 5..8: packed-pair FP32 kernel; 9..12: its cube-element form
  const int nvar = precision == EDGE_FP64 ? 5 : (P.cube ? 16 : 9);
  const bool sweep = can_time_sweep(P, precision);
  const bool mix = sweep && precision != EDGE_FP64;  // time the whole per-iteration mix
  for (int v = 0; v < nvar; ++v)
    for (int bi = 0; bi < 8; ++bi) {
      P.tile_variant = v;
      P.blocks_per_sm = bps_list[bi];
      const double ms = time_fine(P, precision, sweep, reps, mix);
      if (ms < best) {
        best = ms;
        bv = v;
        bb = bps_list[bi];
      }
    }
  check_err(P);
  P.tile_variant = bv;
  P.blocks_per_sm = bb;
  for (int k = 0; k < 3; ++k) {
    P.kind_variant[k] = -1;
    P.kind_bps[k] = 0;
  }
  if (mix && P.kind_tune && cube_fusable(P)) {
    // each fused launch kind alone: the variants of the cube kernel (their register caps and
    // stage counts suit the three epilogues differently) at the mix's y-chunking and one
    // either side of it; a kind keeps the mix's tile unless another is 2 % faster
    const int cube_v[6] = {9, 10, 11, 12, 13, 15};
    for (int k = 0; k < 3; ++k) {
      P.kind_variant[k] = bv;
      P.kind_bps[k] = bb;
      const double base = time_fine(P, precision, sweep, reps, true, k);
      double kb = base;
      int kv = bv, kbps = bb;
      for (int v : cube_v)
        for (int b : {bb / 2, bb, bb * 2}) {
          if (b < 1 || b > 64 || (v == bv && b == bb)) continue;
          P.kind_variant[k] = v;
          P.kind_bps[k] = b;
          const double ms = time_fine(P, precision, sweep, reps, true, k);
          if (ms < kb) {
            kb = ms;
            kv = v;
            kbps = b;
          }
        }
      const bool keep = kb < 0.98 * base;
      P.kind_variant[k] = keep ? kv : -1;
      P.kind_bps[k] = keep ? kbps : 0;
    }
    check_err(P);
  }
  if (best_ms) *best_ms = best;
  if (best_variant) *best_variant = bv;
  if (best_bps) *best_bps = bb;
  API_END
}

int edge_fine_kind_tiles(const edge_problem* p, int* variants, int* blocks_per_sm) {
  API_BEGIN
  if (!p || !variants || !blocks_per_sm) fail(EDGE_EINVAL, "null argument");
  for (int k = 0; k < 3; ++k) {
    variants[k] = p->P.kind_variant[k];
    blocks_per_sm[k] = p->P.kind_bps[k];
  }
  API_END
}

int edge_set_kind_tune(edge_problem* p, int enable) {
  API_BEGIN
  if (!p) fail(EDGE_EINVAL, "null handle");
  p->P.kind_tune = enable != 0;
  if (!enable)
    for (int k = 0; k < 3; ++k) {
      p->P.kind_variant[k] = -1;
      p->P.kind_bps[k] = 0;
    }
  API_END
}

int edge_time_level(edge_problem* p, int level, int reps, double* ms) {
  API_BEGIN
  if (!p || !ms || reps < 1) fail(EDGE_EINVAL, "bad argument");
  Prob& P = p->P;
  if (P.lv.empty() || level < 1 || level >= P.n_level) fail(EDGE_EINVAL, "level must be a smoothed coarse level");
  *ms = P.prec == EDGE_FP64 ? time_level<double>(P, level, reps) : time_level<float>(P, level, reps);
  API_END
}

int edge_time_fine(edge_problem* p, int precision, int variant, int blocks_per_sm, int sweep, int reps,
                   double* ms) {
  API_BEGIN
  if (!p || !ms || reps < 1 || variant < 0 || variant > 15 || blocks_per_sm < 1 || blocks_per_sm > 64)
    fail(EDGE_EINVAL, "bad argument");
  Prob& P = p->P;
  if (!P.has_rho) fail(EDGE_ESTATE, "rho not set");
  if (sweep && !can_time_sweep(P, precision)) fail(EDGE_ESTATE, "the sweep needs the multigrid of this precision");
  const int v0 = P.tile_variant, b0 = P.blocks_per_sm;
  P.tile_variant = variant;
  P.blocks_per_sm = blocks_per_sm;
  *ms = time_fine(P, precision, sweep != 0, reps);
  P.tile_variant = v0;
  P.blocks_per_sm = b0;
  check_err(P);
  API_END
}

int edge_set_tma(edge_problem* p, int enable) {
  API_BEGIN
  if (!p) fail(EDGE_EINVAL, "null handle");
  p->P.use_tma = enable != 0;
  API_END
}


int edge_set_constraints(edge_problem* p, const uint8_t* cons_dev) {
  API_BEGIN
  if (!p || !cons_dev) fail(EDGE_EINVAL, "null argument");
  Prob& P = p->P;
  launch(P, k_mask_from_user, cdiv(P.g0.n, 256), 256, 0, P.g0, cons_dev, P.mask);
  if (P.eflag16)
    launch(P, k_flag_pitch16, cdiv(P.g0.n, 256), 256, 0, P.g0, (const uint8_t*)P.mask, P.eflag16, P.mpz);
  launch(P, k_elem_flags, cdiv(P.g0.n, 256), 256, 0, P.g0, P.mask, P.eflag);
  KCHECK();
  P.has_cons = true;
  API_END
}

int edge_set_rho(edge_problem* p, const double* E_dev) {
  API_BEGIN
  if (!p || !E_dev) fail(EDGE_EINVAL, "null argument");
  Prob& P = p->P;
  launch(P, k_elem_user_to_slots<double>, cdiv(P.g0.n, 256), 256, 0, P.g0, E_dev, P.E64);
  if (P.E32) launch(P, k_elem_user_to_slots<float>, cdiv(P.g0.n, 256), 256, 0, P.g0, E_dev, P.E32);
  KCHECK();
  P.has_rho = true;
  API_END
}

// The real grid of nel_real elements per axis inside the problem's (padded) grid.
static Geo real_geo(const Prob& P, const int* nel_real) {
  for (int d = 0; d < P.dim; ++d)
    if (nel_real[d] < 1 || nel_real[d] > P.nel[d]) fail(EDGE_EINVAL, "real extents outside the problem's grid");
  Geo gr = P.g0;
  gr.nx = nel_real[0] + 1;
  gr.ny = nel_real[1] + 1;
  if (P.dim == 3) gr.nz = nel_real[2] + 1;
  return gr;
}

int edge_set_rho_embedded(edge_problem* p, const double* E_dev, const int* nel_real) {
  API_BEGIN
  if (!p || !E_dev || !nel_real) fail(EDGE_EINVAL, "null argument");
  Prob& P = p->P;
  const Geo gr = real_geo(P, nel_real);
  launch(P, k_elem_user_to_slots_emb<double>, cdiv(P.g0.n, 256), 256, 0, P.g0, gr, E_dev, P.E64);
  if (P.E32) launch(P, k_elem_user_to_slots_emb<float>, cdiv(P.g0.n, 256), 256, 0, P.g0, gr, E_dev, P.E32);
  KCHECK();
  P.has_rho = true;
  API_END
}

int edge_mg_solve_embedded(edge_problem* p, const int* nel_real, const double* f_dev, double* x_dev, int use_last,
                           double tol, int maxiter, double* residual_out, int* iters_out) {
  API_BEGIN
  if (!p || !nel_real || !f_dev || !x_dev) fail(EDGE_EINVAL, "null argument");
  Prob& P = p->P;
  const Geo& g = P.g0;
  const Geo gr = real_geo(P, nel_real);
  launch(P, k_user_to_slots_emb<double>, cdiv(g.n, 256), 256, 0, g, gr, f_dev, P.b64);
  if (use_last)
    launch(P, k_user_to_slots_emb<double>, cdiv(g.n, 256), 256, 0, g, gr, (const double*)x_dev, P.x64);
  else
    CK(cudaMemsetAsync(P.x64, 0, (size_t)g.dof * g.n * sizeof(double), P.stream));
  KCHECK();
  solve_internal(P, tol, maxiter);
  launch(P, k_slots_to_user_emb<double>, cdiv(g.n, 256), 256, 0, g, gr, P.x64, x_dev);
  KCHECK();
  CK(cudaStreamSynchronize(P.stream));
  if (residual_out) *residual_out = P.st_h->res;
  if (iters_out) *iters_out = P.st_h->iter;
  API_END
}

int edge_matvec(edge_problem* p, const double* u_dev, double* out_dev) {
  API_BEGIN
  if (!p || !u_dev || !out_dev) fail(EDGE_EINVAL, "null argument");
  Prob& P = p->P;
  if (!P.has_rho) fail(EDGE_ESTATE, "Rho has not been set. dot works only after setting rho.");
  const Geo& g = P.g0;
  launch(P, k_user_to_slots<double>, cdiv(g.n, 256), 256, 0, g, u_dev, P.b64);
  EpiStore<double, double> e{P.r64, g.n};
  fine_apply<double>(P, P.b64, e, nullptr);
  springs_apply(P, (const double*)P.b64, P.r64, 1.0, nullptr);
  launch(P, k_slots_to_user<double>, cdiv(g.n, 256), 256, 0, g, P.r64, out_dev);
  KCHECK();
  API_END
}

// The product through the FP32 operator of the mixed-precision solver (FP32 E and u).
int edge_matvec_f32(edge_problem* p, const double* u_dev, double* out_dev) {
  API_BEGIN
  if (!p || !u_dev || !out_dev) fail(EDGE_EINVAL, "null argument");
  Prob& P = p->P;
  if (!P.has_rho) fail(EDGE_ESTATE, "Rho has not been set. dot works only after setting rho.");
  const Geo& g = P.g0;
  float* u32 = (float*)P.p;
  float* o32 = (float*)P.q;
  launch(P, k_user_to_slots<float>, cdiv(g.n, 256), 256, 0, g, u_dev, u32);
  EpiStore<float, float> e{o32, g.n};
  fine_apply<float>(P, u32, e, nullptr);
  springs_apply(P, (const float*)u32, o32, 1.0, nullptr);
  launch(P, k_slots_to_user<float>, cdiv(g.n, 256), 256, 0, g, (const float*)o32, out_dev);
  API_END
}

// Same product through the dense kernel (used by tests as an independent path).
int edge_matvec_dense(edge_problem* p, const double* u_dev, double* out_dev) {
  API_BEGIN
  if (!p || !u_dev || !out_dev) fail(EDGE_EINVAL, "null argument");
  Prob& P = p->P;
  if (!P.has_rho) fail(EDGE_ESTATE, "Rho has not been set. dot works only after setting rho.");
  const Geo& g = P.g0;
  launch(P, k_user_to_slots<double>, cdiv(g.n, 256), 256, 0, g, u_dev, P.b64);
  EpiStore<double, double> e{P.r64, g.n};
  fine_apply_dense<double>(P, P.b64, e, nullptr);
  springs_apply(P, (const double*)P.b64, P.r64, 1.0, nullptr);
  launch(P, k_slots_to_user<double>, cdiv(g.n, 256), 256, 0, g, P.r64, out_dev);
  KCHECK();
  API_END
}

int edge_diagonal(edge_problem* p, double* diag_dev) {
  API_BEGIN
  if (!p || !diag_dev) fail(EDGE_EINVAL, "null argument");
  Prob& P = p->P;
  if (!P.has_rho) fail(EDGE_ESTATE, "Rho has not been set. diagonal works only after setting rho or if rho is provided.");
  const Geo& g = P.g0;
  launch(P, k_fine_dinv<double, double>, cdiv(g.n, 256), 256, 0, g, P.E64, P.mask, P.dK0diag, P.r64, diag_dev);
  if (P.n_springs)
    launch(P, k_springs_diag, 1, 64, 0, P.n_springs, (const long long*)P.spr_flat, (const long long*)P.spr_user,
           (const double*)P.spr_k, g.n, (const uint8_t*)P.mask, diag_dev);
  KCHECK();
  API_END
}

int edge_process_grad(edge_problem* p, const double* U_dev, double* dk_dev) {
  API_BEGIN
  if (!p || !U_dev || !dk_dev) fail(EDGE_EINVAL, "null argument");
  Prob& P = p->P;
  const Geo& g = P.g0;
  launch(P, k_user_to_slots<double>, cdiv(g.n, 256), 256, 0, g, U_dev, P.b64);
  launch(P, k_dk<double>, cdiv(P.n_el, 256), 256, 0, g, P.b64, P.ei.k3, P.ei.k2, P.dK0b, P.ei.wht ? 1 : 0, dk_dev,
                                                         nullptr, nullptr, 0.0, 0.0);
  KCHECK();
  API_END
}

int edge_process_grad_adjoint(edge_problem* p, const double* U_dev, const double* V_dev, double* dk_dev) {
  API_BEGIN
  if (!p || !U_dev || !V_dev || !dk_dev) fail(EDGE_EINVAL, "null argument");
  Prob& P = p->P;
  const Geo& g = P.g0;
  launch(P, k_user_to_slots<double>, cdiv(g.n, 256), 256, 0, g, U_dev, P.b64);
  launch(P, k_user_to_slots<double>, cdiv(g.n, 256), 256, 0, g, V_dev, P.r64);
  launch(P, k_dk2, cdiv(P.n_el, 256), 256, 0, g, (const double*)P.b64, (const double*)P.r64, P.ei.k3, P.ei.k2,
         (const double*)P.dK0b, P.ei.wht ? 1 : 0, dk_dev);
  KCHECK();
  API_END
}

int edge_set_springs(edge_problem* p, int n, const long long* dofs, const double* k) {
  API_BEGIN
  if (!p) fail(EDGE_EINVAL, "null handle");
  Prob& P = p->P;
  if (n < 0 || n > Prob::MAX_SPRINGS)
    fail(EDGE_EINVAL, "number of springs must be in [0, " + std::to_string(Prob::MAX_SPRINGS) + "]");
  if (n > 0 && (!dofs || !k)) fail(EDGE_EINVAL, "null argument");
  const Geo& g = P.g0;
  const long long ndof = P.n_dof;
  std::vector<long long> flat(n), user(n);
  std::vector<double> kv(n);
  for (int t = 0; t < n; ++t) {
    if (dofs[t] < 0 || dofs[t] >= ndof) fail(EDGE_EINVAL, "spring DOF index out of range");
    if (!(k[t] >= 0.0) || !std::isfinite(k[t])) fail(EDGE_EINVAL, "spring stiffness must be finite and >= 0");
    const long long node = dofs[t] / g.dof;
    const int c = (int)(dofs[t] % g.dof);
    long long slot;
    if (g.dim == 3) {
      const long long per_j = (long long)g.nx * g.nz;
      const int j = (int)(node / per_j), i = (int)((node % per_j) / g.nz), kz = (int)(node % g.nz);
      slot = g.slot3(i, j, kz);
    } else {
      const int j = (int)(node / g.nx), i = (int)(node % g.nx);
      slot = g.slot2(i, j);
    }
    flat[t] = (long long)c * g.n + slot;
    user[t] = dofs[t];
    kv[t] = k[t];
  }
  if (!P.spr_flat) {
    P.spr_flat = P.alloc<long long>(Prob::MAX_SPRINGS);
    P.spr_user = P.alloc<long long>(Prob::MAX_SPRINGS);
    P.spr_k = P.alloc<double>(Prob::MAX_SPRINGS);
  }
  CK(cudaStreamSynchronize(P.stream));
  if (n) {
    CK(cudaMemcpy(P.spr_flat, flat.data(), n * sizeof(long long), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(P.spr_user, user.data(), n * sizeof(long long), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(P.spr_k, kv.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  }
  P.n_springs = n;
  API_END
}

int edge_mg_config(edge_problem* p, int n_level, int n_smooth, double omega, double min_omega, int cycle_w,
                   const int* w_levels, int n_w, int precision) {
  API_BEGIN
  if (!p) fail(EDGE_EINVAL, "null handle");
  Prob& P = p->P;
  if (precision != EDGE_FP64 && precision != EDGE_MIXED) fail(EDGE_EINVAL, "unknown precision");
  if (n_level < 1 || n_smooth < 0) fail(EDGE_EINVAL, "n_level must be >= 1 and n_smooth >= 0");
  for (int l = 1; l <= n_level; ++l) {
    Geo g = level_geo(P, l);
    if (g.nx < 2 || g.ny < 2 || (P.dim == 3 && g.nz < 2))
      fail(EDGE_EINVAL, "n_level too large for this mesh: level " + std::to_string(l) + " has no elements");
  }
  cudaStreamSynchronize(P.stream);
  const bool realloc = (n_level != P.n_level) || (precision != P.prec);
  P.n_smooth = n_smooth;
  P.omega = omega;
  P.min_omega = std::max(omega / 2, min_omega);
  P.cycle_w = cycle_w != 0;
  P.w_levels.assign(w_levels, w_levels + (w_levels ? n_w : 0));
  if (realloc) {
    // free the old hierarchy
    for (auto& Lv : P.lv) {
      for (void* q : {Lv.b, Lv.xa, Lv.xb, Lv.r, Lv.ea, Lv.eb, Lv.res, Lv.S, Lv.S16, Lv.S16t, Lv.dinv}) {
        if (!q) continue;
        auto it = std::find(P.allocs.begin(), P.allocs.end(), q);
        if (it != P.allocs.end()) {
          cudaFree(q);
          P.allocs.erase(it);
        }
      }
    }
    for (void* q : {(void*)P.Adense, (void*)P.Ainv, (void*)P.Ut, (void*)P.gal_t1, (void*)P.gal_t2}) {
      if (!q) continue;
      auto it = std::find(P.allocs.begin(), P.allocs.end(), q);
      if (it != P.allocs.end()) {
        cudaFree(q);
        P.allocs.erase(it);
      }
    }
    // p and q are shared by both precisions (FP64-sized, read as FP32 by the mixed path): the
    // operator never writes their padding slots, which the PCG vector kernels sweep over, so
    // bytes left by the other precision must not survive a switch
    if (precision != P.prec) {
      const size_t nv = (size_t)P.g0.dof * P.g0.n;
      CK(cudaMemsetAsync(P.p, 0, nv * sizeof(double), P.stream));
      CK(cudaMemsetAsync(P.q, 0, nv * sizeof(double), P.stream));
    }
    P.n_level = n_level;
    P.prec = precision;
    P.tmaps.clear();
    P.sg_key.clear();  // the solve graph refers to the old buffers: capture again
    mg_allocate(P);
  }
  API_END
}

int edge_mg_solve(edge_problem* p, const double* f_dev, double* x_dev, int use_last, double tol, int maxiter,
                  double* residual_out, int* iters_out) {
  API_BEGIN
  if (!p || !f_dev || !x_dev) fail(EDGE_EINVAL, "null argument");
  Prob& P = p->P;
  const Geo& g = P.g0;
  launch(P, k_user_to_slots<double>, cdiv(g.n, 256), 256, 0, g, f_dev, P.b64);
  if (use_last)
    launch(P, k_user_to_slots<double>, cdiv(g.n, 256), 256, 0, g, x_dev, P.x64);
  else
    CK(cudaMemsetAsync(P.x64, 0, (size_t)g.dof * g.n * sizeof(double), P.stream));
  KCHECK();
  solve_internal(P, tol, maxiter);
  launch(P, k_slots_to_user<double>, cdiv(g.n, 256), 256, 0, g, P.x64, x_dev);
  KCHECK();
  CK(cudaStreamSynchronize(P.stream));
  if (residual_out) *residual_out = P.st_h->res;
  if (iters_out) *iters_out = P.st_h->iter;
  API_END
}

int edge_cg_solve(edge_problem* p, const double* f_dev, double* x_dev, int use_last, double tol, int maxiter,
                  double* residual_out, int* iters_out) {
  API_BEGIN
  if (!p || !f_dev || !x_dev) fail(EDGE_EINVAL, "null argument");
  if (tol <= 0.0 || maxiter < 1) fail(EDGE_EINVAL, "tol must be > 0 and maxiter >= 1");
  Prob& P = p->P;
  if (!P.has_rho) fail(EDGE_ESTATE, "Solver requires a density vector to be passed or set on the kernel.");
  const Geo& g = P.g0;
  launch(P, k_user_to_slots<double>, cdiv(g.n, 256), 256, 0, g, f_dev, P.b64);
  if (use_last)
    launch(P, k_user_to_slots<double>, cdiv(g.n, 256), 256, 0, g, x_dev, P.x64);
  else
    CK(cudaMemsetAsync(P.x64, 0, (size_t)g.dof * g.n * sizeof(double), P.stream));
  solve_graph(P, tol, maxiter, true);
  check_err(P);
  launch(P, k_slots_to_user<double>, cdiv(g.n, 256), 256, 0, g, P.x64, x_dev);
  CK(cudaStreamSynchronize(P.stream));
  if (residual_out) *residual_out = P.st_h->res;
  if (iters_out) *iters_out = P.st_h->iter;
  API_END
}

int edge_fea_integrals(edge_problem* p, const double* U_dev, const double* w_dev, const double* B_dev,
                       const double* D_dev, int nb, double* strain_dev, double* stress_dev, double* energy_dev) {
  API_BEGIN
  if (!p || !U_dev || !w_dev || !B_dev || !D_dev || !strain_dev || !stress_dev || !energy_dev)
    fail(EDGE_EINVAL, "null argument");
  Prob& P = p->P;
  if (nb < 1 || nb > 6) fail(EDGE_EINVAL, "strain size must be in 1..6");
  launch(P, k_fea_integrals, std::min<unsigned>(cdiv(P.n_el, 128), 148u * 32u), 128, 0, P.dim, P.nel[0], P.nel[1],
         P.dim == 3 ? P.nel[2] : 1, P.n_el, U_dev, w_dev, (const double*)P.dK0ref, B_dev, D_dev, nb, strain_dev,
         stress_dev, energy_dev);
  CK(cudaStreamSynchronize(P.stream));
  API_END
}

int edge_profile_begin(edge_problem* p, int max_launches) {
  API_BEGIN
  if (!p || max_launches < 1) fail(EDGE_EINVAL, "bad argument");
  Prob& P = p->P;
  while ((int)P.pev.size() < 2 * max_launches) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    P.pev.push_back(e);
  }
  P.pev_used = 0;
  P.pbytes.clear();
  P.pbytes.reserve(max_launches);
  P.prof = true;
  P.nlaunch = 0;
  API_END
}

int edge_profile_end(edge_problem* p, double* kernel_ms, double* kernel_bytes, int* kernel_launches,
                     long long* total_launches) {
  API_BEGIN
  if (!p) fail(EDGE_EINVAL, "null handle");
  Prob& P = p->P;
  CK(cudaStreamSynchronize(P.stream));
  double ms = 0.0, by = 0.0;
  for (size_t i = 0; i + 1 < P.pev_used; i += 2) {
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, P.pev[i], P.pev[i + 1]));
    ms += t;
    by += P.pbytes[i / 2];
  }
  if (kernel_ms) *kernel_ms = ms;
  if (kernel_bytes) *kernel_bytes = by;
  if (kernel_launches) *kernel_launches = (int)(P.pev_used / 2);
  if (total_launches) *total_launches = P.nlaunch;
  P.prof = false;
  API_END
}

int edge_mg_setup(edge_problem* p) {
  API_BEGIN
  if (!p) fail(EDGE_EINVAL, "null handle");
  Prob& P = p->P;
  ensure_mg(P);
  if (!P.has_rho) fail(EDGE_ESTATE, "rho not set");
  if (P.prec == EDGE_FP64)
    mg_setup<double, double>(P);
  else
    mg_setup<float, __nv_bfloat16>(P);
  CK(cudaStreamSynchronize(P.stream));
  API_END
}

int edge_mg_level_dense(edge_problem* p, int level, double* out_dev, long long n) {
  API_BEGIN
  if (!p || !out_dev) fail(EDGE_EINVAL, "null argument");
  Prob& P = p->P;
  ensure_mg(P);
  if (level < 1 || level > P.n_level) fail(EDGE_EINVAL, "level must be in [1, n_level]");
  const Geo& g = P.lv[level].g;
  const long long nd = (long long)g.nx * g.ny * g.nz * g.dof;
  if (n != nd) fail(EDGE_EINVAL, "dense size mismatch: level has " + std::to_string(nd) + " DOFs");
  CK(cudaMemsetAsync(out_dev, 0, (size_t)nd * nd * sizeof(double), P.stream));
  if (P.prec == EDGE_FP64)
    launch(P, k_st_to_dense<double>, cdiv(g.n, 256), 256, 0, g, (const double*)P.lv[level].S, out_dev, (int)nd);
  else
    launch(P, k_st_to_dense<float>, cdiv(g.n, 256), 256, 0, g, (const float*)P.lv[level].S, out_dev, (int)nd);
  CK(cudaStreamSynchronize(P.stream));
  API_END
}

int edge_jacobi_sweep(edge_problem* p, int level, const double* x_dev, const double* b_dev, double omega, int n_step,
                      double* out_dev) {
  API_BEGIN
  if (!p || !x_dev || !b_dev || !out_dev) fail(EDGE_EINVAL, "null argument");
  Prob& P = p->P;
  ensure_mg(P);
  if (P.prec != EDGE_FP64) fail(EDGE_ESTATE, "the standalone smoother needs the FP64 hierarchy (precision EDGE_FP64)");
  if (level < 0 || level >= P.n_level || (int)P.lv.size() <= level)
    fail(EDGE_EINVAL, "level must be a smoothed level, 0 <= level < n_level");
  if (!P.has_rho) fail(EDGE_ESTATE, "rho not set");
  if (n_step < 0) fail(EDGE_EINVAL, "n_step must be >= 0");
  Level& Lv = P.lv[level];
  const Geo& g = Lv.g;
  double* x = (double*)Lv.xa;
  double* y = (double*)Lv.xb;
  double* b = (double*)Lv.r;
  launch(P, k_user_to_slots<double>, cdiv(g.n, 256), 256, 0, g, x_dev, x);
  launch(P, k_user_to_slots<double>, cdiv(g.n, 256), 256, 0, g, b_dev, b);
  CK(cudaMemcpyAsync(P.scal + 8, &omega, sizeof(double), cudaMemcpyHostToDevice, P.stream));
  for (int s = 0; s < n_step; ++s) {
    EpiJacobi<double, double, double> e{b, (const double*)Lv.dinv, y, P.scal + 8, 1.0, g.n};
    level_apply<double>(P, level, x, e);
    std::swap(x, y);
  }
  launch(P, k_slots_to_user<double>, cdiv(g.n, 256), 256, 0, g, (const double*)x, out_dev);
  KCHECK();
  CK(cudaStreamSynchronize(P.stream));
  check_err(P);
  API_END
}

int edge_breakdown_begin(edge_problem* p, int max_launches) {
  API_BEGIN
  if (!p || max_launches < 1) fail(EDGE_EINVAL, "bad argument");
  Prob& P = p->P;
  while ((int)P.bev.size() < 2 * max_launches) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    P.bev.push_back(e);
  }
  P.bev_used = 0;
  P.bcat.clear();
  P.bd = true;
  API_END
}

int edge_breakdown_end(edge_problem* p, double* ms_by_cat, int* n_by_cat, int n_cat) {
  API_BEGIN
  if (!p || !ms_by_cat || !n_by_cat) fail(EDGE_EINVAL, "null argument");
  Prob& P = p->P;
  CK(cudaStreamSynchronize(P.stream));
  for (int c = 0; c < n_cat; ++c) {
    ms_by_cat[c] = 0.0;
    n_by_cat[c] = 0;
  }
  for (size_t i = 0; i + 1 < P.bev_used; i += 2) {
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, P.bev[i], P.bev[i + 1]));
    const int c = P.bcat[i / 2];
    if (c < n_cat) {
      ms_by_cat[c] += t;
      n_by_cat[c] += 1;
    }
  }
  P.bd = false;
  API_END
}

int edge_last_solve_stats(const edge_problem* p, double* setup_ms, double* solve_ms, int* pcg_iters,
                          int* true_residuals) {
  API_BEGIN
  if (!p) fail(EDGE_EINVAL, "null handle");
  const Prob& P = p->P;
  if (setup_ms) *setup_ms = P.last_setup_ms;
  if (solve_ms) *solve_ms = P.last_solve_ms;
  if (pcg_iters) *pcg_iters = P.last_iters;
  if (true_residuals) *true_residuals = P.last_true_res;
  API_END
}

static void transfer(int dim, const int* nel, const double* in_dev, double* out_dev, void* stream, bool restrict_) {
  if (dim != 2 && dim != 3) fail(EDGE_EINVAL, "dim must be 2 or 3");
  Geo gf = make_geo(dim, nel[0], nel[1], dim == 3 ? nel[2] : 0);
  Geo gc = make_geo(dim, nel[0] / 2, nel[1] / 2, dim == 3 ? nel[2] / 2 : 0);
  cudaStream_t s = (cudaStream_t)stream;
  double *vf = nullptr, *vc = nullptr;
  CK(cudaMallocAsync((void**)&vf, (size_t)gf.dof * gf.n * sizeof(double), s));
  CK(cudaMallocAsync((void**)&vc, (size_t)gc.dof * gc.n * sizeof(double), s));
  if (restrict_) {
    k_user_to_slots<double><<<cdiv(gf.n, 256), 256, 0, s>>>(gf, in_dev, vf);
    if (dim == 3)
      k_restrict3<double, double><<<dim3(cdiv((long long)gc.nz * gc.nx, 256), gc.ny), 256, 0, s>>>(gf, gc, vf, vc);
    else
      k_restrict2<double, double><<<dim3(cdiv(gc.nx, 64), gc.ny), 64, 0, s>>>(gf, gc, vf, vc);
    k_slots_to_user<double><<<cdiv(gc.n, 256), 256, 0, s>>>(gc, vc, out_dev);
  } else {
    CK(cudaMemsetAsync(vc, 0, (size_t)gc.dof * gc.n * sizeof(double), s));
    k_user_to_slots<double><<<cdiv(gc.n, 256), 256, 0, s>>>(gc, in_dev, vc);
    if (dim == 3)
      k_prolong3<double, double><<<dim3(cdiv((long long)gc.nz * gc.nx, 256), gc.ny), 256, 0, s>>>(gf, gc, vc, vf);
    else
      k_prolong2<double, double><<<dim3(cdiv(gf.nx, 64), gf.ny), 64, 0, s>>>(gf, gc, vc, vf);
    k_slots_to_user<double><<<cdiv(gf.n, 256), 256, 0, s>>>(gf, vf, out_dev);
  }
  KCHECK();
  CK(cudaFreeAsync(vf, s));
  CK(cudaFreeAsync(vc, s));
}

int edge_mm_law(long long n_el, int n_mat, const double* rho_dev, const double* E_mat, double void_, double penalty,
                int plain, double* E_dev, double* dE_dev, void* stream) {
  API_BEGIN
  if (!rho_dev || !E_mat || !E_dev) fail(EDGE_EINVAL, "null argument");
  if (n_el < 0 || n_mat < 1 || n_mat > MM_MAX)
    fail(EDGE_EINVAL, "n_mat must be in 1.." + std::to_string(MM_MAX) + " and n_el >= 0");
  if (!std::isfinite(penalty) || !std::isfinite(void_)) fail(EDGE_EINVAL, "penalty and void must be finite");
  if (n_el == 0) return EDGE_OK;
  MMat em{};
  for (int m = 0; m < n_mat; ++m) em.e[m] = E_mat[m];
  k_mm_law<<<std::min<unsigned>(cdiv(n_el, 256), 148u * 16u), 256, 0, (cudaStream_t)stream>>>(
      n_el, n_mat, rho_dev, em, void_, penalty, plain, E_dev, dE_dev);
  KCHECK();
  API_END
}

int edge_oc_update_multi(long long n_el, int n_sets, const double* rho_dev, const double* ocp_dev, const double* A_dev,
                         int A_per_element, double move, double vol, const double* mass, const double* rho_mat,
                         double* rho_new_dev, void* stream) {
  API_BEGIN
  if (!rho_dev || !ocp_dev || !A_dev || !mass || !rho_new_dev) fail(EDGE_EINVAL, "null argument");
  if (n_el < 1 || n_sets < 1 || n_sets > MM_MAX)
    fail(EDGE_EINVAL, "n_sets must be in 1.." + std::to_string(MM_MAX) + " and n_el >= 1");
  if (!(vol > 0.0)) fail(EDGE_EINVAL, "vol must be positive");
  MmOcCon cn{};
  cn.ns = n_sets;
  cn.shared = rho_mat ? 1 : 0;
  for (int m = 0; m < n_sets; ++m) {
    cn.mass[m] = rho_mat ? mass[0] : mass[m];
    cn.rm[m] = rho_mat ? rho_mat[m] : 0.0;
  }
  k_oc_multi<<<1, 1024, 0, (cudaStream_t)stream>>>(n_el, cn, rho_dev, ocp_dev, A_dev, A_per_element ? 1 : 0, move,
                                                   vol, rho_new_dev, nullptr);
  KCHECK();
  API_END
}

int edge_restrict(int dim, const int* nel, const double* in_dev, double* out_dev, void* stream) {
  API_BEGIN
  if (!nel || !in_dev || !out_dev) fail(EDGE_EINVAL, "null argument");
  transfer(dim, nel, in_dev, out_dev, stream, true);
  API_END
}

int edge_prolong(int dim, const int* nel, const double* in_dev, double* out_dev, void* stream) {
  API_BEGIN
  if (!nel || !in_dev || !out_dev) fail(EDGE_EINVAL, "null argument");
  transfer(dim, nel, in_dev, out_dev, stream, false);
  API_END
}

int edge_filter_create(int dim, const int* nel, int n_taps, const int* offsets, const double* weights,
                       edge_filter** out) {
  API_BEGIN
  if (!nel || !offsets || !weights || !out) fail(EDGE_EINVAL, "null argument");
  if (dim != 2 && dim != 3) fail(EDGE_EINVAL, "dim must be 2 or 3");
  if (n_taps < 1 || n_taps > MAX_TAPS) fail(EDGE_EINVAL, "filter radius gives " + std::to_string(n_taps) + " taps (max " + std::to_string(MAX_TAPS) + ")");
  auto* f = new edge_filter();
  f->g = make_geo(dim, nel[0], nel[1], dim == 3 ? nel[2] : 0);
  f->n_el = (long long)nel[0] * nel[1] * (dim == 3 ? nel[2] : 1);
  f->taps.n = n_taps;
  for (int t = 0; t < n_taps; ++t) {
    for (int d = 0; d < 3; ++d) f->taps.off[t][d] = offsets[t * 3 + d];
    f->taps.w[t] = weights[t];
  }
  cudaError_t e = cudaMalloc(&f->N, f->n_el * sizeof(double));
  if (e != cudaSuccess) {
    delete f;
    fail(EDGE_ECUDA, cudaGetErrorString(e));
  }
  k_filter_norm<<<cdiv(f->n_el, 256), 256>>>(f->g, f->taps, f->N);
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    delete f;
    fail(EDGE_ECUDA, cudaGetErrorString(e));
  }
  *out = f;
  API_END
}

int edge_filter_destroy(edge_filter* f) {
  API_BEGIN
  delete f;
  API_END
}

int edge_filter_apply(edge_filter* f, const double* in_dev, double* out_dev, void* stream) {
  API_BEGIN
  if (!f || !in_dev || !out_dev) fail(EDGE_EINVAL, "null argument");
  k_filter<<<cdiv(f->n_el, 256), 256, 0, (cudaStream_t)stream>>>(f->g, f->taps, in_dev, out_dev);
  KCHECK();
  API_END
}

int edge_filter_apply_T(edge_filter* f, const double* in_dev, double* out_dev, void* stream) {
  API_BEGIN
  if (!f || !in_dev || !out_dev) fail(EDGE_EINVAL, "null argument");
  k_filter_T<<<cdiv(f->n_el, 256), 256, 0, (cudaStream_t)stream>>>(f->g, f->taps, f->N, in_dev, out_dev);
  KCHECK();
  API_END
}

static void oc_run(Prob& P, long long n, const double* rho, const double* dr, double A, double vol, double vf,
                   double move, double* rho_new) {
  CatScope cat(P, CAT_OC);
  if (n != P.n_el) fail(EDGE_EINVAL, "OC vector length does not match the number of elements");
  const unsigned nb = std::min<unsigned>(ew_blocks(n), 1024);
  launch(P, k_oc_prep, nb, 256, 0, n, rho, dr, A, P.ocp, P.part, P.ticket, P.scal);
  launch(P, k_oc_floor, nb, 256, 0, n, P.ocp, P.scal);
  OcState init{};
  init.l1 = 1e-9;
  init.l2 = 1e9;
  init.last = 0.5 * (init.l1 + init.l2);
  init.vf = vf;
  init.vol = vol;
  *P.oc_h = init;
  CK(cudaMemcpyAsync(P.oc, P.oc_h, sizeof(OcState), cudaMemcpyHostToDevice, P.stream));
  const unsigned nbp = std::min<unsigned>(nb, (unsigned)(P.part_cap / OC_NODES));
  const int max_pass = (200 + OC_DEPTH - 1) / OC_DEPTH;
  for (int pass = 0; pass < max_pass; ++pass) {
    launch(P, k_oc_pass, nbp, 256, 0, n, rho, P.ocp, A, move, P.oc, P.part, P.ticket);
    if ((pass & 3) == 3) {
      CK(cudaMemcpyAsync(P.oc_h, P.oc, sizeof(OcState), cudaMemcpyDeviceToHost, P.stream));
      CK(cudaStreamSynchronize(P.stream));
      if (P.oc_h->done) break;
    }
  }
  KCHECK();
  launch(P, k_oc_final, nb, 256, 0, n, rho, P.ocp, move, P.oc, rho_new, P.part, P.ticket, P.scal + 1);
  KCHECK();
  CK(cudaMemcpyAsync(P.oc_h, P.oc, sizeof(OcState), cudaMemcpyDeviceToHost, P.stream));
  CK(cudaMemcpyAsync(P.scal_h, P.scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, P.stream));
  CK(cudaStreamSynchronize(P.stream));
}


// ---- unstructured meshes (kernels/_cuda.py:305-815, solvers/_gpu.py:11-58, geom/_filters.py:278-298)
int edge_gen_create(int dof, long long n_nodes, long long n_el, const int* elem_ptr, const int* elem_flat,
                    const double* K, const long long* K_ptr, edge_gen** out) {
  API_BEGIN
  if (!out || !elem_ptr || !elem_flat || !K || !K_ptr) fail(EDGE_EINVAL, "null argument");
  if (dof < 1 || dof > 3 || n_nodes < 1 || n_el < 1) fail(EDGE_EINVAL, "bad mesh sizes");
  const long long nflat = elem_ptr[n_el];
  for (long long e = 0; e < n_el; ++e) {
    const int sz = elem_ptr[e + 1] - elem_ptr[e];
    if (sz < 1 || sz > 27) fail(EDGE_EINVAL, "element " + std::to_string(e) + " has " + std::to_string(sz) + " nodes");
    const long long nk = (long long)sz * dof;
    if (K_ptr[e + 1] - K_ptr[e] != nk * nk)
      fail(EDGE_EINVAL, "element " + std::to_string(e) + ": matrix size does not match its node count");
  }
  for (long long a = 0; a < nflat; ++a)
    if (elem_flat[a] < 0 || elem_flat[a] >= n_nodes) fail(EDGE_EINVAL, "connectivity refers to a missing node");
  // node -> (element, local corner), sorted by node, then element (counting sort)
  std::vector<long long> adj_ptr(n_nodes + 1, 0);
  for (long long a = 0; a < nflat; ++a) ++adj_ptr[elem_flat[a] + 1];
  for (long long i = 0; i < n_nodes; ++i) adj_ptr[i + 1] += adj_ptr[i];
  std::vector<long long> fill(adj_ptr.begin(), adj_ptr.end() - 1);
  std::vector<int> adj_el(nflat);
  std::vector<unsigned char> adj_loc(nflat);
  for (long long e = 0; e < n_el; ++e)
    for (int c = elem_ptr[e]; c < elem_ptr[e + 1]; ++c) {
      const long long slot = fill[elem_flat[c]]++;
      adj_el[slot] = (int)e;
      adj_loc[slot] = (unsigned char)(c - elem_ptr[e]);
    }
  std::unique_ptr<edge_gen> M(new edge_gen());
  M->G.dof = dof;
  M->G.n_nodes = n_nodes;
  M->G.n_el = n_el;
  M->n_dof = n_nodes * dof;
  M->G.elem_ptr = M->upload(elem_ptr, n_el + 1);
  M->G.elem_flat = M->upload(elem_flat, nflat);
  M->G.K_ptr = M->upload(K_ptr, n_el + 1);
  M->G.K = M->upload(K, (size_t)K_ptr[n_el]);
  M->G.adj_ptr = M->upload(adj_ptr.data(), n_nodes + 1);
  M->G.adj_el = M->upload(adj_el.data(), nflat);
  M->G.adj_loc = M->upload(adj_loc.data(), nflat);
  M->rho = M->alloc<double>(n_el);
  M->cons = M->alloc<uint8_t>(M->n_dof);
  CK(cudaMemset(M->cons, 0, M->n_dof));
  for (double** v : {&M->x, &M->r, &M->p, &M->q, &M->b}) *v = M->alloc<double>(M->n_dof);
  M->st = M->alloc<PcgState>(1);
  CK(cudaMallocHost(&M->st_h, sizeof(PcgState)));
  M->part = M->alloc<double>(1024);
  M->ticket = M->alloc<unsigned>(1);
  CK(cudaMemset(M->ticket, 0, sizeof(unsigned)));
  M->zero = M->alloc<int>(1);
  CK(cudaMemset(M->zero, 0, sizeof(int)));
  *out = M.release();
  API_END
}

int edge_gen_destroy(edge_gen* m) {
  API_BEGIN
  delete m;
  API_END
}

int edge_gen_set_stream(edge_gen* m, void* stream) {
  API_BEGIN
  if (!m) fail(EDGE_EINVAL, "null handle");
  m->stream = (cudaStream_t)stream;
  API_END
}

int edge_gen_set_rho(edge_gen* m, const double* rho_dev) {
  API_BEGIN
  if (!m || !rho_dev) fail(EDGE_EINVAL, "null argument");
  CK(cudaMemcpyAsync(m->rho, rho_dev, m->G.n_el * sizeof(double), cudaMemcpyDeviceToDevice, m->stream));
  m->has_rho = true;
  API_END
}

int edge_gen_set_constraints(edge_gen* m, const uint8_t* cons_dev) {
  API_BEGIN
  if (!m || !cons_dev) fail(EDGE_EINVAL, "null argument");
  CK(cudaMemcpyAsync(m->cons, cons_dev, m->n_dof, cudaMemcpyDeviceToDevice, m->stream));
  API_END
}

int edge_gen_matvec(edge_gen* m, const double* u_dev, double* out_dev) {
  API_BEGIN
  if (!m || !u_dev || !out_dev) fail(EDGE_EINVAL, "null argument");
  if (!m->has_rho) fail(EDGE_ESTATE, "Rho has not been set. dot works only after setting rho.");
  gen_matvec(*m, u_dev, out_dev, nullptr);
  API_END
}

int edge_gen_diagonal(edge_gen* m, double* diag_dev) {
  API_BEGIN
  if (!m || !diag_dev) fail(EDGE_EINVAL, "null argument");
  if (!m->has_rho) fail(EDGE_ESTATE, "Rho has not been set. diagonal works only after setting rho or if rho is provided.");
  glaunch(*m, k_gen_diagonal, gen_blocks(m->n_dof), 256, m->G, (const double*)m->rho, (const uint8_t*)m->cons,
          diag_dev);
  API_END
}

int edge_gen_process_grad(edge_gen* m, const double* U_dev, double* dk_dev) {
  API_BEGIN
  if (!m || !U_dev || !dk_dev) fail(EDGE_EINVAL, "null argument");
  glaunch(*m, k_gen_dk, gen_blocks(m->G.n_el), 256, m->G, U_dev, dk_dev);
  API_END
}

// CG without a preconditioner (cupyx.scipy.sparse.linalg.cg with M = None, as the reference's
// CG solver runs on general meshes), FP64, the structured solver's CG kernels on these
// vectors; one state read per iteration decides convergence (where cupyx's loop checks it).
int edge_gen_cg_solve(edge_gen* m, const double* f_dev, double* x_dev, int use_last, double tol, int maxiter,
                      double* residual_out, int* iters_out) {
  API_BEGIN
  if (!m || !f_dev || !x_dev) fail(EDGE_EINVAL, "null argument");
  if (!m->has_rho) fail(EDGE_ESTATE, "Solver requires a density vector to be passed or set on the kernel.");
  edge_gen& M = *m;
  const long long nv = M.n_dof;
  const unsigned nb = std::min<unsigned>(gen_blocks(nv), 1024);
  CK(cudaMemcpyAsync(M.b, f_dev, nv * sizeof(double), cudaMemcpyDeviceToDevice, M.stream));
  if (use_last)
    CK(cudaMemcpyAsync(M.x, x_dev, nv * sizeof(double), cudaMemcpyDeviceToDevice, M.stream));
  else
    CK(cudaMemsetAsync(M.x, 0, nv * sizeof(double), M.stream));
  glaunch(M, k_pcg_init, 1, 1, M.st, tol, maxiter, 0.0, 0.0, 0.0, 0);
  gen_matvec(M, M.x, M.r, nullptr);  // r = b - A x
  glaunch(M, k_axpby, gen_blocks(nv), 256, nv, 1.0, (const double*)M.b, -1.0, M.r);
  glaunch(M, k_dot<double, double>, nb, 256, nv, (const double*)M.b, (const double*)M.b, M.part, M.ticket, &M.st->bb);
  glaunch(M, k_dot<double, double>, nb, 256, nv, (const double*)M.r, (const double*)M.r, M.part, M.ticket, &M.st->rr);
  glaunch(M, k_pcg_check_bb, 1, 1, M.st, (const int*)M.zero);
  auto read = [&]() {
    CK(cudaMemcpyAsync(M.st_h, M.st, sizeof(PcgState), cudaMemcpyDeviceToHost, M.stream));
    CK(cudaStreamSynchronize(M.stream));
  };
  read();
  while (!M.st_h->done) {
    glaunch(M, k_cg_rz, 1, 1, M.st);
    glaunch(M, k_pcg_p<double>, gen_blocks(nv), 256, nv, M.p, (const double*)M.r, (const PcgState*)M.st);
    gen_matvec(M, M.p, M.q, &M.st->pq);
    glaunch(M, k_pcg_xr<double, double>, nb, 256, nv, M.x, (const double*)M.p, M.r, (const double*)M.q, M.st, M.part,
            M.ticket, (float*)nullptr);
    read();
  }
  M.last_iters = M.st_h->iter;
  // true residual ||f - K x|| / ||f||, as the reference reports it
  gen_matvec(M, M.x, M.r, nullptr);
  glaunch(M, k_axpby, gen_blocks(nv), 256, nv, 1.0, (const double*)M.b, -1.0, M.r);
  glaunch(M, k_dot<double, double>, nb, 256, nv, (const double*)M.r, (const double*)M.r, M.part, M.ticket, &M.st->rr);
  glaunch(M, k_final_res, 1, 1, M.st);
  CK(cudaMemcpyAsync(x_dev, M.x, nv * sizeof(double), cudaMemcpyDeviceToDevice, M.stream));
  read();
  if (residual_out) *residual_out = M.st_h->res;
  if (iters_out) *iters_out = M.last_iters;
  API_END
}

// CSR density filter of a general mesh: H and its transpose both stored as CSR (the
// transpose built on the host), applied by gather SpMVs in stored order.
struct edge_csr {
  long long n = 0;
  long long *ptr = nullptr, *ptrT = nullptr;
  int *idx = nullptr, *idxT = nullptr;
  double *val = nullptr, *valT = nullptr;
  ~edge_csr() {
    for (void* q : {(void*)ptr, (void*)ptrT, (void*)idx, (void*)idxT, (void*)val, (void*)valT})
      if (q) cudaFree(q);
  }
};

int edge_csr_create(long long n, const long long* indptr, const int* indices, const double* data, edge_csr** out) {
  API_BEGIN
  if (!out || !indptr || !indices || !data) fail(EDGE_EINVAL, "null argument");
  if (n < 1) fail(EDGE_EINVAL, "empty matrix");
  const long long nnz = indptr[n];
  for (long long a = 0; a < nnz; ++a)
    if (indices[a] < 0 || indices[a] >= n) fail(EDGE_EINVAL, "column index out of range");
  std::vector<long long> pT(n + 1, 0);
  for (long long a = 0; a < nnz; ++a) ++pT[indices[a] + 1];
  for (long long i = 0; i < n; ++i) pT[i + 1] += pT[i];
  std::vector<long long> fill(pT.begin(), pT.end() - 1);
  std::vector<int> iT(nnz);
  std::vector<double> vT(nnz);
  for (long long i = 0; i < n; ++i)
    for (long long a = indptr[i]; a < indptr[i + 1]; ++a) {
      const long long s = fill[indices[a]]++;
      iT[s] = (int)i;
      vT[s] = data[a];
    }
  std::unique_ptr<edge_csr> F(new edge_csr());
  F->n = n;
  auto up = [](auto*& d, const auto* h, size_t k) {
    CK(cudaMalloc((void**)&d, std::max<size_t>(k, 1) * sizeof(*h)));
    CK(cudaMemcpy(d, h, k * sizeof(*h), cudaMemcpyHostToDevice));
  };
  up(F->ptr, indptr, n + 1);
  up(F->idx, indices, nnz);
  up(F->val, data, nnz);
  up(F->ptrT, pT.data(), n + 1);
  up(F->idxT, iT.data(), nnz);
  up(F->valT, vT.data(), nnz);
  *out = F.release();
  API_END
}

int edge_csr_destroy(edge_csr* f) {
  API_BEGIN
  delete f;
  API_END
}

int edge_csr_apply(edge_csr* f, const double* in_dev, double* out_dev, int transpose, void* stream) {
  API_BEGIN
  if (!f || !in_dev || !out_dev) fail(EDGE_EINVAL, "null argument");
  const long long n = f->n;
  const unsigned nb = (unsigned)std::min<long long>(cdiv(n, 256), 148LL * 8);
  if (transpose)
    k_csr_spmv<<<nb, 256, 0, (cudaStream_t)stream>>>(n, f->ptrT, f->idxT, f->valT, in_dev, out_dev);
  else
    k_csr_spmv<<<nb, 256, 0, (cudaStream_t)stream>>>(n, f->ptr, f->idx, f->val, in_dev, out_dev);
  KCHECK();
  API_END
}

int edge_oc_update(edge_problem* p, const double* rho_dev, const double* dr_dev, double A, double vol, double vf,
                   double move, double* rho_new_dev, double* lambda_out, int* steps_out, double* sqchange_out) {
  API_BEGIN
  if (!p || !rho_dev || !dr_dev || !rho_new_dev) fail(EDGE_EINVAL, "null argument");
  Prob& P = p->P;
  oc_run(P, P.n_el, rho_dev, dr_dev, A, vol, vf, move, rho_new_dev);
  if (lambda_out) *lambda_out = P.oc_h->last;
  if (steps_out) *steps_out = P.oc_h->steps;
  if (sqchange_out) *sqchange_out = P.scal_h[1];
  API_END
}

int edge_oc_update_static(long long n, const double* rho_dev, const double* dr_dev, double A, double vol, double vf,
                          double move, double* rho_new_dev, double* lambda_out, int* steps_out, double* sqchange_out,
                          void* stream) {
  API_BEGIN
  if (!rho_dev || !dr_dev || !rho_new_dev) fail(EDGE_EINVAL, "null argument");
  if (n <= 0) fail(EDGE_EINVAL, "n must be positive");
  if (n > OC_STATIC_MAX_EL)
    fail(EDGE_EINVAL, "n = " + std::to_string(n) + " elements exceeds the fixed OC workspace (at most " +
                          std::to_string(OC_STATIC_MAX_EL) + " elements); use edge_oc_update");
  cudaStream_t st = (cudaStream_t)stream;
  OcStaticScratch* s = oc_static_scratch(st);
  const unsigned nb = std::min<unsigned>(ew_blocks(n), OC_STATIC_MAX_BLOCKS);
  k_oc_static_init<<<1, 1, 0, st>>>(s, vf, vol);
  k_oc_prep<<<nb, 256, 0, st>>>(n, rho_dev, dr_dev, A, s->ocp, s->part, &s->ticket, &s->scal[0]);
  k_oc_floor<<<nb, 256, 0, st>>>(n, s->ocp, &s->scal[0]);
  KCHECK();
  OcState h{};
  const int max_pass = (200 + OC_DEPTH - 1) / OC_DEPTH;
  for (int pass = 0; pass < max_pass; ++pass) {
    k_oc_pass<<<nb, 256, 0, st>>>(n, rho_dev, s->ocp, A, move, &s->st, s->part, &s->ticket);
    if ((pass & 3) == 3) {
      KCHECK();
      CK(cudaMemcpyAsync(&h, &s->st, sizeof(OcState), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      if (h.done) break;
    }
  }
  k_oc_final<<<nb, 256, 0, st>>>(n, rho_dev, s->ocp, move, &s->st, rho_new_dev, s->part, &s->ticket, &s->scal[1]);
  KCHECK();
  double chg = 0.0;
  CK(cudaMemcpyAsync(&h, &s->st, sizeof(OcState), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(&chg, &s->scal[1], sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (lambda_out) *lambda_out = h.last;
  if (steps_out) *steps_out = h.steps;
  if (sqchange_out) *sqchange_out = chg;
  API_END
}

// One SIMP iteration, OC update then analysis, as one graph launch and one host read
// (TopOpt/_cuda.py:242-302: update_design followed by solve_and_process).
int edge_simp_iteration(edge_problem* p, edge_filter* f, const double* rho_dev, const double* dr_dev, double A,
                        double vol, double vf, double move, double penalty, double void_, const double* f_dev,
                        double* U_dev, int use_last, double tol, int maxiter, double* rho_new_dev, double* dr_new_dev,
                        double* rho_f_dev, double* compliance_out, double* residual_out, int* iters_out,
                        double* lambda_out, int* oc_steps_out, double* sqchange_out) {
  API_BEGIN
  if (!p || !f || !rho_dev || !dr_dev || !f_dev || !U_dev || !rho_new_dev || !dr_new_dev)
    fail(EDGE_EINVAL, "null argument");
  Prob& P = p->P;
  if (f->n_el != P.n_el) fail(EDGE_EINVAL, "filter and mesh sizes differ");
  if (!P.use_graph || P.prof || P.bd)
    fail(EDGE_ESTATE, "edge_simp_iteration needs the graph solve (no profiling or breakdown in progress)");
  ensure_mg(P);
  const Geo& g = P.g0;
  const size_t eb = (size_t)P.n_el * sizeof(double);
  if (!P.it_rho) {  // once per problem
    P.it_rho = P.alloc<double>(P.n_el);
    P.it_dr = P.alloc<double>(P.n_el);
    P.it_rho_new = P.alloc<double>(P.n_el);
    P.it_dr_new = P.alloc<double>(P.n_el);
  }
  std::vector<double> key = graph_key(P, tol, maxiter);
  for (double v : {(double)(uintptr_t)f, A, vol, vf, move, penalty, void_}) key.push_back(v);
  if (!P.it_exec || key != P.it_key) {
    capture_iteration(P, *f, A, vol, vf, move, penalty, void_, tol, maxiter);
    P.it_key = key;
  }
  CK(cudaMemcpyAsync(P.it_rho, rho_dev, eb, cudaMemcpyDeviceToDevice, P.stream));
  CK(cudaMemcpyAsync(P.it_dr, dr_dev, eb, cudaMemcpyDeviceToDevice, P.stream));
  launch(P, k_user_to_slots<double>, cdiv(g.n, 256), 256, 0, g, f_dev, P.b64);
  if (use_last)
    launch(P, k_user_to_slots<double>, cdiv(g.n, 256), 256, 0, g, (const double*)U_dev, P.x64);
  else
    CK(cudaMemsetAsync(P.x64, 0, (size_t)g.dof * g.n * sizeof(double), P.stream));
  CK(cudaEventRecord(P.ev[0], P.stream));
  CK(cudaGraphLaunch(P.it_exec, P.stream));
  CK(cudaEventRecord(P.ev[2], P.stream));
  P.has_rho = true;
  P.omega_started = true;
  CK(cudaMemcpyAsync(rho_new_dev, P.it_rho_new, eb, cudaMemcpyDeviceToDevice, P.stream));
  CK(cudaMemcpyAsync(dr_new_dev, P.it_dr_new, eb, cudaMemcpyDeviceToDevice, P.stream));
  if (rho_f_dev) CK(cudaMemcpyAsync(rho_f_dev, P.rho_f, eb, cudaMemcpyDeviceToDevice, P.stream));
  launch(P, k_slots_to_user<double>, cdiv(g.n, 256), 256, 0, g, (const double*)P.x64, U_dev);
  int status = 0;
  CK(cudaMemcpyAsync(&status, P.chol_status, sizeof(int), cudaMemcpyDeviceToHost, P.stream));
  CK(cudaMemcpyAsync(P.oc_h, P.oc, sizeof(OcState), cudaMemcpyDeviceToHost, P.stream));
  CK(cudaMemcpyAsync(P.scal_h, P.scal, 4 * sizeof(double), cudaMemcpyDeviceToHost, P.stream));
  read_state(P);  // synchronises the stream: the one host read of the iteration
  if (status) fail(EDGE_ENOTPD, "coarsest Galerkin matrix is not positive definite (missing boundary conditions?)");
  check_err(P);
  P.last_iters = P.st_h->iter;
  P.last_true_res = (P.prec != EDGE_FP64) ? 1 + P.st_h->n_true : 0;
  const long long passes = (P.oc_h->steps + OC_DEPTH - 1) / OC_DEPTH;
  P.nlaunch += P.it_fixed + P.it_body * (long long)P.st_h->iter + P.it_rep * (long long)P.st_h->n_true +
               P.it_oc_body * passes;
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, P.ev[0], P.ev[2]));
  P.last_setup_ms = 0.0;
  P.last_solve_ms = ms;
  if (compliance_out) *compliance_out = P.scal_h[2];
  if (residual_out) *residual_out = P.st_h->res;
  if (iters_out) *iters_out = P.st_h->iter;
  if (lambda_out) *lambda_out = P.oc_h->last;
  if (oc_steps_out) *oc_steps_out = P.oc_h->steps;
  if (sqchange_out) *sqchange_out = P.scal_h[1];
  API_END
}

int edge_simp_solve_and_process(edge_problem* p, edge_filter* f, const double* rho_dev, double penalty, double void_,
                                const double* f_dev, double* U_dev, int use_last, double tol, int maxiter,
                                double* compliance_out, double* dr_dev, double* rho_f_dev, double* residual_out,
                                int* iters_out) {
  API_BEGIN
  if (!p || !f || !rho_dev || !f_dev || !U_dev || !dr_dev) fail(EDGE_EINVAL, "null argument");
  Prob& P = p->P;
  CatScope cat(P, CAT_SENS);
  const Geo& g = P.g0;
  if (f->n_el != P.n_el) fail(EDGE_EINVAL, "filter and mesh sizes differ");
  double* rf = rho_f_dev ? rho_f_dev : P.rho_f;
  const unsigned nbe = cdiv(P.n_el, 256);
  // rho_f = H rho ; E = clip(rho_f^p, void, 1)
  launch(P, k_filter_material<double, float>, nbe, 256, 0, g, f->taps, rho_dev, rf, P.E64, P.E32, penalty, void_, 0);
  KCHECK();
  P.has_rho = true;
  // U = K(E)^-1 f (warm start from U_dev)
  launch(P, k_user_to_slots<double>, cdiv(g.n, 256), 256, 0, g, f_dev, P.b64);
  if (use_last)
    launch(P, k_user_to_slots<double>, cdiv(g.n, 256), 256, 0, g, U_dev, P.x64);
  else
    CK(cudaMemsetAsync(P.x64, 0, (size_t)g.dof * g.n * sizeof(double), P.stream));
  KCHECK();
  solve_internal(P, tol, maxiter);
  const long long nv = (long long)g.dof * g.n;
  // compliance c = f . U
  launch(P, k_dot<double, double>, std::min<unsigned>(ew_blocks(nv), 1024), 256, 0, nv, P.b64, P.x64, P.part,
                                                                                       P.ticket, P.scal + 2);
  // dr = H^T (p clip(rho_f)^(p-1) dk)
  launch(P, k_dk<double>, nbe, 256, 0, g, P.x64, P.ei.k3, P.ei.k2, P.dK0b, P.ei.wht ? 1 : 0, nullptr, rf, P.gsens,
                                          penalty, void_);
  launch(P, k_filter_T, nbe, 256, 0, f->g, f->taps, f->N, P.gsens, dr_dev);
  launch(P, k_slots_to_user<double>, cdiv(g.n, 256), 256, 0, g, P.x64, U_dev);
  KCHECK();
  CK(cudaMemcpyAsync(P.scal_h + 2, P.scal + 2, sizeof(double), cudaMemcpyDeviceToHost, P.stream));
  CK(cudaStreamSynchronize(P.stream));
  if (compliance_out) *compliance_out = P.scal_h[2];
  if (residual_out) *residual_out = P.st_h->res;
  if (iters_out) *iters_out = P.st_h->iter;
  API_END
}


}  // extern "C"

// ------------------------------------------------------------------ many 2-D problems, one solve launch
struct edge_batch {
  std::vector<edge_problem*> probs;
  std::vector<edge_filter*> filters;
  std::vector<int> nxr, nyr;  // real node extents (the problem's grid may be padded beyond them)
  // queue order of the solve: problems by decreasing expected cost, DOFs times the PCG
  // iterations of the problem's previous batched solve (DOFs alone before the first), so the
  // longest solves start first
  std::vector<int> order;
  std::vector<long long> cost;
  int threads = 512;
  int team = 1;  // blocks per problem (a thread block cluster when > 1)
  // with team > 1: problems with fewer DOFs than this are solved by single blocks of
  // small_threads threads in a launch beside the teams' (0, the default: every problem by a team;
  // at 256 problems of 5k-260k DOFs the split changed the solve launch's time by under 1 %)
  long long split_dof = 0;
  int small_threads = 1024;
  BatchDesc* d_desc = nullptr;
  BatchDesc* h_desc = nullptr;
  double** d_scal = nullptr;
  double** h_scal = nullptr;
  unsigned* queue = nullptr;
  double *d_res = nullptr, *d_comp = nullptr;
  int *d_iters = nullptr, *d_done = nullptr;
  double *h_res = nullptr, *h_comp = nullptr;
  int *h_iters = nullptr, *h_done = nullptr;
  BatchOcDesc* d_oc = nullptr;
  BatchOcDesc* h_oc = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // around the three phases of the last call
  long long* d_tns = nullptr;  // per problem (queue order): start and end of its solve (global timer, ns)
  long long* h_tns = nullptr;
  // the per-problem preparation and post-processing run on these streams side by side,
  // forked from and joined back into the caller's stream
  static constexpr int NSIDE = 16;
  cudaStream_t side[NSIDE] = {};
  cudaEvent_t fork = nullptr, join[NSIDE] = {};
  ~edge_batch() {
    for (auto st : side)
      if (st) cudaStreamDestroy(st);
    if (fork) cudaEventDestroy(fork);
    for (auto e : join)
      if (e) cudaEventDestroy(e);
    if (d_tns) cudaFree(d_tns);
    if (h_tns) cudaFreeHost(h_tns);
    for (auto e : ev)
      if (e) cudaEventDestroy(e);
    if (d_oc) cudaFree(d_oc);
    if (h_oc) cudaFreeHost(h_oc);
    for (void* q : {(void*)d_desc, (void*)d_scal, (void*)queue, (void*)d_res, (void*)d_comp, (void*)d_iters,
                    (void*)d_done})
      if (q) cudaFree(q);
    for (void* q : {(void*)h_desc, (void*)h_scal, (void*)h_res, (void*)h_comp, (void*)h_iters, (void*)h_done})
      if (q) cudaFreeHost(q);
  }
};

namespace edge {
// One persistent solve launch over the problems [off, off + cnt) of the queue order, on
// `stream`, with at most `sm_budget` SMs' worth of blocks (0: as many as fit).
template <typename TV, typename TD0, typename TS, int BT, int C>
static void batch_go(Prob& P0, edge_batch& B, int off, int cnt, int qslot, int sm_budget, cudaStream_t stream,
                     double tol, int maxiter) {
  auto kern = k_batch_pcg<TV, TD0, TS, BT, C>;
  int dev = 0, sms = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int budget = sm_budget > 0 ? std::min(sm_budget, sms) : sms;
  const BatchDesc* D = B.d_desc + off;
  long long* tns = B.d_tns + 2 * off;
  if constexpr (C == 1) {
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BT, 0));
    const int grid = std::max(1, std::min(cnt, std::max(1, per_sm) * budget));
    kern<<<grid, BT, 0, stream>>>(D, cnt, B.queue + qslot, tol, maxiter, tns);
  } else {
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C * sms);
    cfg.blockDim = dim3(BT);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int clusters = 0;
    CK(cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg));
    const int fit = std::max(1, clusters * budget / sms);
    const int teams = std::max(1, std::min(cnt, fit));
    cfg.gridDim = dim3(C * teams);
    CK(cudaLaunchKernelEx(&cfg, kern, D, cnt, B.queue + qslot, tol, maxiter, tns));
  }
  ++P0.nlaunch;
  KCHECK();
}
template <typename TV, typename TD0, typename TS, int BT>
static void batch_go_team(Prob& P0, edge_batch& B, int team, int off, int cnt, int qslot, int sm_budget,
                          cudaStream_t stream, double tol, int maxiter) {
  switch (team) {
    case 2: batch_go<TV, TD0, TS, BT, 2>(P0, B, off, cnt, qslot, sm_budget, stream, tol, maxiter); break;
    case 4: batch_go<TV, TD0, TS, BT, 4>(P0, B, off, cnt, qslot, sm_budget, stream, tol, maxiter); break;
    case 8: batch_go<TV, TD0, TS, BT, 8>(P0, B, off, cnt, qslot, sm_budget, stream, tol, maxiter); break;
    default: batch_go<TV, TD0, TS, BT, 1>(P0, B, off, cnt, qslot, sm_budget, stream, tol, maxiter); break;
  }
}
template <typename TV, typename TD0, typename TS>
static void batch_group(Prob& P0, edge_batch& B, int threads, int team, int off, int cnt, int qslot, int sm_budget,
                        cudaStream_t stream, double tol, int maxiter) {
  if (threads == 1024)
    batch_go_team<TV, TD0, TS, 1024>(P0, B, team, off, cnt, qslot, sm_budget, stream, tol, maxiter);
  else if (threads == 256 && team == 1)
    batch_go<TV, TD0, TS, 256, 1>(P0, B, off, cnt, qslot, sm_budget, stream, tol, maxiter);
  else
    batch_go_team<TV, TD0, TS, 512>(P0, B, team, off, cnt, qslot, sm_budget, stream, tol, maxiter);
}
// The solve launch(es): problems below B.split_dof DOFs (when a team of several blocks is
// configured) are solved by single blocks in a second launch beside the teams' launch, on its
// own share of the SMs (proportional to the groups' expected work), since a team's barriers
// dominate a small problem's iteration.
template <typename TV, typename TD0, typename TS>
static void batch_launch(Prob& P0, edge_batch& B, int n, int n_large, double w_large, double w_small,
                         cudaStream_t s, double tol, int maxiter) {
  if (B.team == 1 || n_large == n || n_large == 0) {
    batch_group<TV, TD0, TS>(P0, B, B.threads, B.team, 0, n, 0, 0, s, tol, maxiter);
    return;
  }
  int dev = 0, sms = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  int sm_large = (int)std::lround(sms * w_large / std::max(1e-30, w_large + w_small));
  sm_large = std::max(B.team, std::min(sms - 1, sm_large)) / B.team * B.team;
  CK(cudaEventRecord(B.fork, s));
  CK(cudaStreamWaitEvent(B.side[0], B.fork, 0));
  batch_group<TV, TD0, TS>(P0, B, B.threads, B.team, 0, n_large, 0, sm_large, s, tol, maxiter);
  batch_group<TV, TD0, TS>(P0, B, B.small_threads, 1, n_large, n - n_large, 1, sms - sm_large, B.side[0], tol,
                           maxiter);
  CK(cudaEventRecord(B.join[0], B.side[0]));
  CK(cudaStreamWaitEvent(s, B.join[0], 0));
}
}  // namespace edge

extern "C" {

int edge_batch_create(int n, edge_problem* const* problems, edge_filter* const* filters, const int* nelx,
                      const int* nely, edge_batch** out) {
  API_BEGIN
  if (n < 1 || !problems || !filters || !nelx || !nely || !out) fail(EDGE_EINVAL, "null argument or n < 1");
  auto B = std::make_unique<edge_batch>();
  std::vector<long long> dofs(n);
  for (int i = 0; i < n; ++i) {
    if (!problems[i] || !filters[i]) fail(EDGE_EINVAL, "null problem or filter");
    const Prob& P = problems[i]->P;
    const edge_filter& F = *filters[i];
    if (P.dim != 2 || F.g.dim != 2) fail(EDGE_EINVAL, "batched problems must be 2-D");
    if (nelx[i] < 1 || nely[i] < 1 || nelx[i] > P.nel[0] || nely[i] > P.nel[1])
      fail(EDGE_EINVAL, "problem " + std::to_string(i) + ": real extents outside the problem's grid");
    if (F.n_el != (long long)nelx[i] * nely[i])
      fail(EDGE_EINVAL, "problem " + std::to_string(i) + ": filter and real extents differ");
    B->probs.push_back(problems[i]);
    B->filters.push_back(filters[i]);
    B->nxr.push_back(nelx[i] + 1);
    B->nyr.push_back(nely[i] + 1);
    dofs[i] = P.n_dof;
  }
  B->order.resize(n);
  for (int i = 0; i < n; ++i) B->order[i] = i;
  B->cost = dofs;
  std::stable_sort(B->order.begin(), B->order.end(), [&](int a, int b) { return dofs[a] > dofs[b]; });
  CK(cudaMalloc(&B->d_desc, n * sizeof(BatchDesc)));
  CK(cudaMallocHost(&B->h_desc, n * sizeof(BatchDesc)));
  CK(cudaMalloc(&B->d_scal, n * sizeof(double*)));
  CK(cudaMallocHost(&B->h_scal, n * sizeof(double*)));
  CK(cudaMalloc(&B->queue, 2 * sizeof(unsigned)));
  CK(cudaMalloc(&B->d_res, n * sizeof(double)));
  CK(cudaMalloc(&B->d_comp, n * sizeof(double)));
  CK(cudaMalloc(&B->d_iters, n * sizeof(int)));
  CK(cudaMalloc(&B->d_done, n * sizeof(int)));
  CK(cudaMallocHost(&B->h_res, n * sizeof(double)));
  CK(cudaMallocHost(&B->h_comp, n * sizeof(double)));
  CK(cudaMallocHost(&B->h_iters, n * sizeof(int)));
  CK(cudaMallocHost(&B->h_done, n * sizeof(int)));
  std::memset(B->h_desc, 0, n * sizeof(BatchDesc));
  CK(cudaMalloc(&B->d_oc, n * sizeof(BatchOcDesc)));
  CK(cudaMallocHost(&B->h_oc, n * sizeof(BatchOcDesc)));
  for (auto& e : B->ev) CK(cudaEventCreate(&e));
  CK(cudaMalloc(&B->d_tns, 2 * n * sizeof(long long)));
  CK(cudaMallocHost(&B->h_tns, 2 * n * sizeof(long long)));
  for (auto& st : B->side) CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming));
  for (auto& e : B->join) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  *out = B.release();
  API_END
}

int edge_batch_destroy(edge_batch* b) {
  API_BEGIN
  delete b;
  API_END
}

int edge_batch_set_split(edge_batch* b, long long split_dof, int small_threads) {
  API_BEGIN
  if (!b || split_dof < 0 || (small_threads != 256 && small_threads != 512 && small_threads != 1024))
    fail(EDGE_EINVAL, "split_dof must be >= 0 and small_threads 256, 512 or 1024");
  b->split_dof = split_dof;
  b->small_threads = small_threads;
  API_END
}

int edge_batch_set_threads(edge_batch* b, int threads, int team) {
  API_BEGIN
  if (!b) fail(EDGE_EINVAL, "null handle");
  const bool ok = (team == 1 && (threads == 256 || threads == 512 || threads == 1024)) ||
                  ((team == 2 || team == 4 || team == 8) && (threads == 512 || threads == 1024));
  if (!ok) fail(EDGE_EINVAL, "supported: team 1 with 256, 512 or 1024 threads; team 2, 4 or 8 with 512 or 1024");
  b->threads = threads;
  b->team = team;
  API_END
}

int edge_batch_last_times(const edge_batch* b, double* setup_ms, double* solve_ms, double* post_ms) {
  API_BEGIN
  if (!b) fail(EDGE_EINVAL, "null handle");
  float a = 0, c = 0, d = 0;
  CK(cudaEventElapsedTime(&a, b->ev[0], b->ev[1]));
  CK(cudaEventElapsedTime(&c, b->ev[1], b->ev[2]));
  CK(cudaEventElapsedTime(&d, b->ev[2], b->ev[3]));
  if (setup_ms) *setup_ms = a;
  if (solve_ms) *solve_ms = c;
  if (post_ms) *post_ms = d;
  API_END
}

int edge_batch_last_problem_times(edge_batch* b, double* start_ms, double* end_ms) {
  API_BEGIN
  if (!b || !start_ms || !end_ms) fail(EDGE_EINVAL, "null argument");
  const int n = (int)b->probs.size();
  CK(cudaMemcpy(b->h_tns, b->d_tns, 2 * n * sizeof(long long), cudaMemcpyDeviceToHost));
  long long t0 = b->h_tns[0];
  for (int k = 0; k < n; ++k) t0 = std::min(t0, b->h_tns[2 * k]);
  for (int k = 0; k < n; ++k) {
    const int i = b->order[k];
    start_ms[i] = 1e-6 * (double)(b->h_tns[2 * k] - t0);
    end_ms[i] = 1e-6 * (double)(b->h_tns[2 * k + 1] - t0);
  }
  API_END
}

int edge_batch_oc_update(edge_batch* b, const double* const* rho, const double* const* dr, const double* A,
                         const double* vol, const double* vf, double move, double* const* rho_new, double* lambda_out,
                         int* steps_out, void* stream) {
  API_BEGIN
  if (!b || !rho || !dr || !A || !vol || !vf || !rho_new) fail(EDGE_EINVAL, "null argument");
  edge_batch& B = *b;
  const int n = (int)B.probs.size();
  cudaStream_t s = (cudaStream_t)stream;
  for (int k = 0; k < n; ++k) {
    const int i = B.order[k];
    if (!rho[i] || !dr[i] || !rho_new[i]) fail(EDGE_EINVAL, "null array of problem " + std::to_string(i));
    Prob& P = B.probs[i]->P;
    BatchOcDesc& d = B.h_oc[k];
    d.n = B.filters[i]->n_el;
    d.rho = rho[i];
    d.dr = dr[i];
    d.ocp = P.ocp;  // sized for the problem's grid, at least the real element count
    d.rho_new = rho_new[i];
    d.A = A[i];
    d.vol = vol[i];
    d.vf = vf[i];
  }
  Prob& P0 = B.probs[B.order[0]]->P;
  const cudaStream_t saved0 = P0.stream;
  P0.stream = s;
  try {
    CK(cudaMemcpyAsync(B.d_oc, B.h_oc, n * sizeof(BatchOcDesc), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(B.queue, 0, sizeof(unsigned), s));
    int per_sm = 0, sms = 0, dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_oc<512>, 512, 0));
    const int grid = std::max(1, std::min(n, std::max(1, per_sm) * sms));
    launch(P0, k_batch_oc<512>, dim3(grid), dim3(512), 0, (const BatchOcDesc*)B.d_oc, n, B.queue, move, B.d_res,
           B.d_iters);
  } catch (...) {
    P0.stream = saved0;
    throw;
  }
  P0.stream = saved0;
  if (lambda_out || steps_out) {
    CK(cudaMemcpyAsync(B.h_res, B.d_res, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(B.h_iters, B.d_iters, n * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (int k = 0; k < n; ++k) {
      if (lambda_out) lambda_out[B.order[k]] = B.h_res[k];
      if (steps_out) steps_out[B.order[k]] = B.h_iters[k];
    }
  }
  API_END
}

int edge_batch_solve_and_process(edge_batch* b, const double* const* rho, double penalty, double void_,
                                 const double* const* f, double* const* U, int use_last, double tol, int maxiter,
                                 double* compliance, double* const* dr, double* residual, int* iters, void* stream) {
  API_BEGIN
  if (!b || !rho || !f || !U || !dr) fail(EDGE_EINVAL, "null argument");
  if (tol <= 0.0 || maxiter < 1) fail(EDGE_EINVAL, "tol must be > 0 and maxiter >= 1");
  edge_batch& B = *b;
  const int n = (int)B.probs.size();
  cudaStream_t s = (cudaStream_t)stream;
  int prec = -1;
  bool bf16 = true;
  for (int i = 0; i < n; ++i) {
    if (!rho[i] || !f[i] || !U[i] || !dr[i]) fail(EDGE_EINVAL, "null array of problem " + std::to_string(i));
    Prob& P = B.probs[i]->P;
    ensure_mg(P);
    if (P.n_level < 1 || P.n_level >= BATCH_MAXL)
      fail(EDGE_EINVAL, "batched solves need 1 <= n_level < " + std::to_string(BATCH_MAXL));
    if (P.cycle_w) fail(EDGE_EINVAL, "batched solves run the V-cycle only");
    if (P.n_springs) fail(EDGE_EINVAL, "batched solves take no springs");
    if (prec >= 0 && P.prec != prec) fail(EDGE_EINVAL, "every problem of a batch must have the same precision");
    prec = P.prec;
    bf16 = bf16 && P.st_bf16;
  }
  const bool mixed = prec != EDGE_FP64;
  std::stable_sort(B.order.begin(), B.order.end(), [&](int a, int c) { return B.cost[a] > B.cost[c]; });
  // teams take the problems of at least split_dof DOFs (queue positions [0, n_large)), single
  // blocks the rest; expected work per group: sum of (DOFs + a fixed share for the per-iteration
  // steps) x the previous PCG iterations
  int n_large = n;
  double w_large = 0.0, w_small = 0.0;
  if (B.team > 1 && B.split_dof > 0) {
    auto big = [&](int i) { return B.probs[i]->P.n_dof >= B.split_dof; };
    std::stable_partition(B.order.begin(), B.order.end(), big);
    n_large = (int)std::count_if(B.order.begin(), B.order.end(), big);
    for (int k = 0; k < n; ++k) {
      const int i = B.order[k];
      const double its = (double)std::max<long long>(1, B.cost[i] / std::max<long long>(1, B.probs[i]->P.n_dof));
      const double w = its * ((double)B.probs[i]->P.n_dof + 25000.0);
      if (k < n_large) w_large += 1.2 * w;
      else w_small += w;
    }
  }
  CK(cudaEventRecord(B.ev[0], s));
  const int nside = std::min(n, edge_batch::NSIDE);
  auto fork = [&]() {
    CK(cudaEventRecord(B.fork, s));
    for (int q = 0; q < nside; ++q) CK(cudaStreamWaitEvent(B.side[q], B.fork, 0));
  };
  auto join = [&]() {
    for (int q = 0; q < nside; ++q) {
      CK(cudaEventRecord(B.join[q], B.side[q]));
      CK(cudaStreamWaitEvent(s, B.join[q], 0));
    }
  };
  // per problem: filter + SIMP law into the (possibly padded) grid, loads and warm starts,
  // the hierarchy for the new E
  fork();
  for (int k = 0; k < n; ++k) {
    const int i = B.order[k];
    Prob& P = B.probs[i]->P;
    const edge_filter& F = *B.filters[i];
    const cudaStream_t saved = P.stream;
    P.stream = B.side[k % nside];
    try {
      const Geo& g = P.g0;
      Geo gr = g;  // the real grid's extents in the problem's slot layout
      gr.nx = B.nxr[i];
      gr.ny = B.nyr[i];
      const unsigned nbe = cdiv(F.n_el, 256);
      launch(P, k_filter_material<double, float>, nbe, 256, 0, gr, F.taps, rho[i], P.rho_f, P.E64, P.E32, penalty,
             void_, 0);
      P.has_rho = true;
      launch(P, k_user_to_slots_pad, cdiv(g.n, 256), 256, 0, g, B.nxr[i], B.nyr[i], f[i], P.b64);
      if (use_last)
        launch(P, k_user_to_slots_pad, cdiv(g.n, 256), 256, 0, g, B.nxr[i], B.nyr[i], (const double*)U[i], P.x64);
      else
        CK(cudaMemsetAsync(P.x64, 0, (size_t)g.dof * g.n * sizeof(double), P.stream));
      mg_setup_prec(P);
      BatchDesc& d = B.h_desc[k];
      std::memset(&d, 0, sizeof(d));
      d.n_level = P.n_level;
      d.nd = P.nd;
      d.keep_omega = (P.omega_carry && P.omega_started) ? 1 : 0;
      for (int l = 0; l < BATCH_MAXL; ++l) {
        d.sweeps[l] = l < P.n_level ? P.sweeps(l) : 0;
        d.wscale[l] = std::pow(1.06, l);
      }
      d.omega = P.omega;
      d.min_omega = P.min_omega;
      d.omega0 = P.omega_carry ? P.omega : P.min_omega;
      d.mask = P.mask;
      d.E64 = P.E64;
      d.ET = mixed ? (const void*)P.E32 : (const void*)P.E64;
      d.K0_64 = P.dK0b;
      d.K0_T = mixed ? (const void*)P.dK0bf : (const void*)P.dK0b;
      d.b64 = P.b64;
      d.x64 = P.x64;
      d.r64 = P.r64;
      d.p64 = (double*)P.p;
      d.q64 = (double*)P.q;
      d.Ainv = P.Ainv;
      d.st = P.st;
      d.chol_status = P.chol_status;
      for (int l = 0; l <= P.n_level; ++l) {
        const Level& Lv = P.lv[l];
        BatchLevel& bl = d.lv[l];
        bl.g = Lv.g;
        bl.b = Lv.b;
        bl.xa = Lv.xa;
        bl.xb = Lv.xb;
        bl.r = Lv.r;
        bl.ea = Lv.ea;
        bl.eb = Lv.eb;
        bl.res = Lv.res;
        bl.S = (mixed && bf16 && Lv.S16) ? Lv.S16 : Lv.S;
        bl.dinv = Lv.dinv;
      }
      B.h_scal[k] = P.scal;
    } catch (...) {
      P.stream = saved;
      throw;
    }
    P.stream = saved;
  }
  join();
  // all solves in one launch
  Prob& P0 = B.probs[B.order[0]]->P;
  const cudaStream_t saved0 = P0.stream;
  P0.stream = s;
  try {
    CK(cudaMemcpyAsync(B.d_desc, B.h_desc, n * sizeof(BatchDesc), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(B.d_scal, B.h_scal, n * sizeof(double*), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(B.queue, 0, 2 * sizeof(unsigned), s));
    CK(cudaEventRecord(B.ev[1], s));
    if (!mixed)
      batch_launch<double, double, double>(P0, B, n, n_large, w_large, w_small, s, tol, maxiter);
    else if (bf16)
      batch_launch<float, __nv_bfloat16, __nv_bfloat16>(P0, B, n, n_large, w_large, w_small, s, tol, maxiter);
    else
      batch_launch<float, __nv_bfloat16, float>(P0, B, n, n_large, w_large, w_small, s, tol, maxiter);
  } catch (...) {
    P0.stream = saved0;
    throw;
  }
  P0.stream = saved0;
  CK(cudaEventRecord(B.ev[2], s));
  // per problem: compliance f . U, dr = H^T (dE/drho_f dk), U back in the user layout
  fork();
  for (int k = 0; k < n; ++k) {
    const int i = B.order[k];
    Prob& P = B.probs[i]->P;
    const edge_filter& F = *B.filters[i];
    const cudaStream_t saved = P.stream;
    P.stream = B.side[k % nside];
    try {
      const Geo& g = P.g0;
      Geo gr = g;
      gr.nx = B.nxr[i];
      gr.ny = B.nyr[i];
      const long long nv = (long long)g.dof * g.n;
      const unsigned nbe = cdiv(F.n_el, 256);
      launch(P, k_dot<double, double>, std::min<unsigned>(ew_blocks(nv), 1024), 256, 0, nv, (const double*)P.b64,
             (const double*)P.x64, P.part, P.ticket, P.scal + 2);
      launch(P, k_dk<double>, nbe, 256, 0, gr, (const double*)P.x64, P.ei.k3, P.ei.k2, (const double*)P.dK0b,
             P.ei.wht ? 1 : 0, (double*)nullptr, (const double*)P.rho_f, P.gsens, penalty, void_);
      launch(P, k_filter_T, nbe, 256, 0, F.g, F.taps, (const double*)F.N, (const double*)P.gsens, dr[i]);
      launch(P, k_slots_to_user_pad, cdiv(g.n, 256), 256, 0, g, B.nxr[i], B.nyr[i], (const double*)P.x64, U[i]);
    } catch (...) {
      P.stream = saved;
      throw;
    }
    P.stream = saved;
  }
  join();
  CK(cudaEventRecord(B.ev[3], s));
  k_batch_gather<<<cdiv(n, 128), 128, 0, s>>>(B.d_desc, (const double* const*)B.d_scal, n, B.d_res, B.d_comp,
                                               B.d_iters, B.d_done);
  KCHECK();
  CK(cudaMemcpyAsync(B.h_res, B.d_res, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(B.h_comp, B.d_comp, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(B.h_iters, B.d_iters, n * sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(B.h_done, B.d_done, n * sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  int bad = -1;
  for (int k = 0; k < n; ++k) {
    const int i = B.order[k];
    Prob& P = B.probs[i]->P;
    if (residual) residual[i] = B.h_res[k];
    if (iters) iters[i] = B.h_iters[k];
    if (compliance) compliance[i] = B.h_comp[k];
    P.st_h->res = B.h_res[k];
    P.st_h->iter = B.h_iters[k];
    P.st_h->done = B.h_done[k];
    P.last_iters = B.h_iters[k];
    P.last_true_res = 0;
    P.omega_started = true;
    B.cost[i] = P.n_dof * std::max(1, B.h_iters[k]);
    if (B.h_done[k] == 3 && bad < 0) bad = i;
  }
  if (bad >= 0)
    fail(EDGE_ENOTPD, "problem " + std::to_string(bad) +
                          ": coarsest Galerkin matrix is not positive definite (missing boundary conditions?)");
  API_END
}

}  // extern "C"
