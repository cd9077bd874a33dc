// Host runtime of the projection hot path: solver construction (flags, face
// lists, multigrid upload), launch orchestration of the substep / projection /
// Poisson solves, and the C ABI declared in include/pycfd_b200.h.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/pycfd_b200.h"
#include "boundary.cuh"
#include "common.cuh"
#include "multigrid.cuh"
#include "persistent.cuh"
#include "masks.cuh"
#include "adjoint.cuh"
#include "poisson.cuh"
#include "stencil.cuh"

using namespace pcfd;

static thread_local std::string g_err;

static int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CU(x)                                                                        \
  do {                                                                               \
    cudaError_t e_ = (x);                                                            \
    if (e_ != cudaSuccess)                                                           \
      return fail(PCFD_E_CUDA, "%s failed: %s (%s:%d)", #x, cudaGetErrorString(e_),  \
                  __FILE__, __LINE__);                                               \
  } while (0)

// Every kernel launch is followed by exactly one CHECK_LAUNCH, which also
// counts it (pycfd_launch_count) -- recorded launches count once, when recorded.
static std::atomic<long long> g_launches{0};
#define CHECK_LAUNCH()          \
  do {                          \
    g_launches.fetch_add(1);    \
    CU(cudaGetLastError());     \
  } while (0)
#define TRY(x)             \
  do {                     \
    int rc_ = (x);         \
    if (rc_ != 0) return rc_; \
  } while (0)

namespace {

template <class T>
struct DevEll {
  int* col = nullptr;
  T* val = nullptr;
  int n = 0, K = 0, rowmajor = 0, lanes = 1;
  int xl = 1;   // lanes per row of the per-phase kernels (1 with the column-major layout)
  Ell<T> view() const { return Ell<T>{col, val, n, K, rowmajor}; }
};

template <class T>
struct LevelBuf {
  T *b = nullptr, *xa = nullptr, *xb = nullptr, *res = nullptr;
};

struct Level {
  int n = 0, sx = 0, sy = 0;
  double weight = 1.0;
  DevEll<double> A, P, R;   // P: rows of the finer level; R = P^T: rows of this level
  DevEll<float> Af, Pf, Rf;
  DevEll<double> M;          // fused restriction R (I - A W) from the finer level (optional)
  DevEll<float> Mf;
  double* wd = nullptr;
  float* wdf = nullptr;
  LevelBuf<double> d;
  LevelBuf<float> f;
};

int choose_lanes(int K) {
  if (K <= 8) return 1;
  if (K <= 32) return 4;
  if (K <= 96) return 8;
  if (K <= 200) return 16;
  return 32;
}

// Lanes per row of the per-phase ELL kernels (row-major layouts; the column-
// major one is read by one lane per row): about four entries per lane -- one
// round of gathers -- up to eight warps per row, but no more lanes than keep
// all rows x lanes within `budget` resident threads, so a pass is one round.
// budget < 0: the storage lane count.
int exec_lanes(int K, int rowmajor, int lanes, int n, long budget) {
  if (!rowmajor) return 1;
  if (budget < 0) return lanes;
  int L = 2;
  while (L < 256 && L * 4 < K && (long)n * L * 2 <= budget) L <<= 1;
  return L;
}

}  // namespace

struct pycfd_solver {
  Geo g{};
  BcTable bc{};
  int solver_kind = 0, maxiter = 0, mg_sweeps = 1, scheme = 2, precision = 0;
  double tol = 1e-10, omega = 1.8, inner_tol = 1e-4;
  int singular = 1;
  std::vector<void*> allocs;

  uint8_t* flags = nullptr;
  uint8_t* solid = nullptr;
  int* mask_u = nullptr;
  int* mask_v = nullptr;
  int* bc_kind_dev = nullptr;
  double* profile[4] = {nullptr, nullptr, nullptr, nullptr};

  double* S = nullptr;
  int* I = nullptr;
  double* partials = nullptr;
  unsigned int* counter = nullptr;
  double* hS = nullptr;   // pinned mirrors
  int* hI = nullptr;

  // state work buffers
  double *us1 = nullptr, *vs1 = nullptr, *us2 = nullptr, *vs2 = nullptr;
  double *hu0 = nullptr, *hv0 = nullptr, *hu = nullptr, *hv = nullptr, *hp = nullptr;
  // Poisson
  double *b = nullptr, *x = nullptr, *x_api = nullptr, *r = nullptr, *pa = nullptr,
         *pb = nullptr, *q = nullptr, *z = nullptr, *xtmp = nullptr;
  bool has_guess = false;
  // mixed-form inner vectors
  float *r32 = nullptr, *x32 = nullptr, *pa32 = nullptr, *pb32 = nullptr, *q32 = nullptr,
        *z32 = nullptr;
  std::vector<Level> lv;
  double* C = nullptr;
  float* Cf = nullptr;
  int nc = 0;
  int tail_level = 0;           // level whose cycle is one dense operator (0: none)
  int fused = 0;                // down sweep by fused restrictions onto levels 1..tail_level
  long ell_budget = 0;          // resident threads a per-phase ELL pass may use (< 0: storage lanes)
  int ell_blocks = kWaveBlocks; // grid cap of the per-phase ELL kernels
  double* tail = nullptr;
  float* tailf = nullptr;
  int last_ir = 0;
  // per-kernel timing of eager launches (measurement support)
  int prof_id = 0;
  std::vector<cudaEvent_t> prof_ev;
  int prof_n = 0;
  int pdl = 1;                  // programmatic dependent launch between step kernels
  int cluster_from = 1 << 30;   // first level run inside the coarse cluster kernel
  int cluster_size = 0;         // CTAs per cluster (0: not used)
  // whole CG / MG-PCG solves as one cooperative launch
  int persistent = 0;           // CTAs of that launch (0: one kernel per phase)
  unsigned long long wait_ns = kPWaitLimitNs;   // limit of one grid-barrier wait of that launch
  unsigned* pbar = nullptr;     // barrier words, zeroed before every launch
  double* ppart = nullptr;      // per-CTA partial sums
  unsigned long long* ptrace = nullptr;   // phase trace (measurement support)
  int trace_on = 0;
  double* hist = nullptr;       // device history of a device-side run loop (kHistRows x kHistCols)
  int les = 0;                  // Smagorinsky closure on
  double les_coeff = 0.0;       // (Cs Delta)^2
  double* met = nullptr;        // stretched mesh: the packed metrics (Geo::met)
  double* les_coeff_c = nullptr;  // stretched mesh with LES: (Cs Delta)^2 per ghosted cell
  double* les_nu_c = nullptr;   // (nx+2) x (ny+2) effective viscosity of the current stage
  double* les_nu_k = nullptr;   // (nx+1) x (ny+1) its corner average
  // CUDA-graph recording of whole steps
  bool capturing = false;
  cudaStream_t aux = nullptr;   // records the bodies of the solve loops
  cudaStream_t aux2 = nullptr;  // records loop bodies nested one level deeper
  cudaStream_t gate = nullptr;  // records the gated body of a device-loop step
  cudaStream_t rec = nullptr;   // records whole steps
  struct GraphEntry {
    const void* key[5];
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    int adaptive;
    DtControl ctl;
  };
  std::vector<GraphEntry> graphs;

  dim3 cgrid, cblock;   // 2D launch over the fine cells
  RedBuf rb() const { return RedBuf{partials, counter}; }
  SolveCfg cfg() const { return SolveCfg{tol, maxiter, singular, 0}; }
  long ncell() const { return (long)g.nx * g.ny; }
};

namespace {

template <class T>
int dalloc(pycfd_solver* s, T** p, size_t count) {
  void* ptr = nullptr;
  CU(cudaMalloc(&ptr, std::max<size_t>(count, 1) * sizeof(T)));
  CU(cudaMemset(ptr, 0, std::max<size_t>(count, 1) * sizeof(T)));
  s->allocs.push_back(ptr);
  *p = (T*)ptr;
  return 0;
}

template <class T>
int upload(pycfd_solver* s, T** p, const T* host, size_t count) {
  TRY(dalloc(s, p, count));
  if (count) CU(cudaMemcpy(*p, host, count * sizeof(T), cudaMemcpyHostToDevice));
  return 0;
}

// CSR -> ELL (entries of a row sorted by column) in the layout its lane count wants.
template <class T>
int make_ell(pycfd_solver* s, DevEll<T>* E, int n, const int64_t* indptr, const int32_t* idx,
             const double* data) {
  int K = 0;
  for (int r = 0; r < n; ++r) K = std::max<int>(K, (int)(indptr[r + 1] - indptr[r]));
  K = std::max(K, 1);
  const int L = choose_lanes(K);
  const int rowmajor = L > 1;
  const int Kp = rowmajor ? ((K + L - 1) / L) * L : K;
  std::vector<int> col((size_t)n * Kp);
  std::vector<T> val((size_t)n * Kp, (T)0);
  std::vector<std::pair<int, double>> row;
  for (int r = 0; r < n; ++r) {
    row.clear();
    for (int64_t e = indptr[r]; e < indptr[r + 1]; ++e) row.push_back({idx[e], data[e]});
    std::sort(row.begin(), row.end(),
              [](const std::pair<int, double>& a, const std::pair<int, double>& b) { return a.first < b.first; });
    const int pad_col = row.empty() ? 0 : row[0].first;
    for (int k = 0; k < Kp; ++k) {
      const size_t at = rowmajor ? (size_t)r * Kp + k : (size_t)k * n + r;
      if (k < (int)row.size()) {
        col[at] = row[k].first;
        val[at] = (T)row[k].second;
      } else {
        col[at] = pad_col;
        val[at] = (T)0;
      }
    }
  }
  TRY(upload(s, &E->col, col.data(), col.size()));
  TRY(upload(s, &E->val, val.data(), val.size()));
  E->n = n;
  E->K = Kp;
  E->rowmajor = rowmajor;
  E->lanes = L;
  E->xl = exec_lanes(Kp, rowmajor, L, n, s->ell_budget);
  return 0;
}

// CSR transpose (rows = columns of the input).
void csr_transpose(int nrows, int ncols, const int64_t* indptr, const int32_t* idx,
                   const double* data, std::vector<int64_t>& tp, std::vector<int32_t>& ti,
                   std::vector<double>& td) {
  tp.assign(ncols + 1, 0);
  const int64_t nnz = indptr[nrows];
  for (int64_t e = 0; e < nnz; ++e) tp[idx[e] + 1]++;
  for (int c = 0; c < ncols; ++c) tp[c + 1] += tp[c];
  ti.resize(nnz);
  td.resize(nnz);
  std::vector<int64_t> pos(tp.begin(), tp.end() - 1);
  for (int r = 0; r < nrows; ++r)
    for (int64_t e = indptr[r]; e < indptr[r + 1]; ++e) {
      const int64_t at = pos[idx[e]]++;
      ti[at] = r;
      td[at] = data[e];
    }
}

cudaStream_t st(void* stream) { return (cudaStream_t)stream; }

// Bracket one launch of the profiled kernel with a pair of events on its
// stream (eager launches only: recorded graphs carry no events).
constexpr int kProfPairs = 4096;
inline void prof_mark(pycfd_solver* s, int id, cudaStream_t stream) {
  if (s->prof_id != id || s->capturing || s->prof_n >= 2 * kProfPairs) return;
  if (s->prof_ev.empty()) {
    s->prof_ev.resize(2 * kProfPairs);
    for (auto& e : s->prof_ev) cudaEventCreate(&e);
  }
  cudaEventRecord(s->prof_ev[s->prof_n++], stream);
}

// ---- launch helpers ---------------------------------------------------------
// Launch a kernel of the step with the programmatic-serialization attribute
// (see pdl_begin): the launch of a dependent kernel overlaps its predecessor.
// Launch errors surface through the CHECK_LAUNCH that follows every launch.
template <class... P, class... A>
inline void pdl_launch(pycfd_solver* s, void (*kernel)(P...), dim3 grid, dim3 block, size_t smem,
                       cudaStream_t stream, A&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = s->pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}
int launch_boundary(pycfd_solver* s, double* u, double* v, std::initializer_list<int> ops,
                    cudaStream_t stream) {
  BcProgram prog{};
  int k = 0;
  for (int op : ops) prog.op[k++] = op;
  prog.op[k] = OP_END;
  pdl_launch(s, k_boundary, 1, 1024, 0, stream, u, v, s->g, s->bc, prog, s->S);
  CHECK_LAUNCH();
  return 0;
}

int grid1(pycfd_solver* s) { return grid_for(s->ncell(), kRedThreads, kMaxRedBlocks); }

// Generic dispatcher over the lane count of an ELL block.
#define ELL_DISPATCH(LANES, CALL)                   \
  switch (LANES) {                                  \
    case 1: { constexpr int L = 1; CALL; } break;    \
    case 2: { constexpr int L = 2; CALL; } break;    \
    case 4: { constexpr int L = 4; CALL; } break;    \
    case 8: { constexpr int L = 8; CALL; } break;    \
    case 16: { constexpr int L = 16; CALL; } break;  \
    case 32: { constexpr int L = 32; CALL; } break;  \
    case 64: { constexpr int L = 64; CALL; } break;  \
    case 128: { constexpr int L = 128; CALL; } break; \
    default: { constexpr int L = 256; CALL; } break;  \
  }

inline int ell_grid(const pycfd_solver* s, int n, int L) {
  return (int)std::min<long>(((long)n * L + 255) / 256, s->ell_blocks);
}

template <class T>
const DevEll<T>& lvA(const Level& l);
template <>
const DevEll<double>& lvA<double>(const Level& l) { return l.A; }
template <>
const DevEll<float>& lvA<float>(const Level& l) { return l.Af; }
template <class T>
const DevEll<T>& lvP(const Level& l);
template <>
const DevEll<double>& lvP<double>(const Level& l) { return l.P; }
template <>
const DevEll<float>& lvP<float>(const Level& l) { return l.Pf; }
template <class T>
const DevEll<T>& lvR(const Level& l);
template <>
const DevEll<double>& lvR<double>(const Level& l) { return l.R; }
template <>
const DevEll<float>& lvR<float>(const Level& l) { return l.Rf; }
template <class T>
LevelBuf<T>& lvB(Level& l);
template <>
LevelBuf<double>& lvB<double>(Level& l) { return l.d; }
template <>
LevelBuf<float>& lvB<float>(Level& l) { return l.f; }
template <class T>
T* lvWd(Level& l);
template <>
double* lvWd<double>(Level& l) { return l.wd; }
template <>
float* lvWd<float>(Level& l) { return l.wdf; }
template <class T>
const DevEll<T>& lvM(const Level& l);
template <>
const DevEll<double>& lvM<double>(const Level& l) { return l.M; }
template <>
const DevEll<float>& lvM<float>(const Level& l) { return l.Mf; }
template <class T>
const T* tailM(pycfd_solver* s);
template <>
const double* tailM<double>(pycfd_solver* s) { return s->tail; }
template <>
const float* tailM<float>(pycfd_solver* s) { return s->tailf; }
template <class T>
const T* coarseC(pycfd_solver* s);
template <>
const double* coarseC<double>(pycfd_solver* s) { return s->C; }
template <>
const float* coarseC<float>(pycfd_solver* s) { return s->Cf; }

// Launch the cluster kernel over levels [lc, Lv) of the hierarchy; returns in
// *out the buffer that holds x_lc afterwards (the kernel's ping-pong, replayed).
template <class T>
int launch_coarse_cluster(pycfd_solver* s, int lc, const T* res_in, T** out, cudaStream_t stream) {
  const int Lv = (int)s->lv.size();
  CTable<T> t{};
  t.nlev = Lv - lc;
  t.res_in = res_in;
  t.C = coarseC<T>(s);
  t.nc = s->nc;
  t.sweeps = s->mg_sweeps;
  for (int k = 0; k < t.nlev; ++k) {
    Level& L = s->lv[lc + k];
    CLevel<T>& c = t.lv[k];
    if (lc + k < Lv - 1) {
      c.A = lvA<T>(L).view();
      c.la = lvA<T>(L).lanes;
    }
    c.R = lvR<T>(L).view();
    c.lr = lvR<T>(L).lanes;
    c.P = lvP<T>(L).view();
    c.lp = lvP<T>(L).lanes;
    c.wd = lvWd<T>(L);
    LevelBuf<T>& B = lvB<T>(L);
    c.b = B.b;
    c.xa = B.xa;
    c.xb = B.xb;
    c.res = B.res;
  }
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(s->cluster_size);
  cfg.blockDim = dim3(1024);
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = s->cluster_size;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  prof_mark(s, 4, stream);
  CU(cudaLaunchKernelEx(&cfg, k_coarse_cycle<T>, t));
  g_launches.fetch_add(1);
  prof_mark(s, 4, stream);
  // where x_lc ends: the first sweep writes xa; each further sweep swaps
  LevelBuf<T>& B = lvB<T>(s->lv[lc]);
  T* xf = B.xa;
  if (lc < Lv - 1) {
    if (s->mg_sweeps > 1 && ((s->mg_sweeps - 1) & 1)) xf = B.xb;
    if (s->mg_sweeps & 1) xf = (xf == B.xa) ? B.xb : B.xa;
  }
  *out = xf;
  return 0;
}

// One V-cycle from zero applied to the CG residual r: z_out gets the
// unprojected result; the last fine sweep's finisher leaves mean(z) and r.z
// in the scalar slots (pycfd/core/multigrid.py:430-474).
template <class T>
int vcycle_pcg(pycfd_solver* s, const T* r, T* z_out, cudaStream_t stream) {
  const int Lv = (int)s->lv.size();
  const Geo& g = s->g;
  const int sw = s->mg_sweeps;
  const int G = grid1(s);
  // Materialise the projected fine right-hand side b0 = r - mean(r) (solvable
  // rows; the mean was left in S_MEAN_R by the kernel that produced r) into
  // level 0's b buffer; the fine kernels read it as a stored vector.
  LevelBuf<T>& B0 = lvB<T>(s->lv[0]);
  BFromRS<T> bf0{r, s->flags, s->S, s->singular, 0.0};
  if (Lv == 1) {
    pdl_launch(s, k_fine_store_from_r<T>, s->cgrid, s->cblock, 0, stream, r, s->flags, g, s->S, s->singular, B0.b);
    CHECK_LAUNCH();
    pdl_launch(s, k_dense<T>, 1, 256, 0, stream, coarseC<T>(s), s->nc, B0.b, z_out);
    CHECK_LAUNCH();
    pdl_launch(s, k_fine_sums<T, 1>, s->cgrid, s->cblock, 0, stream, z_out, s->flags, g, r, s->singular, s->S, s->rb());
    CHECK_LAUNCH();
    return 0;
  }
  const double w0 = s->lv[0].weight;
  if (s->fused && sw == 1 && s->tail_level > 0 && s->tail_level < std::min(s->cluster_from, Lv)) {
    // ---- down: b_l = M_l b_{l-1} (first sweep + restriction in one pass), then the tail
    const int tl = s->tail_level;
    {
      const DevEll<T>& M = lvM<T>(s->lv[1]);
      ELL_DISPATCH(M.xl, (pdl_launch(s, k_ell_fused_restrict0<L, T, BFromRS<T>>, ell_grid(s, M.n, L), 256, 0, stream,
                                        M.view(), bf0, lvB<T>(s->lv[1]).b)));
      CHECK_LAUNCH();
    }
    for (int l = 2; l <= tl; ++l) {
      const DevEll<T>& M = lvM<T>(s->lv[l]);
      ELL_DISPATCH(M.xl, (pdl_launch(s, k_ell_spmv<L, false, T>, ell_grid(s, M.n, L), 256, 0, stream, M.view(),
                                        (const T*)lvB<T>(s->lv[l - 1]).b, lvB<T>(s->lv[l]).b)));
      CHECK_LAUNCH();
    }
    LevelBuf<T>& Bt = lvB<T>(s->lv[tl]);
    pdl_launch(s, k_tail<T>, (s->lv[tl].n + kTailRowsPerBlock - 1) / kTailRowsPerBlock, 256, 0, stream, tailM<T>(s),
               s->lv[tl].n, (const T*)Bt.b, Bt.xa);
    CHECK_LAUNCH();
    // ---- up: x_l = (T)(W b_l) + P x_{l+1}, one sweep
    const T* xc = Bt.xa;
    for (int l = tl - 1; l >= 1; --l) {
      Level& Lf = s->lv[l];
      LevelBuf<T>& Bf = lvB<T>(Lf);
      const DevEll<T>& P = lvP<T>(s->lv[l + 1]);
      ELL_DISPATCH(P.xl, (pdl_launch(s, k_ell_prolong_wb<L, T>, ell_grid(s, P.n, L), 256, 0, stream, P.view(),
                                        (const T*)lvWd<T>(Lf), (const T*)Bf.b, xc, Bf.xa)));
      CHECK_LAUNCH();
      const DevEll<T>& A = lvA<T>(Lf);
      ELL_DISPATCH(A.xl, (pdl_launch(s, k_ell_smooth<L, T>, ell_grid(s, A.n, L), 256, 0, stream, A.view(),
                                        (const T*)lvWd<T>(Lf), (const T*)Bf.b, (const T*)Bf.xa, Bf.xb)));
      CHECK_LAUNCH();
      xc = Bf.xb;
    }
    const DevEll<T>& P1 = lvP<T>(s->lv[1]);
    ELL_DISPATCH(P1.xl, (pdl_launch(s, k_ell_prolong0_wb<L, T, BFromRS<T>>, ell_grid(s, P1.n, L), 256, 0, stream,
                                       P1.view(), bf0, s->flags, g, w0, xc, B0.xa)));
    CHECK_LAUNCH();
    prof_mark(s, 2, stream);
    pdl_launch(s, k_fine_smooth<T, BFromRS<T>, 1>, dim3(strip_grid(s->g)), dim3(kStripThreads), 0, stream, bf0, s->flags, g, w0,
               (const T*)B0.xa, z_out, r, s->singular, s->S, s->rb());
    prof_mark(s, 2, stream);
    CHECK_LAUNCH();
    return 0;
  }
  // ---- down ----
  T* cur[32];
  if (sw == 1) {
    prof_mark(s, 3, stream);
    pdl_launch(s, k_fine_pre<T, BFromRS<T>>, dim3(strip_grid(s->g)), dim3(kStripThreads), 0, stream, bf0, s->flags, g, w0, B0.xa, B0.res);
    prof_mark(s, 3, stream);
    CHECK_LAUNCH();
    cur[0] = B0.xa;
  } else {
    pdl_launch(s, k_fine_wdb<T, BFromRS<T>>, s->cgrid, s->cblock, 0, stream, bf0, s->flags, g, w0, B0.xa);
    CHECK_LAUNCH();
    T* a = B0.xa;
    T* bb = B0.xb;
    for (int k = 1; k < sw; ++k) {
      pdl_launch(s, k_fine_smooth<T, BFromRS<T>, 0>, dim3(strip_grid(s->g)), dim3(kStripThreads), 0, stream, bf0, s->flags, g, w0, a, bb, r,
                                                                      s->singular, s->S, s->rb());
      CHECK_LAUNCH();
      std::swap(a, bb);
    }
    pdl_launch(s, k_fine_resid<T, BFromRS<T>>, dim3(strip_grid(s->g)), dim3(kStripThreads), 0, stream, bf0, s->flags, g, a, B0.res);
    CHECK_LAUNCH();
    cur[0] = a;
  }
  const int lc = std::max(1, std::min(s->cluster_from, Lv));
  int bottom = Lv - 1;   // level where the down sweep ends
  for (int l = 1; l < Lv; ++l) {
    if (l >= lc) {   // the rest of the cycle below l runs in one cluster
      TRY(launch_coarse_cluster<T>(s, l, lvB<T>(s->lv[l - 1]).res, &cur[l], stream));
      bottom = l;
      break;
    }
    Level& Lc = s->lv[l];
    LevelBuf<T>& Bc = lvB<T>(Lc);
    const T* res_f = lvB<T>(s->lv[l - 1]).res;
    const DevEll<T>& R = lvR<T>(Lc);
    if (l == Lv - 1) {   // coarsest: restriction and dense solve in one block
      pdl_launch(s, k_restrict_dense<T>, 1, 1024, R.n * sizeof(double), stream, R.view(), R.lanes, res_f, coarseC<T>(s),
                                                                    Bc.b, Bc.xa);
      CHECK_LAUNCH();
      cur[l] = Bc.xa;
      break;
    }
    ELL_DISPATCH(R.xl, (pdl_launch(s, k_ell_spmv<L, false, T>, ell_grid(s, R.n, L), 256, 0, stream, R.view(), res_f, Bc.b)));
    CHECK_LAUNCH();
    if (l == s->tail_level) {   // the cycle at and below l as one dense operator
      pdl_launch(s, k_tail<T>, (Lc.n + kTailRowsPerBlock - 1) / kTailRowsPerBlock, 256, 0, stream, tailM<T>(s), Lc.n,
                 (const T*)Bc.b, Bc.xa);
      CHECK_LAUNCH();
      cur[l] = Bc.xa;
      bottom = l;
      break;
    }
    const DevEll<T>& A = lvA<T>(Lc);
    T* wd = lvWd<T>(Lc);
    ELL_DISPATCH(A.xl, (pdl_launch(s, k_ell_pre<L, T>, ell_grid(s, A.n, L), 256, 0, stream, A.view(), wd, Bc.b, Bc.xa, Bc.res)));
    CHECK_LAUNCH();
    T* a = Bc.xa;
    T* bb = Bc.xb;
    if (sw > 1) {
      for (int k = 1; k < sw; ++k) {
        ELL_DISPATCH(A.xl, (pdl_launch(s, k_ell_smooth<L, T>, ell_grid(s, A.n, L), 256, 0, stream, A.view(), wd, Bc.b, a, bb)));
        CHECK_LAUNCH();
        std::swap(a, bb);
      }
      ELL_DISPATCH(A.xl, (pdl_launch(s, k_ell_resid<L, T>, ell_grid(s, A.n, L), 256, 0, stream, A.view(), Bc.b, a, Bc.res)));
      CHECK_LAUNCH();
    }
    cur[l] = a;
  }
  // ---- up ----
  for (int l = bottom - 1; l >= 0; --l) {
    Level& Lf = s->lv[l];
    LevelBuf<T>& Bf = lvB<T>(Lf);
    const DevEll<T>& P = lvP<T>(s->lv[l + 1]);
    T* xf = cur[l];
    ELL_DISPATCH(P.xl, (pdl_launch(s, k_ell_spmv<L, true, T>, ell_grid(s, P.n, L), 256, 0, stream, P.view(), cur[l + 1], xf)));
    CHECK_LAUNCH();
    T* other = (xf == Bf.xa) ? Bf.xb : Bf.xa;
    for (int k = 1; k <= sw; ++k) {
      if (l == 0) {
        T* dst = (k == sw) ? z_out : other;
        if (k == sw)
          {
            prof_mark(s, 2, stream);
            pdl_launch(s, k_fine_smooth<T, BFromRS<T>, 1>, dim3(strip_grid(s->g)), dim3(kStripThreads), 0, stream, bf0, s->flags, g, w0, xf, dst, r,
                                                                          s->singular, s->S, s->rb());
            prof_mark(s, 2, stream);
          }
        else
          pdl_launch(s, k_fine_smooth<T, BFromRS<T>, 0>, dim3(strip_grid(s->g)), dim3(kStripThreads), 0, stream, bf0, s->flags, g, w0, xf, dst, r,
                                                                          s->singular, s->S, s->rb());
        CHECK_LAUNCH();
        other = xf;
        xf = dst;
      } else {
        const DevEll<T>& A = lvA<T>(Lf);
        T* wd = lvWd<T>(Lf);
        ELL_DISPATCH(A.xl, (pdl_launch(s, k_ell_smooth<L, T>, ell_grid(s, A.n, L), 256, 0, stream, A.view(), wd, Bf.b, xf, other)));
        CHECK_LAUNCH();
        std::swap(xf, other);
      }
    }
    cur[l] = xf;
  }
  return 0;
}

// One standalone V-cycle from the current fine iterate x with right-hand side
// b (both double).  Leaves the fine mean of the result in S_MEAN_X.
int vcycle_standalone(pycfd_solver* s, double* b, double* x, cudaStream_t stream) {
  const int Lv = (int)s->lv.size();
  const Geo& g = s->g;
  const int sw = s->mg_sweeps;
  const int G = grid1(s);
  BStored<double> bf{b};
  LevelBuf<double>& B0 = s->lv[0].d;
  if (Lv == 1) {
    pdl_launch(s, k_dense<double>, 1, 256, 0, stream, s->C, s->nc, b, x);
    CHECK_LAUNCH();
    pdl_launch(s, k_fine_sums<double, 2>, s->cgrid, s->cblock, 0, stream, x, s->flags, g, nullptr, s->singular, s->S, s->rb());
    CHECK_LAUNCH();
    return 0;
  }
  const double w0 = s->lv[0].weight;
  double* a = x;
  double* t = s->xtmp;
  for (int k = 0; k < sw; ++k) {
    pdl_launch(s, k_fine_smooth<double, BStored<double>, 0>, dim3(strip_grid(s->g)), dim3(kStripThreads), 0, stream, bf, s->flags, g, w0, a, t, nullptr,
                                                                             s->singular, s->S, s->rb());
    CHECK_LAUNCH();
    std::swap(a, t);
  }
  pdl_launch(s, k_fine_resid<double, BStored<double>>, dim3(strip_grid(s->g)), dim3(kStripThreads), 0, stream, bf, s->flags, g, a, B0.res);
  CHECK_LAUNCH();
  double* cur[32];
  cur[0] = a;
  for (int l = 1; l < Lv; ++l) {
    Level& Lc = s->lv[l];
    const double* res_f = s->lv[l - 1].d.res;
    ELL_DISPATCH(Lc.R.xl, (pdl_launch(s, k_ell_spmv<L, false, double>, ell_grid(s, Lc.R.n, L), 256, 0, stream, Lc.R.view(), res_f, Lc.d.b)));
    CHECK_LAUNCH();
    if (l == Lv - 1) {
      pdl_launch(s, k_dense<double>, 1, 256, 0, stream, s->C, s->nc, Lc.d.b, Lc.d.xa);
      CHECK_LAUNCH();
      cur[l] = Lc.d.xa;
      break;
    }
    ELL_DISPATCH(Lc.A.xl, (pdl_launch(s, k_ell_pre<L, double>, ell_grid(s, Lc.A.n, L), 256, 0, stream, Lc.A.view(), Lc.wd, Lc.d.b, Lc.d.xa, Lc.d.res)));
    CHECK_LAUNCH();
    double* p = Lc.d.xa;
    double* o = Lc.d.xb;
    if (sw > 1) {
      for (int k = 1; k < sw; ++k) {
        ELL_DISPATCH(Lc.A.xl, (pdl_launch(s, k_ell_smooth<L, double>, ell_grid(s, Lc.A.n, L), 256, 0, stream, Lc.A.view(), Lc.wd, Lc.d.b, p, o)));
        CHECK_LAUNCH();
        std::swap(p, o);
      }
      ELL_DISPATCH(Lc.A.xl, (pdl_launch(s, k_ell_resid<L, double>, ell_grid(s, Lc.A.n, L), 256, 0, stream, Lc.A.view(), Lc.d.b, p, Lc.d.res)));
      CHECK_LAUNCH();
    }
    cur[l] = p;
  }
  for (int l = Lv - 2; l >= 0; --l) {
    Level& Lf = s->lv[l];
    const DevEll<double>& P = s->lv[l + 1].P;
    double* xf = cur[l];
    ELL_DISPATCH(P.xl, (pdl_launch(s, k_ell_spmv<L, true, double>, ell_grid(s, P.n, L), 256, 0, stream, P.view(), cur[l + 1], xf)));
    CHECK_LAUNCH();
    if (l == 0) {
      double* o = (xf == x) ? s->xtmp : x;
      for (int k = 1; k <= sw; ++k) {
        if (k == sw)
          pdl_launch(s, k_fine_smooth<double, BStored<double>, 2>, dim3(strip_grid(s->g)), dim3(kStripThreads), 0, stream, bf, s->flags, g, w0, xf, o, nullptr,
                                                                                   s->singular, s->S, s->rb());
        else
          pdl_launch(s, k_fine_smooth<double, BStored<double>, 0>, dim3(strip_grid(s->g)), dim3(kStripThreads), 0, stream, bf, s->flags, g, w0, xf, o, nullptr,
                                                                                   s->singular, s->S, s->rb());
        CHECK_LAUNCH();
        std::swap(xf, o);
      }
      if (xf != x) CU(cudaMemcpyAsync(x, xf, s->ncell() * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    } else {
      double* o = (xf == Lf.d.xa) ? Lf.d.xb : Lf.d.xa;
      for (int k = 1; k <= sw; ++k) {
        ELL_DISPATCH(Lf.A.xl, (pdl_launch(s, k_ell_smooth<L, double>, ell_grid(s, Lf.A.n, L), 256, 0, stream, Lf.A.view(), Lf.wd, Lf.d.b, xf, o)));
        CHECK_LAUNCH();
        std::swap(xf, o);
      }
      cur[l] = xf;
    }
  }
  return 0;
}

int read_flags(pycfd_solver* s, cudaStream_t stream) {
  CU(cudaMemcpyAsync(s->hI, s->I, sizeof(int) * I_COUNT, cudaMemcpyDeviceToHost, stream));
  CU(cudaStreamSynchronize(stream));
  return 0;
}

// ---- iteration loops -------------------------------------------------------
// A solve's iteration loop runs either on the host (read the done flag after
// every pass) or, while a step is being recorded into a CUDA graph, as a
// conditional WHILE node whose body is recorded on the auxiliary stream and
// whose condition the converging kernel sets on the device.
struct Loop {
  LoopCtl ctl{0, 0};
  cudaGraph_t body = nullptr;
};

int loop_handle(pycfd_solver* s, cudaStream_t stream, Loop* L) {
  if (!s->capturing) return 0;
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  CU(cudaStreamGetCaptureInfo(stream, &cs, nullptr, &g, nullptr, nullptr));
  cudaGraphConditionalHandle h;
  CU(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
  L->ctl = LoopCtl{h, 1};
  return 0;
}

// Append the WHILE node after everything captured so far; begin recording its body on aux.
int loop_open(pycfd_solver* s, cudaStream_t stream, Loop* L) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  CU(cudaStreamGetCaptureInfo(stream, &cs, nullptr, &g, &deps, &nd));
  cudaGraphNodeParams np{};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = L->ctl.handle;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  CU(cudaGraphAddNode(&node, g, deps, nd, &np));
  L->body = np.conditional.phGraph_out[0];
  CU(cudaStreamUpdateCaptureDependencies(stream, &node, 1, cudaStreamSetCaptureDependencies));
  CU(cudaStreamBeginCaptureToGraph(s->aux, L->body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  return 0;
}

int loop_close(pycfd_solver* s) {
  cudaGraph_t out = nullptr;
  CU(cudaStreamEndCapture(s->aux, &out));
  return 0;
}

// ---- mixed form: FP64 iterative refinement around an FP32 MG-PCG ----------
// Outer passes r = b - A x (FP64) until ||r|| < tol ||b||; each pass solves
// A e = r in FP32 storage with the FP32 copy of the hierarchy to a relative
// inner_tol and adds e to x.  Recorded, the outer loop and the inner CG loop
// are nested WHILE nodes.
constexpr int kIrMaxPasses = 40;
constexpr int kInnerMaxIter = 200;

int solve_mixed(pycfd_solver* s, double* x, bool has_x0, cudaStream_t stream) {
  const Geo& g = s->g;
  const SolveCfg cfg = s->cfg();
  const SolveCfg icfg{s->inner_tol, kInnerMaxIter, s->singular, 0};
  const bool cap = s->capturing;
  Loop outer, inner;
  TRY(loop_handle(s, stream, &outer));
  pdl_launch(s, k_ir_residual, s->cgrid, s->cblock, 0, stream, s->b, x, s->r32, s->x32, s->flags, g, cfg,
                                                    s->inner_tol, kIrMaxPasses, 1, has_x0, s->S, s->I,
                                                    s->rb(), outer.ctl);
  CHECK_LAUNCH();
  auto inner_pass = [&](cudaStream_t st) -> int {
    TRY(vcycle_pcg<float>(s, s->r32, s->z32, st));
    pdl_launch(s, k_cg_pq<float, PC_MG>, dim3(strip_grid(s->g)), dim3(kStripThreads), 0, st, s->r32, s->z32, s->pa32, s->pb32, s->q32, s->flags,
                                                          g, s->S, s->I, s->rb());
    CHECK_LAUNCH();
    pdl_launch(s, k_cg_xr<float, PC_MG>, dim3(strip_grid(s->g)), dim3(kStripThreads), 0, st, s->x32, s->r32, s->pb32, s->q32, s->pa32, s->flags,
                                                          g, icfg, s->S, s->I, s->rb(), inner.ctl);
    CHECK_LAUNCH();
    return 0;
  };
  auto refine = [&](cudaStream_t st) -> int {
    pdl_launch(s, k_ir_update, s->cgrid, s->cblock, 0, st, x, s->x32, s->flags, g, s->I);
    CHECK_LAUNCH();
    pdl_launch(s, k_ir_residual, s->cgrid, s->cblock, 0, st, s->b, x, s->r32, s->x32, s->flags, g, cfg, s->inner_tol,
                                                  kIrMaxPasses, 0, 1, s->S, s->I, s->rb(), outer.ctl);
    CHECK_LAUNCH();
    return 0;
  };
  if (cap) {
    TRY(loop_open(s, stream, &outer));          // outer body recorded on aux
    // inner loop inside the outer body: handle on the body graph, body on aux2
    {
      cudaGraphConditionalHandle h;
      CU(cudaGraphConditionalHandleCreate(&h, outer.body, 0, 0));
      inner.ctl = LoopCtl{h, 1};
      pdl_launch(s, k_ir_arm, 1, 32, 0, s->aux, s->I, inner.ctl);
      CHECK_LAUNCH();
      cudaStreamCaptureStatus cs;
      cudaGraph_t gb = nullptr;
      const cudaGraphNode_t* deps = nullptr;
      size_t nd = 0;
      CU(cudaStreamGetCaptureInfo(s->aux, &cs, nullptr, &gb, &deps, &nd));
      cudaGraphNodeParams np{};
      np.type = cudaGraphNodeTypeConditional;
      np.conditional.handle = h;
      np.conditional.type = cudaGraphCondTypeWhile;
      np.conditional.size = 1;
      cudaGraphNode_t node;
      CU(cudaGraphAddNode(&node, gb, deps, nd, &np));
      CU(cudaStreamUpdateCaptureDependencies(s->aux, &node, 1, cudaStreamSetCaptureDependencies));
      if (!s->aux2) CU(cudaStreamCreateWithFlags(&s->aux2, cudaStreamNonBlocking));
      CU(cudaStreamBeginCaptureToGraph(s->aux2, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                       cudaStreamCaptureModeRelaxed));
      TRY(inner_pass(s->aux2));
      cudaGraph_t dummy = nullptr;
      CU(cudaStreamEndCapture(s->aux2, &dummy));
    }
    TRY(refine(s->aux));
    TRY(loop_close(s));
  } else {
    for (;;) {
      TRY(read_flags(s, stream));
      if (s->hI[I_IR_DONE]) break;
      for (;;) {
        TRY(read_flags(s, stream));
        if (s->hI[I_DONE]) break;
        TRY(inner_pass(stream));
      }
      TRY(refine(stream));
    }
  }
  pdl_launch(s, k_finish_stats<double>, s->cgrid, s->cblock, 0, stream, x, s->b, s->flags, g, cfg, 1, s->S, s->I, s->rb());
  CHECK_LAUNCH();
  pdl_launch(s, k_finish_apply<double>, s->cgrid, s->cblock, 0, stream, x, x, s->flags, g, s->S, s->I);
  CHECK_LAUNCH();
  return 0;
}

// ---- CG / MG-PCG as one cooperative launch ---------------------------------
// The kernel conditions b, runs the passes, leaves ||b - A x|| and the mean of
// x in the scalar slots and removes the mean (k_rhs_init ... k_finish_apply);
// the barrier
// words start at zero for every launch, so a wait that gave up in an earlier
// launch leaves no trace.
int solve_persistent(pycfd_solver* s, double* x, bool has_x0, cudaStream_t stream) {
  PSolve<double> t{};
  const int Lv = (int)s->lv.size();
  const bool mg = s->solver_kind == PCFD_SOLVER_MGCG;
  if (mg) {
    t.nlev = Lv;
    for (int l = 0; l < Lv; ++l) {
      Level& L = s->lv[l];
      PLevel<double>& c = t.lv[l];
      if (l >= 1) {
        if (l < Lv - 1) {
          c.A = L.A.view();
          c.la = L.A.lanes;
        }
        c.R = L.R.view();
        c.lr = L.R.lanes;
        c.P = L.P.view();
        c.lp = L.P.lanes;
        c.wd = L.wd;
      }
      c.b = L.d.b;
      c.xa = L.d.xa;
      c.xb = L.d.xb;
      c.res = L.d.res;
    }
    t.C = s->C;
    t.nc = s->nc;
    t.tail = s->tail;
    t.tail_level = s->tail_level;
    t.w0 = s->lv[0].weight;
  }
  t.flags = s->flags;
  t.g = s->g;
  t.sweeps = s->mg_sweeps;
  t.cfg = s->cfg();
  t.has_x0 = has_x0 ? 1 : 0;
  t.b = s->b;
  t.x = x;
  t.r = s->r;
  t.z = s->z;
  t.pa = s->pa;
  t.pb = s->pb;
  t.q = s->q;
  t.S = s->S;
  t.I = s->I;
  t.partials = s->ppart;
  t.bar = s->pbar;
  t.trace = s->trace_on ? s->ptrace : nullptr;
  t.wait_ns = s->wait_ns;
  CU(cudaMemsetAsync(s->pbar, 0, 64 * sizeof(unsigned), stream));
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(s->persistent);
  cfg.blockDim = dim3(kPThreads);
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  prof_mark(s, 8, stream);
  if (mg) CU(cudaLaunchKernelEx(&cfg, k_solve_persistent<double, PC_MG>, t));
  else CU(cudaLaunchKernelEx(&cfg, k_solve_persistent<double, PC_JACOBI>, t));
  prof_mark(s, 8, stream);
  CHECK_LAUNCH();
  return 0;
}

// ---- Poisson solve on the prepared raw right-hand side s->b --------------
// Result (normalised) in x.  has_x0: x holds the warm start on entry.
int solve_prepared(pycfd_solver* s, double* x, bool has_x0, cudaStream_t stream) {
  const Geo& g = s->g;
  const int G = grid1(s);
  const SolveCfg cfg = s->cfg();
  const int kind = s->solver_kind;
  const bool cap = s->capturing;
  if (s->persistent && (kind == PCFD_SOLVER_CG || kind == PCFD_SOLVER_MGCG)) {
    return solve_persistent(s, x, has_x0, stream);   // mean removal included
  }
  if (kind == PCFD_SOLVER_CG || kind == PCFD_SOLVER_MGCG) {
    Loop L;
    TRY(loop_handle(s, stream, &L));
    pdl_launch(s, k_rhs_init<double>, s->cgrid, s->cblock, 0, stream, s->b, x, s->r, s->flags, g, cfg, has_x0, s->S,
                                                      s->I, s->rb(), L.ctl);
    CHECK_LAUNCH();
    // one pass of the recurrence on stream `st`; p_old -> p_new
    auto pass = [&](cudaStream_t st, double* p_old, double* p_new, double* keep) -> int {
      if (kind == PCFD_SOLVER_CG) {
        pdl_launch(s, k_cg_pq<double, PC_JACOBI>, dim3(strip_grid(s->g)), dim3(kStripThreads), 0, st, s->r, nullptr, p_old, p_new, s->q, s->flags,
                                                              g, s->S, s->I, s->rb());
        CHECK_LAUNCH();
        pdl_launch(s, k_cg_xr<double, PC_JACOBI>, dim3(strip_grid(s->g)), dim3(kStripThreads), 0, st, x, s->r, p_new, s->q, keep, s->flags, g, cfg,
                                                              s->S, s->I, s->rb(), L.ctl);
      } else {
        TRY(vcycle_pcg<double>(s, s->r, s->z, st));
        prof_mark(s, 1, st);
        pdl_launch(s, k_cg_pq<double, PC_MG>, dim3(strip_grid(s->g)), dim3(kStripThreads), 0, st, s->r, s->z, p_old, p_new, s->q, s->flags, g,
                                                          s->S, s->I, s->rb());
        prof_mark(s, 1, st);
        CHECK_LAUNCH();
        pdl_launch(s, k_cg_xr<double, PC_MG>, dim3(strip_grid(s->g)), dim3(kStripThreads), 0, st, x, s->r, p_new, s->q, keep, s->flags, g, cfg,
                                                          s->S, s->I, s->rb(), L.ctl);
      }
      CHECK_LAUNCH();
      return 0;
    };
    if (cap) {
      TRY(loop_open(s, stream, &L));
      TRY(pass(s->aux, s->pa, s->pb, s->pa));
      TRY(loop_close(s));
    } else {
      double* pc = s->pa;
      double* po = s->pb;
      for (;;) {
        TRY(read_flags(s, stream));
        if (s->hI[I_DONE]) break;
        TRY(pass(stream, pc, po, nullptr));
        std::swap(pc, po);
      }
    }
    pdl_launch(s, k_finish_stats<double>, s->cgrid, s->cblock, 0, stream, x, s->b, s->flags, g, cfg, 1, s->S, s->I, s->rb());
    CHECK_LAUNCH();
  } else {
    const int project_x0 = kind == PCFD_SOLVER_MULTIGRID;
    pdl_launch(s, k_stationary_init, s->cgrid, s->cblock, 0, stream, s->b, x, s->flags, g, cfg, has_x0, project_x0, s->S,
                                                     s->I, s->rb());
    CHECK_LAUNCH();
    if (kind == PCFD_SOLVER_MULTIGRID) {
      Loop L;
      TRY(loop_handle(s, stream, &L));
      pdl_launch(s, k_apply_mean, s->cgrid, s->cblock, 0, stream, s->b, s->flags, g, s->S, S_MEAN_B);
      CHECK_LAUNCH();
      pdl_launch(s, k_apply_mean, s->cgrid, s->cblock, 0, stream, x, s->flags, g, s->S, S_MEAN_X);
      CHECK_LAUNCH();
      pdl_launch(s, k_resnorm, s->cgrid, s->cblock, 0, stream, x, s->b, s->flags, g, cfg, 1, 0, 0, s->S, s->I, s->rb(), L.ctl);
      CHECK_LAUNCH();
      auto cycle = [&](cudaStream_t st) -> int {
        TRY(vcycle_standalone(s, s->b, x, st));
        pdl_launch(s, k_resnorm, s->cgrid, s->cblock, 0, st, x, s->b, s->flags, g, cfg, 1, 1, 1, s->S, s->I, s->rb(), L.ctl);
        CHECK_LAUNCH();
        pdl_launch(s, k_apply_mean, s->cgrid, s->cblock, 0, st, x, s->flags, g, s->S, S_MEAN_X);
        CHECK_LAUNCH();
        return 0;
      };
      if (cap) {
        TRY(loop_open(s, stream, &L));
        TRY(cycle(s->aux));
        TRY(loop_close(s));
      } else {
        for (;;) {
          TRY(read_flags(s, stream));
          if (s->hI[I_DONE]) break;
          TRY(cycle(stream));
        }
      }
    } else {
      if (cap) return fail(PCFD_E_UNSUPPORTED, "Jacobi/SOR solves are not recorded into graphs");
      double* cur = x;
      double* oth = s->xtmp;
      const int every = kind == PCFD_SOLVER_JACOBI ? 20 : 5;
      for (int it = 1; it <= s->maxiter; ++it) {
        if (kind == PCFD_SOLVER_JACOBI) {
          pdl_launch(s, k_jacobi_sweep, s->cgrid, s->cblock, 0, stream, cur, oth, s->b, s->flags, g, 2.0 / 3.0, s->singular,
                                                        s->S, s->I, s->rb());
          CHECK_LAUNCH();
          std::swap(cur, oth);
        } else {
          pdl_launch(s, k_sor_half, s->cgrid, s->cblock, 0, stream, cur, s->b, s->flags, g, s->omega, 0, s->singular, s->S,
                                                    s->I, s->rb());
          CHECK_LAUNCH();
          pdl_launch(s, k_sor_half, s->cgrid, s->cblock, 0, stream, cur, s->b, s->flags, g, s->omega, 1, s->singular, s->S,
                                                    s->I, s->rb());
          CHECK_LAUNCH();
        }
        if (it % every == 0 || it == s->maxiter) {
          pdl_launch(s, k_resnorm, s->cgrid, s->cblock, 0, stream, cur, s->b, s->flags, g, cfg, 0, 0, 1, s->S, s->I, s->rb(),
                                                   LoopCtl{0, 0});
          CHECK_LAUNCH();
          TRY(read_flags(s, stream));
          if (s->hI[I_DONE]) break;
        }
      }
      if (cur != x) CU(cudaMemcpyAsync(x, cur, s->ncell() * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    }
    pdl_launch(s, k_finish_stats<double>, s->cgrid, s->cblock, 0, stream, x, s->b, s->flags, g, cfg, 0, s->S, s->I, s->rb());
    CHECK_LAUNCH();
  }
  pdl_launch(s, k_finish_apply<double>, s->cgrid, s->cblock, 0, stream, x, x, s->flags, g, s->S, s->I);
  CHECK_LAUNCH();
  return 0;
}

int set_dt(pycfd_solver* s, double dt, double blend, cudaStream_t stream) {
  // Step parameters live in device memory so a recorded step replays with new
  // values; they travel as kernel arguments, so no host synchronisation.
  pdl_launch(s, k_begin, 1, 32, 0, stream, s->S, s->I, dt, blend);
  CHECK_LAUNCH();
  return 0;
}

// ProjectionSolver.project: solve lap p = div(u)/dt with the warm start, then
// correct the solvable faces and write the ghosted p.
int project_impl(pycfd_solver* s, double* u, double* v, double* p, double dt_override,
                 cudaStream_t stream) {
  const int G = grid1(s);
  pdl_launch(s, k_div_rhs, s->cgrid, s->cblock, 0, stream, u, v, nullptr, s->flags, s->g, s->S, s->b, s->rb(), s->S);
  CHECK_LAUNCH();
  if (s->precision == PCFD_MIXED) TRY(solve_mixed(s, s->x, s->has_guess, stream));
  else TRY(solve_prepared(s, s->x, s->has_guess, stream));
  s->has_guess = true;
  const int gc = std::min(s->g.nx + 2, kMaxRedBlocks) + 1;   // rows + the ghost-ring block
  prof_mark(s, 7, stream);
  pdl_launch(s, k_correct, gc, 256, 0, stream, u, v, p, s->x, s->g, s->S, dt_override, s->bc_kind_dev);
  prof_mark(s, 7, stream);
  CHECK_LAUNCH();
  return 0;
}

int substep_impl(pycfd_solver* s, StageIn uin, StageIn vin, double* us, double* vs, double* p,
                 cudaStream_t stream) {
  const Geo& g = s->g;
  dim3 blk(TJ, TI);
  dim3 grd((g.ny + 3 + TJ - 1) / TJ, (g.nx + 3 + TI - 1) / TI);
  if (s->les) {
    // the stage input's effective viscosity, then the predictor in stress-divergence form
    const int lg = grid_for((long)(g.nx + 2) * (g.ny + 2), 256, kWaveBlocks);
    if (g.met)
      pdl_launch(s, k_les_nu<Metrics>, lg, 256, 0, stream, uin, vin, g, Metrics(g), s->les_coeff,
                 (const double*)s->les_coeff_c, s->les_nu_c);
    else
      pdl_launch(s, k_les_nu<UniSp>, lg, 256, 0, stream, uin, vin, g, UniSp{g.dx, g.dy}, s->les_coeff,
                 (const double*)nullptr, s->les_nu_c);
    CHECK_LAUNCH();
    pdl_launch(s, k_les_corner, grid_for((long)(g.nx + 1) * (g.ny + 1), 256, kWaveBlocks), 256, 0, stream,
               (const double*)s->les_nu_c, g, s->les_nu_k);
    CHECK_LAUNCH();
    prof_mark(s, 6, stream);
    pdl_launch(s, k_predictor_les, grd, blk, 0, stream, uin, vin, us, vs, g, (const double*)s->S,
               (const double*)s->les_nu_c, (const double*)s->les_nu_k);
    prof_mark(s, 6, stream);
  } else {
    prof_mark(s, 6, stream);
    pdl_launch(s, k_predictor, grd, blk, 0, stream, uin, vin, us, vs, g, s->S);
    prof_mark(s, 6, stream);
  }
  CHECK_LAUNCH();
  TRY(launch_boundary(s, us, vs, {OP_VEL_PRED, OP_MASS, OP_MASK_RESET, OP_WRAP_FACES}, stream));
  TRY(project_impl(s, us, vs, p, -1.0, stream));
  TRY(launch_boundary(s, us, vs, {OP_MASK_ACC, OP_WRAP_FACES, OP_VEL_CORR}, stream));
  return 0;
}

int step_impl(pycfd_solver* s, const double* u0, const double* v0, double* u, double* v, double* p,
              cudaStream_t stream) {
  const long nu = (long)(s->g.nx + 3) * (s->g.ny + 2), nv = (long)(s->g.nx + 2) * (s->g.ny + 3);
  StageIn U0{u0, nullptr, 1.0, 0.0}, V0{v0, nullptr, 1.0, 0.0};
  if (s->scheme == PCFD_EULER) {
    TRY(substep_impl(s, U0, V0, u, v, p, stream));
    return 0;
  }
  if (s->scheme == PCFD_RK2) {
    TRY(substep_impl(s, U0, V0, s->us1, s->vs1, p, stream));
    TRY(substep_impl(s, StageIn{s->us1, nullptr, 1.0, 0.0}, StageIn{s->vs1, nullptr, 1.0, 0.0}, s->us2,
                     s->vs2, p, stream));
    pdl_launch(s, k_combine, grid_for(nu, 256), 256, 0, stream, u0, s->us2, 0.5, 0.5, u, nu);
    CHECK_LAUNCH();
    pdl_launch(s, k_combine, grid_for(nv, 256), 256, 0, stream, v0, s->vs2, 0.5, 0.5, v, nv);
    CHECK_LAUNCH();
  } else {
    TRY(substep_impl(s, U0, V0, s->us1, s->vs1, p, stream));
    TRY(substep_impl(s, StageIn{s->us1, nullptr, 1.0, 0.0}, StageIn{s->vs1, nullptr, 1.0, 0.0}, s->us2,
                     s->vs2, p, stream));
    TRY(substep_impl(s, StageIn{u0, s->us2, 0.75, 0.25}, StageIn{v0, s->vs2, 0.75, 0.25}, s->us1, s->vs1,
                     p, stream));
    pdl_launch(s, k_combine, grid_for(nu, 256), 256, 0, stream, u0, s->us1, 1.0 / 3.0, 2.0 / 3.0, u, nu);
    CHECK_LAUNCH();
    pdl_launch(s, k_combine, grid_for(nv, 256), 256, 0, stream, v0, s->vs1, 1.0 / 3.0, 2.0 / 3.0, v, nv);
    CHECK_LAUNCH();
  }
  TRY(launch_boundary(s, u, v, {OP_VEL_CORR, OP_WRAP_FACES}, stream));
  return 0;
}

}  // namespace

// ============================================================================
// C ABI
// ============================================================================
extern "C" {

const char* pycfd_last_error(void) { return g_err.c_str(); }
int pycfd_version(void) { return 1; }

int pycfd_solver_destroy(pycfd_solver* s) {
  if (!s) return 0;
  for (auto& e : s->prof_ev) cudaEventDestroy(e);
  for (auto& e : s->graphs) {
    cudaGraphExecDestroy(e.exec);
    cudaGraphDestroy(e.graph);
  }
  if (s->aux) cudaStreamDestroy(s->aux);
  if (s->rec) cudaStreamDestroy(s->rec);
  if (s->aux2) cudaStreamDestroy(s->aux2);
  if (s->gate) cudaStreamDestroy(s->gate);
  for (void* p : s->allocs) cudaFree(p);
  if (s->hS) cudaFreeHost(s->hS);
  if (s->hI) cudaFreeHost(s->hI);
  delete s;
  return 0;
}

int pycfd_solver_create(const pycfd_solver_desc* d, pycfd_solver** out) {
  if (!d || !out) return fail(PCFD_E_ARG, "null descriptor");
  if (d->nx < 4 || d->ny < 4) return fail(PCFD_E_ARG, "mesh must be at least 4x4 cells");
  if (d->solver_kind < PCFD_SOLVER_CG || d->solver_kind > PCFD_SOLVER_MGCG)
    return fail(PCFD_E_UNSUPPORTED, "pressure solver %d is not provided on the GPU path", d->solver_kind);
  if (d->n_bodies < 0 || d->n_bodies > PCFD_MAX_BODIES) return fail(PCFD_E_ARG, "too many bodies");
  pycfd_solver* s = new pycfd_solver();
  auto bail = [&](int rc) { pycfd_solver_destroy(s); return rc; };
  const int nx = d->nx, ny = d->ny;
  Geo& g = s->g;
  g.nx = nx;
  g.ny = ny;
  g.dx = d->dx;
  g.dy = d->dy;
  g.nu = d->nu;
  g.fx = d->body_fx;
  g.fy = d->body_fy;
  g.cx = 1.0 / (d->dx * d->dx);
  g.cy = 1.0 / (d->dy * d->dy);
  const int* K = d->bc_kind;
  g.periodic_x = K[W_LEFT] == BC_PERIODIC;
  g.periodic_y = K[W_BOTTOM] == BC_PERIODIC;
  if ((K[W_LEFT] == BC_PERIODIC) != (K[W_RIGHT] == BC_PERIODIC) ||
      (K[W_BOTTOM] == BC_PERIODIC) != (K[W_TOP] == BC_PERIODIC))
    return bail(fail(PCFD_E_ARG, "periodicity must be set on both walls of an axis"));
  const int PO = BC_PRESSURE_OUTLET;
  // solvable face ranges (pycfd/core/solver.py:235-263)
  g.u_lo = (g.periodic_x || K[W_LEFT] == PO) ? 1 : 2;
  g.u_hi = (K[W_RIGHT] == PO && !g.periodic_x) ? nx + 2 : nx + 1;
  g.v_lo = (g.periodic_y || K[W_BOTTOM] == PO) ? 1 : 2;
  g.v_hi = (K[W_TOP] == PO && !g.periodic_y) ? ny + 2 : ny + 1;
  g.dir_w = K[W_LEFT] == PO;
  g.dir_e = K[W_RIGHT] == PO;
  g.dir_s = K[W_BOTTOM] == PO;
  g.dir_n = K[W_TOP] == PO;
  g.pref_w = d->bc_p_ref[W_LEFT];
  g.pref_e = d->bc_p_ref[W_RIGHT];
  g.pref_s = d->bc_p_ref[W_BOTTOM];
  g.pref_n = d->bc_p_ref[W_TOP];
  s->singular = !(g.dir_w || g.dir_e || g.dir_s || g.dir_n);
  s->solver_kind = d->solver_kind;
  s->tol = d->tol;
  s->maxiter = d->maxiter;
  s->omega = d->sor_omega;
  s->mg_sweeps = std::max(1, d->mg_sweeps);
  s->scheme = d->time_scheme;
  if (d->metrics) {   // stretched mesh: the packed metrics, read by every stencil through g.met
    int mrc;
    if ((mrc = upload(s, &s->met, d->metrics, (size_t)metrics_count(nx, ny)))) return bail(mrc);
    g.met = s->met;
    if (d->use_les) {   // the per-cell filter coefficient (Cs Delta)^2 on the ghosted cell grid
      if (!d->les_coeff_field) return bail(fail(PCFD_E_ARG, "LES on a stretched mesh needs les_coeff_field"));
      if ((mrc = upload(s, &s->les_coeff_c, d->les_coeff_field, (size_t)(nx + 2) * (ny + 2)))) return bail(mrc);
    }
  }
  if (d->use_les) {
    if (!(d->les_coeff >= 0.0)) return bail(fail(PCFD_E_ARG, "les_coeff must be non-negative"));
    s->les = 1;
    s->les_coeff = d->les_coeff;
    int lrc;
    if ((lrc = dalloc(s, &s->les_nu_c, (size_t)(d->nx + 2) * (d->ny + 2))) ||
        (lrc = dalloc(s, &s->les_nu_k, (size_t)(d->nx + 1) * (d->ny + 1))))
      return bail(lrc);
  }
  s->precision = d->precision;
  s->inner_tol = d->inner_tol > 0 ? d->inner_tol : 1e-4;
  s->pdl = d->sequential_launch ? 0 : 1;
  {
    int dev = 0, nsm = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // default: eight 256-thread blocks per SM (measured best of 4..12 on the 512^2 vortex;
    // with the ELL kernels' <= 48 registers five are resident, the rest follow as they end)
    s->ell_budget = d->ell_thread_budget ? (long)d->ell_thread_budget : (long)nsm * 8 * 256;
    s->ell_blocks = s->ell_budget > 0 ? (int)std::max<long>(1, s->ell_budget / 256) : kWaveBlocks;
  }

  // ---- cell flags of the fine operator (pycfd/core/pressure.py:209-247) ----
  const long n = (long)nx * ny;
  std::vector<uint8_t> solid(n, 0), flags(n, 0);
  if (d->solid)
    for (long c = 0; c < n; ++c) solid[c] = d->solid[c] ? 1 : 0;
  auto fluid = [&](int i, int j) { return !solid[(long)i * ny + j]; };
  int n_fluid = 0;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      if (!fluid(i, j)) continue;
      uint8_t f = 0;
      const bool in_w = i > 0 || g.periodic_x, in_e = i < nx - 1 || g.periodic_x;
      const bool in_s = j > 0 || g.periodic_y, in_n = j < ny - 1 || g.periodic_y;
      if (in_w && fluid((i + nx - 1) % nx, j)) f |= F_W;
      if (in_e && fluid((i + 1) % nx, j)) f |= F_E;
      if (in_s && fluid(i, (j + ny - 1) % ny)) f |= F_S;
      if (in_n && fluid(i, (j + 1) % ny)) f |= F_N;
      // isolated = no active face and no Dirichlet wall contribution
      const bool dirw = g.dir_w && i == 0, dire = g.dir_e && i == nx - 1;
      const bool dirs = g.dir_s && j == 0, dirn = g.dir_n && j == ny - 1;
      if (f || dirw || dire || dirs || dirn) {
        f |= F_SOLV;
        ++n_fluid;
      }
      flags[(long)i * ny + j] = f;
    }
  g.n_fluid = n_fluid;
  cell_launch(nx, ny, &s->cgrid, &s->cblock);
  if (s->solver_kind == PCFD_SOLVER_SOR) {
    // red/black colouring must not couple a colour to itself (pycfd/core/pressure.py:486-496)
    bool bad = false;
    if (g.periodic_x && (nx % 2 == 1))
      for (int j = 0; j < ny && !bad; ++j) bad = (flags[(long)(nx - 1) * ny + j] & F_E) != 0;
    if (g.periodic_y && (ny % 2 == 1))
      for (int i = 0; i < nx && !bad; ++i) bad = (flags[(long)i * ny + ny - 1] & F_N) != 0;
    if (bad)
      return bail(fail(PCFD_E_ARG,
                       "red/black ordering is invalid for this grid (cells of one colour are coupled "
                       "to each other). This happens with an odd number of cells on a periodic axis; "
                       "use an even nx/ny"));
  }
  int rc;
  if ((rc = upload(s, &s->flags, flags.data(), n))) return bail(rc);
  if ((rc = upload(s, &s->solid, solid.data(), n))) return bail(rc);

  // ---- mask face lists (pycfd/core/solver.py:62-79, :285-296) ----
  auto solid_at = [&](int ci, int cj, int axis) -> int {
    // zero-based cell (ci, cj); off-domain = fluid unless periodic
    if (axis == 0) {
      if (ci < 0 || ci >= nx) {
        if (!g.periodic_x) return 0;
        ci = (ci % nx + nx) % nx;
      }
    } else {
      if (cj < 0 || cj >= ny) {
        if (!g.periodic_y) return 0;
        cj = (cj % ny + ny) % ny;
      }
    }
    const long c = (long)ci * ny + cj;
    if (!solid[c]) return 0;
    return d->body_id ? d->body_id[c] : 1;
  };
  const int nb = d->n_bodies;
  std::vector<std::vector<int>> mu(std::max(nb, 1)), mv(std::max(nb, 1));
  if (d->solid) {
    for (int m = g.u_lo; m < g.u_hi; ++m)
      for (int j = 1; j <= ny; ++j) {
        const int a = solid_at(m - 2, j - 1, 0), b = solid_at(m - 1, j - 1, 0);
        if (a || b) {
          const int body = nb ? std::max(a, b) - 1 : 0;
          mu[std::max(0, std::min(body, std::max(nb, 1) - 1))].push_back(m * (ny + 2) + j);
        }
      }
    for (int i = 1; i <= nx; ++i)
      for (int k = g.v_lo; k < g.v_hi; ++k) {
        const int a = solid_at(i - 1, k - 2, 1), b = solid_at(i - 1, k - 1, 1);
        if (a || b) {
          const int body = nb ? std::max(a, b) - 1 : 0;
          mv[std::max(0, std::min(body, std::max(nb, 1) - 1))].push_back(i * (ny + 3) + k);
        }
      }
  }
  std::vector<int> lu, lvv;
  s->bc.n_bodies = nb;
  for (int b = 0; b < std::max(nb, 1); ++b) {
    s->bc.body_u_start[b] = (int)lu.size();
    s->bc.body_v_start[b] = (int)lvv.size();
    lu.insert(lu.end(), mu[b].begin(), mu[b].end());
    lvv.insert(lvv.end(), mv[b].begin(), mv[b].end());
  }
  s->bc.body_u_start[std::max(nb, 1)] = (int)lu.size();
  s->bc.body_v_start[std::max(nb, 1)] = (int)lvv.size();
  if ((rc = upload(s, &s->mask_u, lu.data(), lu.size()))) return bail(rc);
  if ((rc = upload(s, &s->mask_v, lvv.data(), lvv.size()))) return bail(rc);
  s->bc.mask_u = s->mask_u;
  s->bc.mask_v = s->mask_v;
  s->bc.n_mask_u = (int)lu.size();
  s->bc.n_mask_v = (int)lvv.size();
  s->bc.area = d->dx * d->dy;
  s->bc.met = s->met;
  s->bc.nx = nx;
  s->bc.ny = ny;
  s->bc.outlet_width = d->outlet_width;
  s->bc.has_outlet = 0;
  for (int w = 0; w < 4; ++w) {
    s->bc.kind[w] = K[w];
    s->bc.vel[w] = d->bc_velocity[w];
    s->bc.pref[w] = d->bc_p_ref[w];
    s->bc.profile[w] = nullptr;
    if (K[w] == BC_OUTLET) s->bc.has_outlet = 1;
    if (K[w] == BC_INLET && d->bc_profile[w]) {
      const int len = w < 2 ? ny + 2 : nx + 2;
      if ((rc = upload(s, &s->profile[w], d->bc_profile[w], len))) return bail(rc);
      s->bc.profile[w] = s->profile[w];
    }
  }
  if ((rc = upload(s, &s->bc_kind_dev, K, 4))) return bail(rc);

  // ---- workspace ----
  const long nu_all = (long)(nx + 3) * (ny + 2), nv_all = (long)(nx + 2) * (ny + 3);
  if ((rc = dalloc(s, &s->S, S_COUNT)) || (rc = dalloc(s, &s->I, I_COUNT)) ||
      (rc = dalloc(s, &s->partials, (size_t)kMaxRedBlocks * 8)) || (rc = dalloc(s, &s->counter, 1)) ||
      (rc = dalloc(s, &s->us1, nu_all)) || (rc = dalloc(s, &s->vs1, nv_all)) ||
      (rc = dalloc(s, &s->us2, nu_all)) || (rc = dalloc(s, &s->vs2, nv_all)) ||
      (rc = dalloc(s, &s->b, n)) || (rc = dalloc(s, &s->x, n)) || (rc = dalloc(s, &s->x_api, n)) ||
      (rc = dalloc(s, &s->r, n)) || (rc = dalloc(s, &s->pa, n)) || (rc = dalloc(s, &s->pb, n)) ||
      (rc = dalloc(s, &s->q, n)) || (rc = dalloc(s, &s->z, n)) || (rc = dalloc(s, &s->xtmp, n)))
    return bail(rc);
  if (cudaHostAlloc((void**)&s->hS, S_COUNT * sizeof(double), cudaHostAllocDefault) != cudaSuccess ||
      cudaHostAlloc((void**)&s->hI, I_COUNT * sizeof(int), cudaHostAllocDefault) != cudaSuccess)
    return bail(fail(PCFD_E_CUDA, "pinned allocation failed"));
  memset(s->hS, 0, S_COUNT * sizeof(double));
  memset(s->hI, 0, I_COUNT * sizeof(int));

  // ---- multigrid hierarchy ----
  const bool mg = s->solver_kind == PCFD_SOLVER_MULTIGRID || s->solver_kind == PCFD_SOLVER_MGCG;
  if (mg) {
    if (d->n_levels < 1 || !d->levels || !d->coarsest_inverse)
      return bail(fail(PCFD_E_ARG, "multigrid solver needs a hierarchy"));
    if (d->levels[0].n != n) return bail(fail(PCFD_E_ARG, "level 0 must have nx*ny unknowns"));
    s->lv.resize(d->n_levels);
    for (int l = 0; l < d->n_levels; ++l) {
      const pycfd_mg_level& in = d->levels[l];
      Level& L = s->lv[l];
      L.n = in.n;
      L.sx = in.shape_x;
      L.sy = in.shape_y;
      L.weight = in.weight;
      const bool coarsest = l == d->n_levels - 1;
      if ((rc = dalloc(s, &L.d.b, L.n)) || (rc = dalloc(s, &L.d.xa, L.n)) || (rc = dalloc(s, &L.d.xb, L.n)) ||
          (rc = dalloc(s, &L.d.res, L.n)) || (rc = dalloc(s, &L.f.b, L.n)) || (rc = dalloc(s, &L.f.xa, L.n)) ||
          (rc = dalloc(s, &L.f.xb, L.n)) || (rc = dalloc(s, &L.f.res, L.n)))
        return bail(rc);
      if (l >= 1) {
        const pycfd_mg_level& up = d->levels[l - 1];
        if (!coarsest) {
          if (!in.a_indptr || !in.weighted_dinv) return bail(fail(PCFD_E_ARG, "level %d lacks A", l));
          if ((rc = make_ell(s, &L.A, L.n, in.a_indptr, in.a_indices, in.a_data)) ||
              (rc = make_ell(s, &L.Af, L.n, in.a_indptr, in.a_indices, in.a_data)))
            return bail(rc);
          std::vector<float> wf(in.weighted_dinv, in.weighted_dinv + L.n);
          if ((rc = upload(s, &L.wd, in.weighted_dinv, L.n)) || (rc = upload(s, &L.wdf, wf.data(), L.n)))
            return bail(rc);
        }
        if (!in.p_indptr) return bail(fail(PCFD_E_ARG, "level %d lacks P", l));
        if ((rc = make_ell(s, &L.P, up.n, in.p_indptr, in.p_indices, in.p_data)) ||
            (rc = make_ell(s, &L.Pf, up.n, in.p_indptr, in.p_indices, in.p_data)))
          return bail(rc);
        std::vector<int64_t> tp;
        std::vector<int32_t> ti;
        std::vector<double> td;
        csr_transpose(up.n, L.n, in.p_indptr, in.p_indices, in.p_data, tp, ti, td);
        if ((rc = make_ell(s, &L.R, L.n, tp.data(), ti.data(), td.data())) ||
            (rc = make_ell(s, &L.Rf, L.n, tp.data(), ti.data(), td.data())))
          return bail(rc);
        if (in.m_indptr &&
            ((rc = make_ell(s, &L.M, L.n, in.m_indptr, in.m_indices, in.m_data)) ||
             (rc = make_ell(s, &L.Mf, L.n, in.m_indptr, in.m_indices, in.m_data))))
          return bail(rc);
      }
    }
    const int ncs = d->levels[d->n_levels - 1].n;
    s->nc = ncs;
    std::vector<double> cm((size_t)ncs * ncs);
    std::vector<float> cf((size_t)ncs * ncs);
    for (size_t e = 0; e < (size_t)ncs * ncs; ++e) {   // row-major, as given
      cm[e] = d->coarsest_inverse[e];
      cf[e] = (float)d->coarsest_inverse[e];
    }
    if ((rc = upload(s, &s->C, cm.data(), cm.size())) || (rc = upload(s, &s->Cf, cf.data(), cf.size())))
      return bail(rc);
    const int tl = d->tail_level;
    if (tl > 0) {
      if (tl >= (int)s->lv.size() - 1 || !d->tail_operator)
        return bail(fail(PCFD_E_ARG, "tail_level must name a level above the coarsest, with its operator"));
      const size_t nt = (size_t)s->lv[tl].n;
      std::vector<float> tf(nt * nt);
      for (size_t e = 0; e < nt * nt; ++e) tf[e] = (float)d->tail_operator[e];
      if ((rc = upload(s, &s->tail, d->tail_operator, nt * nt)) || (rc = upload(s, &s->tailf, tf.data(), nt * nt)))
        return bail(rc);
      s->tail_level = tl;
      s->fused = 1;
      for (int l = 1; l <= tl; ++l)
        if (!d->levels[l].m_indptr) s->fused = 0;
    }
  }
  if (mg && d->coarse_cluster_rows > 0 && s->lv.size() > 1) {
    // coarse levels: first level (>= 1) with at most coarse_cluster_rows rows
    for (int l = 1; l < (int)s->lv.size(); ++l)
      if (s->lv[l].n <= d->coarse_cluster_rows) {
        s->cluster_from = l;
        break;
      }
    int best = 0;
    for (int cs : {16, 8}) {
      if (cs == 16) {
        if (cudaFuncSetAttribute(k_coarse_cycle<double>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                cudaSuccess ||
            cudaFuncSetAttribute(k_coarse_cycle<float>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                cudaSuccess) {
          cudaGetLastError();
          continue;
        }
      }
      cudaLaunchConfig_t cfg{};
      cfg.gridDim = dim3(cs);
      cfg.blockDim = dim3(1024);
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = cs;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      int nclusters = 0;
      if (cudaOccupancyMaxActiveClusters(&nclusters, k_coarse_cycle<double>, &cfg) == cudaSuccess &&
          nclusters > 0) {
        best = cs;
        break;
      }
      cudaGetLastError();
    }
    s->cluster_size = best;
    if (!best) s->cluster_from = 1 << 30;
  }
  if (d->persistent_solve && s->precision != PCFD_MIXED &&
      (s->solver_kind == PCFD_SOLVER_CG || s->solver_kind == PCFD_SOLVER_MGCG) &&
      (int)s->lv.size() <= kPMaxLevels) {
    // one CTA pair per SM at most: the grid is resident at once by construction
    int dev = 0, nsm = 0, occ_j = 0, occ_m = 0;
    CU(cudaGetDevice(&dev));
    CU(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_j, k_solve_persistent<double, PC_JACOBI>, kPThreads, 0));
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_m, k_solve_persistent<double, PC_MG>, kPThreads, 0));
    const int per_sm = std::min(2, std::min(occ_j, occ_m));
    if (per_sm < 1) return bail(fail(PCFD_E_CUDA, "persistent solve: no CTA fits an SM"));
    s->persistent = nsm * per_sm;
    if ((rc = dalloc(s, &s->pbar, 64)) || (rc = dalloc(s, &s->ppart, (size_t)s->persistent * 2 * kPMaxNV)))
      return bail(rc);
  }
  if (s->precision == PCFD_MIXED) {
    if ((rc = dalloc(s, &s->r32, n)) || (rc = dalloc(s, &s->x32, n)) || (rc = dalloc(s, &s->pa32, n)) ||
        (rc = dalloc(s, &s->pb32, n)) || (rc = dalloc(s, &s->q32, n)) || (rc = dalloc(s, &s->z32, n)))
      return bail(rc);
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return bail(fail(PCFD_E_CUDA, "setup failed"));
  *out = s;
  return 0;
}

int pycfd_solver_momentum_rhs(pycfd_solver* s, const double* u, const double* v, double blend, double* rhs_u,
                              double* rhs_v, void* stream) {
  if (!s || !u || !v || !rhs_u || !rhs_v) return fail(PCFD_E_ARG, "bad arguments");
  const Geo& g = s->g;
  if (s->les) return fail(PCFD_E_UNSUPPORTED, "use pycfd_momentum_rhs_les for the Smagorinsky closure");
  dim3 blk(TJ, TI), grd((g.ny + 1 + TJ - 1) / TJ, (g.nx + 1 + TI - 1) / TI);
  if (g.met) k_rhs_str<<<grd, blk, 0, st(stream)>>>(u, v, g, blend, rhs_u, rhs_v);
  else k_rhs<<<grd, blk, 0, st(stream)>>>(u, v, g.nx, g.ny, g.dx, g.dy, g.nu, blend, g.fx, g.fy, rhs_u, rhs_v);
  CHECK_LAUNCH();
  return 0;
}

int pycfd_solver_momentum_rhs_les(pycfd_solver* s, const double* u, const double* v, double blend, double* nu_c,
                                  double* nu_corner, double* rhs_u, double* rhs_v, void* stream) {
  if (!s || !u || !v || !nu_c || !nu_corner || !rhs_u || !rhs_v) return fail(PCFD_E_ARG, "bad arguments");
  if (!s->les) return fail(PCFD_E_ARG, "the solver was created without the Smagorinsky closure");
  const Geo& g = s->g;
  cudaStream_t sm = st(stream);
  const StageIn U{u, nullptr, 1.0, 0.0}, V{v, nullptr, 1.0, 0.0};
  const int lg = grid_for((long)(g.nx + 2) * (g.ny + 2), 256, kWaveBlocks);
  if (g.met) k_les_nu<Metrics><<<lg, 256, 0, sm>>>(U, V, g, Metrics(g), s->les_coeff, s->les_coeff_c, nu_c);
  else k_les_nu<UniSp><<<lg, 256, 0, sm>>>(U, V, g, UniSp{g.dx, g.dy}, s->les_coeff, nullptr, nu_c);
  CHECK_LAUNCH();
  k_les_corner<<<grid_for((long)(g.nx + 1) * (g.ny + 1), 256, kWaveBlocks), 256, 0, sm>>>(nu_c, g, nu_corner);
  CHECK_LAUNCH();
  dim3 blk(TJ, TI), grd((g.ny + 1 + TJ - 1) / TJ, (g.nx + 1 + TI - 1) / TI);
  k_rhs_les_g<<<grd, blk, 0, sm>>>(u, v, g, blend, nu_c, nu_corner, rhs_u, rhs_v);
  CHECK_LAUNCH();
  return 0;
}

int pycfd_solver_divergence(pycfd_solver* s, const double* u, const double* v, double* out, void* stream) {
  if (!s || !u || !v || !out) return fail(PCFD_E_ARG, "bad arguments");
  const Geo& g = s->g;
  k_divergence_g<<<grid_for((long)g.nx * g.ny, 256), 256, 0, st(stream)>>>(u, v, g, out);
  CHECK_LAUNCH();
  return 0;
}

int pycfd_momentum_rhs(const double* u, const double* v, int nx, int ny, double dx, double dy, double nu,
                       double blend, double fx, double fy, double* rhs_u, double* rhs_v, void* stream) {
  if (!u || !v || !rhs_u || !rhs_v || nx < 1 || ny < 1) return fail(PCFD_E_ARG, "bad arguments");
  dim3 blk(TJ, TI), grd((ny + 1 + TJ - 1) / TJ, (nx + 1 + TI - 1) / TI);
  k_rhs<<<grd, blk, 0, st(stream)>>>(u, v, nx, ny, dx, dy, nu, blend, fx, fy, rhs_u, rhs_v);
  CHECK_LAUNCH();
  return 0;
}

int pycfd_momentum_rhs_les(const double* u, const double* v, int nx, int ny, double dx, double dy, double nu,
                           double les_coeff, double blend, double fx, double fy, double* nu_c, double* nu_corner,
                           double* rhs_u, double* rhs_v, void* stream) {
  if (!u || !v || !nu_c || !nu_corner || !rhs_u || !rhs_v || nx < 1 || ny < 1 || !(les_coeff >= 0.0))
    return fail(PCFD_E_ARG, "bad arguments");
  cudaStream_t sm = st(stream);
  Geo g{};
  g.nx = nx;
  g.ny = ny;
  g.dx = dx;
  g.dy = dy;
  g.nu = nu;
  const StageIn U{u, nullptr, 1.0, 0.0}, V{v, nullptr, 1.0, 0.0};
  k_les_nu<UniSp><<<grid_for((long)(nx + 2) * (ny + 2), 256, kWaveBlocks), 256, 0, sm>>>(U, V, g, UniSp{dx, dy},
                                                                                         les_coeff, nullptr, nu_c);
  CHECK_LAUNCH();
  k_les_corner<<<grid_for((long)(nx + 1) * (ny + 1), 256, kWaveBlocks), 256, 0, sm>>>(nu_c, g, nu_corner);
  CHECK_LAUNCH();
  dim3 blk(TJ, TI), grd((ny + 1 + TJ - 1) / TJ, (nx + 1 + TI - 1) / TI);
  k_rhs_les<<<grd, blk, 0, sm>>>(u, v, nx, ny, dx, dy, blend, fx, fy, nu_c, nu_corner, rhs_u, rhs_v);
  CHECK_LAUNCH();
  return 0;
}

int pycfd_divergence(const double* u, const double* v, int nx, int ny, double dx, double dy, double* out,
                     void* stream) {
  if (!u || !v || !out || nx < 1 || ny < 1) return fail(PCFD_E_ARG, "bad arguments");
  dim3 cg, cb;
  cell_launch(nx, ny, &cg, &cb);
  k_divergence<<<cg, cb, 0, st(stream)>>>(u, v, nx, ny, dx, dy, out);
  CHECK_LAUNCH();
  return 0;
}

int pycfd_apply_velocity_bc(pycfd_solver* s, double* u, double* v, int predictor, int mass_balance,
                            void* stream) {
  if (!s || !u || !v) return fail(PCFD_E_ARG, "bad arguments");
  if (mass_balance)
    return launch_boundary(s, u, v, {predictor ? OP_VEL_PRED : OP_VEL_CORR, OP_MASS}, st(stream));
  return launch_boundary(s, u, v, {predictor ? OP_VEL_PRED : OP_VEL_CORR}, st(stream));
}

int pycfd_poisson_solve(pycfd_solver* s, const double* rhs, const double* p0, double* p, void* stream) {
  if (!s || !rhs || !p) return fail(PCFD_E_ARG, "bad arguments");
  cudaStream_t sm = st(stream);
  const int G = grid1(s);
  TRY(set_dt(s, 1.0, 0.0, sm));
  pdl_launch(s, k_div_rhs, s->cgrid, s->cblock, 0, sm, nullptr, nullptr, rhs, s->flags, s->g, s->S, s->b, s->rb(), s->S);
  CHECK_LAUNCH();
  if (p0) CU(cudaMemcpyAsync(s->x_api, p0, s->ncell() * sizeof(double), cudaMemcpyDeviceToDevice, sm));
  if (s->precision == PCFD_MIXED) TRY(solve_mixed(s, s->x_api, p0 != nullptr, sm));
  else TRY(solve_prepared(s, s->x_api, p0 != nullptr, sm));
  CU(cudaMemcpyAsync(p, s->x_api, s->ncell() * sizeof(double), cudaMemcpyDeviceToDevice, sm));
  return 0;
}

int pycfd_mg_apply(pycfd_solver* s, const double* r, double* z, void* stream) {
  if (!s || !r || !z) return fail(PCFD_E_ARG, "bad arguments");
  if (s->lv.empty()) return fail(PCFD_E_ARG, "solver has no multigrid hierarchy");
  cudaStream_t sm = st(stream);
  const int G = grid1(s);
  // mean of r over the active set, then one cycle and the projection of z
  pdl_launch(s, k_div_rhs, s->cgrid, s->cblock, 0, sm, nullptr, nullptr, r, s->flags, s->g, s->S, s->b, s->rb(), s->S);
  CHECK_LAUNCH();
  // k_div_rhs left the solvable sum in S_MEAN_B; the cycle reads S_MEAN_R.
  CU(cudaMemcpyAsync(s->S + S_MEAN_R, s->S + S_MEAN_B, sizeof(double), cudaMemcpyDeviceToDevice, sm));
  CU(cudaMemsetAsync(s->S + S_SUM_R, 0, sizeof(double), sm));
  CU(cudaMemsetAsync(s->I + I_ZERO_RHS, 0, sizeof(int), sm));
  TRY(vcycle_pcg<double>(s, r, s->z, sm));
  // z = z_raw - mean_z on solvable rows, 0 elsewhere
  CU(cudaMemcpyAsync(s->S + S_MEAN_X, s->S + S_MEAN_Z, sizeof(double), cudaMemcpyDeviceToDevice, sm));
  pdl_launch(s, k_finish_apply<double>, s->cgrid, s->cblock, 0, sm, s->z, z, s->flags, s->g, s->S, s->I);
  CHECK_LAUNCH();
  return 0;
}

int pycfd_project(pycfd_solver* s, double* u, double* v, double* p, double dt, void* stream) {
  if (!s || !u || !v || !p || !(dt > 0)) return fail(PCFD_E_ARG, "bad arguments");
  cudaStream_t sm = st(stream);
  TRY(set_dt(s, dt, 0.0, sm));
  return project_impl(s, u, v, p, -1.0, sm);
}

int pycfd_initialize(pycfd_solver* s, double* u, double* v, double* p, void* stream) {
  if (!s || !u || !v || !p) return fail(PCFD_E_ARG, "bad arguments");
  cudaStream_t sm = st(stream);
  TRY(set_dt(s, 1.0, 0.0, sm));
  TRY(launch_boundary(s, u, v, {OP_VEL_PRED, OP_MASS, OP_MASK_NONE, OP_WRAP_FACES}, sm));
  TRY(project_impl(s, u, v, p, -1.0, sm));
  TRY(launch_boundary(s, u, v, {OP_MASK_NONE, OP_WRAP_FACES, OP_VEL_CORR}, sm));
  return 0;
}

int pycfd_substep(pycfd_solver* s, const double* u, const double* v, double* us, double* vs, double* p,
                  double dt, double blend, void* stream) {
  if (!s || !u || !v || !us || !vs || !p) return fail(PCFD_E_ARG, "bad arguments");
  cudaStream_t sm = st(stream);
  TRY(set_dt(s, dt, blend, sm));
  return substep_impl(s, StageIn{u, nullptr, 1.0, 0.0}, StageIn{v, nullptr, 1.0, 0.0}, us, vs, p, sm);
}

int pycfd_step(pycfd_solver* s, const double* u0, const double* v0, double* u, double* v, double* p,
               double dt, double blend, void* stream) {
  if (!s || !u0 || !v0 || !u || !v || !p) return fail(PCFD_E_ARG, "bad arguments");
  if (u0 == u || v0 == v) return fail(PCFD_E_ARG, "step outputs must not alias its inputs");
  cudaStream_t sm = st(stream);
  TRY(set_dt(s, dt, blend, sm));
  return step_impl(s, u0, v0, u, v, p, sm);
}

int pycfd_step_graph(pycfd_solver* s, const double* u0, const double* v0, double* u, double* v,
                     double* p, double dt, double blend, void* stream) {
  if (!s || !u0 || !v0 || !u || !v || !p) return fail(PCFD_E_ARG, "bad arguments");
  if (u0 == u || v0 == v) return fail(PCFD_E_ARG, "step outputs must not alias its inputs");
  cudaStream_t sm = st(stream);
  if (s->solver_kind == PCFD_SOLVER_JACOBI || s->solver_kind == PCFD_SOLVER_SOR)
    return pycfd_step(s, u0, v0, u, v, p, dt, blend, stream);   // host-checked cadence
  TRY(set_dt(s, dt, blend, sm));
  const void* key[5] = {u0, v0, u, v, p};
  pycfd_solver::GraphEntry* hit = nullptr;
  for (auto& e : s->graphs)
    if (!e.adaptive && !memcmp(e.key, key, sizeof key)) hit = &e;
  if (!hit) {
    // Record on the solver's own stream (the caller's may be the legacy default
    // stream, which cannot be captured); recording executes nothing.
    if (!s->aux) CU(cudaStreamCreateWithFlags(&s->aux, cudaStreamNonBlocking));
    if (!s->rec) CU(cudaStreamCreateWithFlags(&s->rec, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    CU(cudaStreamBeginCapture(s->rec, cudaStreamCaptureModeThreadLocal));
    s->capturing = true;
    const int rc = step_impl(s, u0, v0, u, v, p, s->rec);
    s->capturing = false;
    const cudaError_t ec = cudaStreamEndCapture(s->rec, &graph);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (ec != cudaSuccess) return fail(PCFD_E_CUDA, "step capture failed: %s", cudaGetErrorString(ec));
    cudaGraphExec_t exec = nullptr;
    CU(cudaGraphInstantiate(&exec, graph, 0));
    if (s->graphs.size() >= 4) {   // small cache: drop the oldest recording
      cudaGraphExecDestroy(s->graphs.front().exec);
      cudaGraphDestroy(s->graphs.front().graph);
      s->graphs.erase(s->graphs.begin());
    }
    pycfd_solver::GraphEntry e{};
    memcpy(e.key, key, sizeof key);
    e.graph = graph;
    e.exec = exec;
    s->graphs.push_back(e);
    hit = &s->graphs.back();
  }
  CU(cudaGraphLaunch(hit->exec, sm));
  return 0;
}

}  // extern "C"

namespace {

// The body of a device-loop step, captured on s->rec after the statistics of
// the input state: the gate kernel sets the condition of an IF node whose body
// is the step, the statistics of its result (and its change) and the history
// row.  A frozen run replays the graph without touching the state.
int record_gated_step(pycfd_solver* s, const double* u0, const double* v0, double* u, double* v, double* p,
                      const DtControl& c) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  CU(cudaStreamGetCaptureInfo(s->rec, &cs, nullptr, &g, nullptr, nullptr));
  cudaGraphConditionalHandle h;
  CU(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
  const LoopCtl gate{h, 1};
  k_step_gate<<<1, 32, 0, s->rec>>>(s->S, s->I, c, gate);
  CHECK_LAUNCH();
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  CU(cudaStreamGetCaptureInfo(s->rec, &cs, nullptr, &g, &deps, &nd));
  cudaGraphNodeParams np{};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeIf;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  CU(cudaGraphAddNode(&node, g, deps, nd, &np));
  CU(cudaStreamUpdateCaptureDependencies(s->rec, &node, 1, cudaStreamSetCaptureDependencies));
  if (!s->gate) CU(cudaStreamCreateWithFlags(&s->gate, cudaStreamNonBlocking));
  // the IF body, recorded on its own stream (the step's solve loops nest inside it)
  CU(cudaStreamBeginCaptureToGraph(s->gate, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                   cudaStreamCaptureModeRelaxed));
  int rc = step_impl(s, u0, v0, u, v, p, s->gate);
  if (!rc) {
    k_field_stats<<<std::min(s->g.nx + 3, kMaxRedBlocks), kRedThreads, 0, s->gate>>>(
        u, v, p, u0, v0, s->solid, s->g, s->rb(), s->S);
    if (cudaGetLastError() != cudaSuccess) rc = fail(PCFD_E_CUDA, "stats launch failed");
    k_history_append<<<1, 32, 0, s->gate>>>(s->S, s->I, s->hist, kHistRows, c);
    if (!rc && cudaGetLastError() != cudaSuccess) rc = fail(PCFD_E_CUDA, "history launch failed");
    g_launches.fetch_add(2);
  }
  cudaGraph_t body = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(s->gate, &body);
  if (rc) return rc;
  if (ec != cudaSuccess) return fail(PCFD_E_CUDA, "gated step capture failed: %s", cudaGetErrorString(ec));
  return 0;
}

}  // namespace

extern "C" {

int pycfd_step_adaptive(pycfd_solver* s, const double* u0, const double* v0, double* u, double* v,
                        double* p, const pycfd_dt_control* ctl, void* stream) {
  if (!s || !u0 || !v0 || !u || !v || !p || !ctl) return fail(PCFD_E_ARG, "bad arguments");
  if (u0 == u || v0 == v) return fail(PCFD_E_ARG, "step outputs must not alias its inputs");
  if (s->solver_kind == PCFD_SOLVER_JACOBI || s->solver_kind == PCFD_SOLVER_SOR)
    return fail(PCFD_E_UNSUPPORTED, "device-side stepping needs a cg, multigrid or mgcg solver");
  cudaStream_t sm = st(stream);
  DtControl c;
  memset(&c, 0, sizeof c);   // compared bytewise below
  c.adaptive = ctl->adaptive;
  c.cfl = ctl->cfl;
  c.visc_limit = ctl->visc_limit;
  c.dt_cap = ctl->dt_cap;
  c.t_end = ctl->t_end;
  c.dx = s->g.dx;
  c.dy = s->g.dy;
  c.blend_mode = ctl->blend_mode;
  c.blend = ctl->blend;
  c.steady_tol = ctl->steady_tol;
  c.history = ctl->history ? 1 : 0;
  c.ke_scale = s->g.met ? 1.0 : s->g.dx * s->g.dy;
  if (c.history && !s->hist) TRY(dalloc(s, &s->hist, (size_t)kHistRows * kHistCols));
  // key: the five addresses plus the control values (recorded into the graph)
  const void* key[5] = {u0, v0, u, v, p};
  pycfd_solver::GraphEntry* hit = nullptr;
  for (auto& e : s->graphs)
    if (e.adaptive && !memcmp(e.key, key, sizeof key) && !memcmp(&e.ctl, &c, sizeof c)) hit = &e;
  if (!hit) {
    if (!s->aux) CU(cudaStreamCreateWithFlags(&s->aux, cudaStreamNonBlocking));
    if (!s->rec) CU(cudaStreamCreateWithFlags(&s->rec, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    CU(cudaStreamBeginCapture(s->rec, cudaStreamCaptureModeThreadLocal));
    s->capturing = true;
    int rc = 0;
    pdl_launch(s, k_field_stats, std::min(s->g.nx + 3, kMaxRedBlocks), kRedThreads, 0, s->rec, 
        u0, v0, nullptr, nullptr, nullptr, s->solid, s->g, s->rb(), s->S);
    if (cudaGetLastError() != cudaSuccess) rc = fail(PCFD_E_CUDA, "stats launch failed");
    g_launches.fetch_add(1);
    if (!c.history) {
      pdl_launch(s, k_adaptive_dt, 1, 32, 0, s->rec, s->S, s->I, c);
      if (!rc && cudaGetLastError() != cudaSuccess) rc = fail(PCFD_E_CUDA, "dt launch failed");
      g_launches.fetch_add(1);
      if (!rc) rc = step_impl(s, u0, v0, u, v, p, s->rec);
    } else if (!rc) {
      // gated step: [gate] -> IF { step, statistics of the new state, history row }
      rc = record_gated_step(s, u0, v0, u, v, p, c);
    }
    s->capturing = false;
    const cudaError_t ec = cudaStreamEndCapture(s->rec, &graph);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (ec != cudaSuccess) return fail(PCFD_E_CUDA, "step capture failed: %s", cudaGetErrorString(ec));
    cudaGraphExec_t exec = nullptr;
    CU(cudaGraphInstantiate(&exec, graph, 0));
    if (s->graphs.size() >= 6) {
      cudaGraphExecDestroy(s->graphs.front().exec);
      cudaGraphDestroy(s->graphs.front().graph);
      s->graphs.erase(s->graphs.begin());
    }
    pycfd_solver::GraphEntry e{};
    memcpy(e.key, key, sizeof key);
    e.graph = graph;
    e.exec = exec;
    e.adaptive = 1;
    e.ctl = c;
    s->graphs.push_back(e);
    hit = &s->graphs.back();
  }
  CU(cudaGraphLaunch(hit->exec, sm));
  return 0;
}

int pycfd_history_read(pycfd_solver* s, double* rows, int max_rows, int* n_rows, int* frozen, void* stream) {
  if (!s || !n_rows || !frozen || max_rows < 0) return fail(PCFD_E_ARG, "bad arguments");
  cudaStream_t sm = st(stream);
  CU(cudaMemcpyAsync(s->hI, s->I, sizeof(int) * I_COUNT, cudaMemcpyDeviceToHost, sm));
  CU(cudaStreamSynchronize(sm));
  const int n = s->hI[I_HIST];
  *frozen = s->hI[I_FROZEN];
  if (n > kHistRows) return fail(PCFD_E_ARG, "%d steps since the history was last read; it holds %d", n, kHistRows);
  *n_rows = n;
  const int c = std::min(n, max_rows);
  if (c > 0 && rows && s->hist)
    CU(cudaMemcpyAsync(rows, s->hist, sizeof(double) * kHistCols * c, cudaMemcpyDeviceToHost, sm));
  CU(cudaMemsetAsync(s->I + I_HIST, 0, sizeof(int), sm));
  CU(cudaStreamSynchronize(sm));
  return 0;
}

int pycfd_set_clock(pycfd_solver* s, double t, void* stream) {
  if (!s) return fail(PCFD_E_ARG, "bad arguments");
  k_set_clock<<<1, 32, 0, st(stream)>>>(s->S, s->I, t);
  CHECK_LAUNCH();
  return 0;
}

int pycfd_get_clock(pycfd_solver* s, double* t, double* dt, int* steps, int* health, void* stream) {
  if (!s || !t || !dt || !steps || !health) return fail(PCFD_E_ARG, "bad arguments");
  cudaStream_t sm = st(stream);
  CU(cudaMemcpyAsync(s->hS, s->S, sizeof(double) * S_COUNT, cudaMemcpyDeviceToHost, sm));
  CU(cudaMemcpyAsync(s->hI, s->I, sizeof(int) * I_COUNT, cudaMemcpyDeviceToHost, sm));
  CU(cudaStreamSynchronize(sm));
  *t = s->hS[S_T];
  *dt = s->hS[S_DT];
  *steps = s->hI[I_STEPS];
  *health = s->hI[I_HEALTH];
  return 0;
}

int pycfd_step_host(pycfd_solver* s, const double* u0h, const double* v0h, double* uh, double* vh,
                    double* ph, double dt, double blend, void* stream) {
  if (!s || !u0h || !v0h || !uh || !vh || !ph) return fail(PCFD_E_ARG, "bad arguments");
  cudaStream_t sm = st(stream);
  const long nu = (long)(s->g.nx + 3) * (s->g.ny + 2), nv = (long)(s->g.nx + 2) * (s->g.ny + 3),
             np = (long)(s->g.nx + 2) * (s->g.ny + 2);
  if (!s->hu0) {
    int rc;
    if ((rc = dalloc(s, &s->hu0, nu)) || (rc = dalloc(s, &s->hv0, nv)) || (rc = dalloc(s, &s->hu, nu)) ||
        (rc = dalloc(s, &s->hv, nv)) || (rc = dalloc(s, &s->hp, np)))
      return rc;
  }
  CU(cudaMemcpyAsync(s->hu0, u0h, nu * sizeof(double), cudaMemcpyHostToDevice, sm));
  CU(cudaMemcpyAsync(s->hv0, v0h, nv * sizeof(double), cudaMemcpyHostToDevice, sm));
  // the device buffers are the solver's own, so the recorded step is replayed
  TRY(pycfd_step_graph(s, s->hu0, s->hv0, s->hu, s->hv, s->hp, dt, blend, stream));
  CU(cudaMemcpyAsync(uh, s->hu, nu * sizeof(double), cudaMemcpyDeviceToHost, sm));
  CU(cudaMemcpyAsync(vh, s->hv, nv * sizeof(double), cudaMemcpyDeviceToHost, sm));
  CU(cudaMemcpyAsync(ph, s->hp, np * sizeof(double), cudaMemcpyDeviceToHost, sm));
  CU(cudaStreamSynchronize(sm));
  return 0;
}

long long pycfd_launch_count(void) { return g_launches.load(); }

int pycfd_solve_trace(pycfd_solver* s, int enable, unsigned long long* out, int cap, void* stream) {
  if (!s || (out && cap < 1)) return fail(PCFD_E_ARG, "bad arguments");
  if (!s->persistent) return fail(PCFD_E_UNSUPPORTED, "the solver does not run persistent solves");
  if (enable == 1 && !s->ptrace) TRY(dalloc(s, &s->ptrace, (size_t)kPTraceCap));
  if (enable == 0 || enable == 1) s->trace_on = enable;
  if (out) {
    if (!s->ptrace) return fail(PCFD_E_ARG, "no trace recorded");
    CU(cudaStreamSynchronize(st(stream)));
    CU(cudaMemcpy(out, s->ptrace, sizeof(unsigned long long) * (size_t)std::min(cap, kPTraceCap),
                  cudaMemcpyDeviceToHost));
  }
  return 0;
}

int pycfd_solver_set_wait_limit(pycfd_solver* s, unsigned long long ns) {
  if (!s || ns == 0) return fail(PCFD_E_ARG, "bad arguments");
  if (!s->persistent) return fail(PCFD_E_UNSUPPORTED, "the solver does not run persistent solves");
  s->wait_ns = ns;
  return 0;
}

int pycfd_solver_persistent(pycfd_solver* s, int* ctas) {
  if (!s || !ctas) return fail(PCFD_E_ARG, "bad arguments");
  *ctas = s->persistent;
  return 0;
}

int pycfd_profile_kernel(pycfd_solver* s, int kernel_id) {
  if (!s || kernel_id < 0 || kernel_id > 8) return fail(PCFD_E_ARG, "bad arguments");
  s->prof_id = kernel_id;
  s->prof_n = 0;
  return 0;
}

int pycfd_profile_read(pycfd_solver* s, double* total_ms, int* launches, void* stream) {
  if (!s || !total_ms || !launches) return fail(PCFD_E_ARG, "bad arguments");
  CU(cudaStreamSynchronize(st(stream)));
  double t = 0.0;
  for (int k = 0; k + 1 < s->prof_n; k += 2) {
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, s->prof_ev[k], s->prof_ev[k + 1]));
    t += ms;
  }
  *total_ms = t;
  *launches = s->prof_n / 2;
  s->prof_n = 0;
  return 0;
}

int pycfd_adjoint_apply(int op, const pycfd_adj_args* a, void* stream) {
  if (!a) return fail(PCFD_E_ARG, "bad arguments");
  cudaStream_t sm = st(stream);
  if (op == PCFD_ADJ_LINCOMB) {   // elementwise: no grid
    if (!a->out || !a->a || !a->b || a->count < 0) return fail(PCFD_E_ARG, "lincomb: bad arguments");
    if (a->count > 0) {
      k_adj_lincomb<<<grid_for(a->count, 256), 256, 0, sm>>>(a->out, a->a, a->ca, a->b, a->cb, a->count);
      CHECK_LAUNCH();
    }
    return 0;
  }
  if (a->n < 2 || !(a->h > 0)) return fail(PCFD_E_ARG, "bad arguments");
  const AdjGeo G{a->n, a->h, a->nu};
  const long nf = (long)(a->n + 3) * (a->n + 2) * 2;   // u and v faces
  const int grid = grid_for(nf, 256);
  auto need = [](std::initializer_list<const void*> ps) {
    for (const void* p : ps)
      if (!p) return false;
    return true;
  };
  switch (op) {
    case PCFD_ADJ_PREDICTOR:
      if (!need({a->u, a->v, a->out_u, a->out_v})) return fail(PCFD_E_ARG, "predictor: null array");
      k_adj_predictor<<<grid, 256, 0, sm>>>(G, a->u, a->v, a->out_u, a->out_v, a->dt);
      break;
    case PCFD_ADJ_WALLS:
      if (!need({a->out_u, a->out_v, a->lid})) return fail(PCFD_E_ARG, "walls: null array");
      k_adj_walls<<<1, 512, 0, sm>>>(G, a->out_u, a->out_v, a->lid);
      break;
    case PCFD_ADJ_MASK:
      if (!need({a->u, a->v, a->out_u, a->out_v, a->cu, a->cv})) return fail(PCFD_E_ARG, "mask: null array");
      k_adj_mask<<<grid, 256, 0, sm>>>(G, a->u, a->v, a->out_u, a->out_v, a->cu, a->cv);
      break;
    case PCFD_ADJ_DIV:
      if (!need({a->u, a->v, a->out}) || !(a->dt > 0)) return fail(PCFD_E_ARG, "div: bad arguments");
      k_adj_div<<<grid, 256, 0, sm>>>(G, a->u, a->v, a->out, a->dt);
      break;
    case PCFD_ADJ_CORRECT:
      if (!need({a->out_u, a->out_v, a->a})) return fail(PCFD_E_ARG, "correct: null array");
      k_adj_correct<<<grid, 256, 0, sm>>>(G, a->out_u, a->out_v, a->a, a->dt);
      break;
    case PCFD_ADJ_OBJECTIVE:
      if (!need({a->u, a->v, a->lower, a->out})) return fail(PCFD_E_ARG, "objective: null array");
      k_adj_objective<<<1, 1024, 0, sm>>>(G, a->u, a->v, a->lower, a->out);
      break;
    case PCFD_ADJ_PREDICTOR_T: {
      if (!need({a->u, a->v, a->gu, a->gv, a->out_u, a->out_v})) return fail(PCFD_E_ARG, "predictor_T: null array");
      const AdjRhs R{G, a->u, a->v, a->gu, a->gv, a->dt};
      k_adj_predictor_T<<<grid, 256, 0, sm>>>(R, a->out_u, a->out_v);
      break;
    }
    case PCFD_ADJ_WALLS_T:
      if (!need({a->out_u, a->out_v, a->acc_u})) return fail(PCFD_E_ARG, "walls_T: null array");
      k_adj_walls_T<<<1, 512, 0, sm>>>(G, a->out_u, a->out_v, a->acc_u);
      break;
    case PCFD_ADJ_MASK_T:
      if (!need({a->u, a->v, a->out_u, a->out_v, a->cu, a->cv, a->acc_u, a->acc_v}))
        return fail(PCFD_E_ARG, "mask_T: null array");
      k_adj_mask_T<<<grid, 256, 0, sm>>>(G, a->u, a->v, a->out_u, a->out_v, a->cu, a->cv, a->acc_u, a->acc_v);
      break;
    case PCFD_ADJ_GRAD_T:
      if (!need({a->gu, a->gv, a->out})) return fail(PCFD_E_ARG, "grad_T: null array");
      k_adj_grad_T<<<grid, 256, 0, sm>>>(G, a->gu, a->gv, a->out);
      break;
    case PCFD_ADJ_DIV_T:
      if (!need({a->out_u, a->out_v, a->a})) return fail(PCFD_E_ARG, "div_T: null array");
      k_adj_div_T<<<grid, 256, 0, sm>>>(G, a->out_u, a->out_v, a->a);
      break;
    case PCFD_ADJ_OBJECTIVE_T:
      if (!need({a->u, a->v, a->lower, a->out_u, a->out_v})) return fail(PCFD_E_ARG, "objective_T: null array");
      k_adj_objective_T<<<grid, 256, 0, sm>>>(G, a->u, a->v, a->lower, a->out_u, a->out_v);
      break;
    default: return fail(PCFD_E_ARG, "unknown adjoint op %d", op);
  }
  CHECK_LAUNCH();
  return 0;
}

int pycfd_rasterize(const pycfd_shape* shape, const double* xf, const double* dx_cells, const double* yf,
                    const double* dy_cells, int nx, int ny, double lx, double ly, int subsamples,
                    double* fraction, uint8_t* mask, void* stream) {
  if (!shape || !xf || !dx_cells || !yf || !dy_cells || !fraction || !mask || nx < 1 || ny < 1)
    return fail(PCFD_E_ARG, "bad arguments");
  if (subsamples < 1 || subsamples > 64) return fail(PCFD_E_ARG, "subsamples must be 1..64, got %d", subsamples);
  ShapeDev d{};
  d.kind = shape->kind;
  d.p0 = shape->p[0];
  d.p1 = shape->p[1];
  d.p2 = shape->p[2];
  d.p3 = shape->p[3];
  d.lx = lx;
  d.ly = ly;
  switch (shape->kind) {
    case PCFD_SHAPE_CIRCLE:
    case PCFD_SHAPE_RECTANGLE: break;
    case PCFD_SHAPE_POLYGON:
      if (!shape->verts || shape->n_verts < 3) return fail(PCFD_E_ARG, "a polygon needs at least 3 vertices");
      d.verts = shape->verts;
      d.n_verts = shape->n_verts;
      break;
    case PCFD_SHAPE_IMAGE:
      if (!shape->image || shape->rows < 1 || shape->cols < 1 || !(lx > 0) || !(ly > 0))
        return fail(PCFD_E_ARG, "bad image");
      d.image = shape->image;
      d.rows = shape->rows;
      d.cols = shape->cols;
      d.threshold = shape->threshold;
      d.invert = shape->invert;
      break;
    default: return fail(PCFD_E_ARG, "unknown shape kind %d", shape->kind);
  }
  const long n = (long)nx * ny;
  k_solid_fraction<<<grid_for(n, 256, 148 * 8), 256, 0, st(stream)>>>(d, xf, dx_cells, yf, dy_cells, nx, ny,
                                                                         subsamples, fraction, mask);
  CHECK_LAUNCH();
  return 0;
}

int pycfd_face_lists(pycfd_solver* s, int* u_faces, int u_cap, int* v_faces, int v_cap, int* n_u,
                     int* n_v, int* body_u_start, int* body_v_start, int* n_bodies, int* lohi) {
  if (!s || !n_u || !n_v || u_cap < 0 || v_cap < 0) return fail(PCFD_E_ARG, "bad arguments");
  *n_u = s->bc.n_mask_u;
  *n_v = s->bc.n_mask_v;
  const int cu = std::min(u_cap, s->bc.n_mask_u), cv = std::min(v_cap, s->bc.n_mask_v);
  if (cu > 0 && u_faces) CU(cudaMemcpy(u_faces, s->mask_u, sizeof(int) * cu, cudaMemcpyDeviceToHost));
  if (cv > 0 && v_faces) CU(cudaMemcpy(v_faces, s->mask_v, sizeof(int) * cv, cudaMemcpyDeviceToHost));
  const int nb = s->bc.n_bodies;
  if (n_bodies) *n_bodies = nb;
  for (int b = 0; b <= std::max(nb, 1) && b <= PCFD_MAX_BODIES; ++b) {
    if (body_u_start) body_u_start[b] = s->bc.body_u_start[b];
    if (body_v_start) body_v_start[b] = s->bc.body_v_start[b];
  }
  if (lohi) {
    lohi[0] = s->g.u_lo;
    lohi[1] = s->g.u_hi;
    lohi[2] = s->g.v_lo;
    lohi[3] = s->g.v_hi;
  }
  return 0;
}

int pycfd_get_stats(pycfd_solver* s, pycfd_stats* o, void* stream) {
  if (!s || !o) return fail(PCFD_E_ARG, "bad arguments");
  cudaStream_t sm = st(stream);
  CU(cudaMemcpyAsync(s->hS, s->S, sizeof(double) * S_COUNT, cudaMemcpyDeviceToHost, sm));
  CU(cudaMemcpyAsync(s->hI, s->I, sizeof(int) * I_COUNT, cudaMemcpyDeviceToHost, sm));
  CU(cudaStreamSynchronize(sm));
  memset(o, 0, sizeof *o);
  o->iterations = s->hI[I_IT];
  o->converged = s->hI[I_CONVERGED];
  o->status = s->hI[I_STATUS];
  o->total_iterations = s->hI[I_TOTAL_IT];
  o->last_residual = s->hS[S_RESID];
  o->fx = s->hS[S_FX];
  o->fy = s->hS[S_FY];
  for (int b = 0; b < PCFD_MAX_BODIES; ++b) {
    o->body_fx[b] = s->hS[S_BODY_FX + b];
    o->body_fy[b] = s->hS[S_BODY_FY + b];
  }
  o->ir_iterations = s->hI[I_IR_IT];
  return 0;
}

int pycfd_reduce_fields(pycfd_solver* s, const double* u, const double* v, const double* p, const double* up,
                      const double* vp, pycfd_field_stats* o, void* stream) {
  if (!s || !u || !v || !o) return fail(PCFD_E_ARG, "bad arguments");
  cudaStream_t sm = st(stream);
  pdl_launch(s, k_field_stats, std::min(s->g.nx + 3, kMaxRedBlocks), kRedThreads, 0, sm, u, v, p, up, vp, s->solid, s->g, s->rb(),
                                                                     s->S);
  CHECK_LAUNCH();
  CU(cudaMemcpyAsync(s->hS + S_STAT0, s->S + S_STAT0, 8 * sizeof(double), cudaMemcpyDeviceToHost, sm));
  CU(cudaStreamSynchronize(sm));
  const double* t = s->hS + S_STAT0;
  o->max_u = t[0];
  o->max_v = t[1];
  o->max_du = t[2];
  o->max_dv = t[3];
  o->max_div = t[4];
  o->kinetic_energy = s->g.met ? t[5] : t[5] * (s->g.dx * s->g.dy);
  o->max_vorticity = t[6];
  o->finite = t[7] == 0.0;
  return 0;
}

}  // extern "C"

// ============================================================================
// Field reduction without device allocation
// ============================================================================
// Some hosts cannot call cudaMalloc at the moment they want a reduction: an
// application that hands every byte of device memory to its own allocator, or a
// loop that must not take the device-wide synchronisation an allocation may
// impose.  This entry point serves them.  Its scratch -- one block of scalar slots laid
// out like a solver's (the results land in the statistics slots), one row of 8
// partial sums per thread block and the ticket counter of the grid reduction --
// is the file-scope array below: PCFD_NOALLOC_MAX_ROWS*8 + S_COUNT + 2 doubles
// (about 258 KiB), held by every GPU that loads this library until the process
// exits.  The kernel runs one block per row of the u array, so nx + 3 rows must
// fit: nx <= PCFD_NOALLOC_MAX_ROWS - 3.
static __device__ __align__(256) double g_noalloc_scratch[S_COUNT + PCFD_NOALLOC_MAX_ROWS * 8 + 2];

namespace {
std::mutex g_noalloc_mu;
double* g_noalloc_addr[128] = {};   // device address of the scratch, per device ordinal

// Host code must not use the array's name as a device address (it names a
// host-side stand-in); the address is looked up once per device, with that
// device current, and cached for the life of the process (a cudaDeviceReset
// makes the cached address stale).
int noalloc_scratch(double** out) {
  int dev = 0;
  CU(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) return fail(PCFD_E_ARG, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    CU(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_addr[dev] = static_cast<double*>(p);
  }
  *out = g_noalloc_addr[dev];
  return 0;
}
}  // namespace

extern "C" int pycfd_reduce_fields_noalloc(const double* u, const double* v, const double* p,
                                           const double* u_prev, const double* v_prev,
                                           const uint8_t* solid, int nx, int ny, double dx, double dy,
                                           pycfd_field_stats* o, void* stream) {
  if (!u || !v || !o || nx < 1 || ny < 1 || !(dx > 0) || !(dy > 0))
    return fail(PCFD_E_ARG, "bad arguments");
  if (nx > PCFD_NOALLOC_MAX_ROWS - 3)
    return fail(PCFD_E_ARG,
                "pycfd_reduce_fields_noalloc handles nx <= %d (its static scratch holds %d block rows); "
                "got nx = %d -- use pycfd_reduce_fields for larger grids",
                PCFD_NOALLOC_MAX_ROWS - 3, PCFD_NOALLOC_MAX_ROWS, nx);
  cudaStream_t sm = st(stream);
  double* scr = nullptr;
  TRY(noalloc_scratch(&scr));
  double* partials = scr + S_COUNT;
  unsigned int* counter = reinterpret_cast<unsigned int*>(partials + PCFD_NOALLOC_MAX_ROWS * 8);
  CU(cudaMemsetAsync(counter, 0, sizeof(unsigned int), sm));   // the ticket must start at zero
  Geo g{};
  g.nx = nx;
  g.ny = ny;
  g.dx = dx;
  g.dy = dy;
  k_field_stats<<<nx + 3, kRedThreads, 0, sm>>>(u, v, p, u_prev, v_prev, solid, g, RedBuf{partials, counter}, scr);
  CHECK_LAUNCH();
  double t[8];
  CU(cudaMemcpyAsync(t, scr + S_STAT0, sizeof t, cudaMemcpyDeviceToHost, sm));
  CU(cudaStreamSynchronize(sm));
  o->max_u = t[0];
  o->max_v = t[1];
  o->max_du = t[2];
  o->max_dv = t[3];
  o->max_div = t[4];
  o->kinetic_energy = t[5] * (dx * dy);
  o->max_vorticity = t[6];
  o->finite = t[7] == 0.0;
  return 0;
}

// Batched stepping: compiled in this translation unit (it builds on the
// single-problem solver's records and upload helpers).
#include "batch_runtime.cuh"
