// Batched projection step: many independent problems -- grids of uneven size,
// their own viscosity, boundary conditions, time step and stopping state --
// advance together, and every stage of the step is ONE launch over all of
// them.  A launch's blocks are listed in a block map of (problem, tile)
// entries built on the host, so one grid covers every problem's cells (or
// multigrid rows) without a per-problem launch.  Reductions are per problem
// (partials per tile, the problem's last tile finishes), and the kernels that
// end an iteration also take a launch-wide ticket whose last block decides
// whether ANY problem still iterates -- the condition of the device-side WHILE
// loop of a recorded step.  A problem that has converged, or is frozen (health
// flag, end time reached), skips its blocks.
//
// The per-problem arithmetic is the single-problem path's, expression by
// expression (pycfd/core/solver.py:612-731, pycfd/core/pressure.py:300-327,
// pycfd/core/multigrid.py:424-474); only the reduction trees differ (tile
// partials instead of grid-stride partials), so results agree with a solve of
// the same problem alone to rounding, and with the reference within the
// solver tolerance.
#pragma once
#include "boundary.cuh"
#include "common.cuh"
#include "multigrid.cuh"
#include "poisson.cuh"
#include "stencil.cuh"

namespace pcfd {

constexpr int kBMaxLevels = 12;
constexpr int kBTileJ = 32;      // fine tile width along y (contiguous) = threads along y
constexpr int kBThreadsI = 8;    // threads along x in a fine tile block
constexpr int kBThreads = 256;   // every batched kernel runs 256-thread blocks

// One coarse level (l >= 1) of a hierarchy shared by the problems of one
// structure (same grid, boundary kinds and solid mask).
template <class T>
struct BLevel {
  Ell<T> A, R, P;   // A, R: rows of this level; P: rows of the finer level
  int la, lr, lp;   // lanes per row of each block
  const T* wd;      // weighted inverse diagonal
  int n;
  Ell<T> M;         // fused restriction R (I - A W) from the finer level (rows of this level), optional
  int lm;
};

template <class T>
struct BHier {
  BLevel<T> lv[kBMaxLevels];
  double w0;        // smoother weight of level 0 (matrix-free)
  const T* C;       // coarsest pseudo-inverse, row-major nc x nc
  int nc;
  int nlev;
  const T* tail;    // dense operator of the cycle at and below tail_level (row-major), or null
  int tail_level, tail_n;
  int fused;        // levels 1..tail_level carry their fused restriction M
  int agg2;         // level 1 aggregates 2 x 2 fine cells: shape (ceil(nx/2), ceil(ny/2))
  int sp0, spn;     // this structure's problems: sprobs[sp0 .. sp0 + spn)
};

// Device record of one problem.  T is the storage type of the (inner) CG and
// multigrid vectors: double for the FP64 form, float for the mixed form.
template <class T>
struct BProb {
  Geo g;
  BcTable bc;
  DtControl dtc;
  int hier, nlev, singular;
  int tail;                              // depth closed by the structure's dense operator (0: none)
  int max_steps;                         // the problem stops after this many steps
  int tile_i, tiles_i, tiles_j, tiles;   // fine tiles: tile_i rows x 32 columns
  int chunk_tiles, chunks;               // a block of a fine launch takes a chunk of tiles
  int s_segs, s_items, s_chunks;         // warp strips of the solver kernels (b_strips)
  int vec, v_chunks;                     // vector strips (b_vstrips) in force; their blocks
  int p_chunks;                          // warp-strip chunks of the predictor (ghosted arrays)
  int h_tr, h_tiles_j, h_tiles;          // staged tiles of the level-0 stencil transfers: rows, tiles
  int red_base;                          // first partial row of this problem
  const uint8_t* flags;
  const uint8_t* solid;
  const int* bc_kind;
  double *u, *v, *p;                     // state (in place)
  double *us1, *vs1, *us2, *vs2;         // stage buffers
  double* S;
  int* I;
  unsigned* counter;                     // per-problem reduction ticket
  double *b, *x;                         // FP64 right-hand side and solution (warm start)
  T *xs, *r, *z, *pa, *pb, *q;           // (inner) CG iterate and vectors
  T *lb[kBMaxLevels], *lxa[kBMaxLevels], *lxb[kBMaxLevels], *lres[kBMaxLevels];
  // fine-operator diagonal and weighted inverse per face-flag pattern (F_W..F_N),
  // formed at set-up with fine_diag's operations; Dirichlet edges use fine_diag
  double dtab[16], wtab[16];
  int any_dir;
  // the problem's copy of its structure's hierarchy (read with the record)
  double w0;
  const T* C;                            // coarsest pseudo-inverse, row-major
  BLevel<T> lv[kBMaxLevels];
};

// Launch-wide state of a batch (device pointers).
struct BShared {
  double* partials;      // per problem: tiles x 8 doubles, from red_base
  unsigned* tickets;     // launch-wide tickets, one per deciding launch site
  int* any;              // last "some problem still iterates" per site (host-driven loops)
  long long* passes;     // per site: how often it let its loop body run (launch accounting)
  unsigned* iters;       // per site: passes of the loop now running (the cap below)
  int* capped;           // per site: set when a loop was ended by its pass cap
  unsigned* cap_set;     // per site: pass cap set by the host (0: the loop's own cap)
  // Per-problem flags indexed by problem, mirrored from the scalar block by the
  // kernels that change them: a block learns whether its problem takes part
  // from one load beside its map entry instead of a chain through the record.
  uint8_t* frozen;       // I_FROZEN != 0
  uint8_t* solving;      // not frozen and the current solve not done
};

enum BTicket { TK_CG = 0, TK_IR = 1, TK_ARM = 2, TK_COUNT = 4 };

// Blocks of problem P in a launch of the FP32 solver kernels (vector or scalar strips).
template <class T>
__device__ __forceinline__ int b_nchunks(const BProb<T>& P) { return P.vec ? P.v_chunks : P.s_chunks; }

__device__ __forceinline__ bool b_frozen(const BShared& sh, int p) { return sh.frozen[p] != 0; }
__device__ __forceinline__ bool b_solving(const BShared& sh, int p) { return sh.solving[p] != 0; }

// Per-problem reduction over the tiles of one launch.  Every block of the
// problem contributes NV values at row `tile`; the last to arrive combines them
// in tile order and calls fin(totals) on its thread 0.  No early return, so a
// launch-wide ticket may follow.
template <int NV, unsigned MAXMASK = 0u, class Fin>
__device__ __forceinline__ void b_reduce(double (&v)[NV], double* partials, unsigned* counter,
                                         int tile, int ntiles, Fin fin) {
  block_reduce<NV, MAXMASK>(v);
  __shared__ bool last;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  const int nthr = blockDim.x * blockDim.y;
  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) partials[(long)tile * NV + k] = v[k];
    __threadfence();
    const unsigned t = atomicAdd(counter, 1u);
    last = (t == (unsigned)ntiles - 1);
  }
  __syncthreads();
  if (last) {
    __threadfence();
    double acc[NV];
    sum_partials<NV, MAXMASK>(partials, ntiles, tid, nthr, acc);
    block_reduce<NV, MAXMASK>(acc);
    if (tid == 0) {
      fin(acc);
      *counter = 0u;
    }
  }
}

// Launch-wide ticket: every block of the launch calls this last; the final
// block sets the loop condition to "some unfrozen problem has flag `slot`
// still 0", mirrors it into the site's `any` and rearms the ticket.  The
// launch that opens a loop passes reset = 1; every later one counts a pass,
// and at `cap` passes (or the host's sh.cap_set[site] when nonzero) the loop
// ends whatever the flags say (each problem's own iteration limit ends it
// first; the cap only bounds the device loop) and sh.capped[site] is set.
template <class T>
__device__ void b_loop_ticket(const BProb<T>* __restrict__ probs, int nprob, const BShared& sh,
                              int site, int slot, int reset, int cap, LoopCtl loop) {
  unsigned* ticket = sh.tickets + site;
  __shared__ bool lastg;
  __syncthreads();
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  const int nthr = blockDim.x * blockDim.y;
  const unsigned nblk = gridDim.x * gridDim.y;
  if (tid == 0) {
    __threadfence();
    const unsigned t = atomicAdd(ticket, 1u);
    lastg = (t == nblk - 1);
  }
  __syncthreads();
  if (!lastg) return;
  __threadfence();
  int any = 0;
  for (int p = tid; p < nprob; p += nthr) {
    const volatile int* I = probs[p].I;
    if (I[I_FROZEN] == 0 && I[slot] == 0) any = 1;
  }
  any = __syncthreads_or(any);
  if (tid == 0) {
    const unsigned it = reset ? 0u : sh.iters[site] + 1u;
    sh.iters[site] = it;
    const unsigned cs = sh.cap_set[site];
    if (any && it >= (cs ? cs : (unsigned)cap)) {
      any = 0;
      sh.capped[site] = 1;
    }
    sh.any[site] = any;
    loop.set(any != 0);
    *ticket = 0u;
    if (any) sh.passes[site] += 1;
  }
}

// ---- iteration over a fine tile -------------------------------------------
// Block (32 x 8 threads) over the cells of one tile: rows [i0, i0+tile_i) of x,
// 32 columns of y.  B_TILE_CELLS visits interior cells (i < nx, j < ny);
// B_TILE_EXT visits a ghosted array of extent EI x EJ, the last tile row and
// column stretching to the array's edge.
#define B_TILE_CELLS(P, tile)                                                               \
  const int ti_ = (tile) / (P).tiles_j, tj_ = (tile) - ti_ * (P).tiles_j;                   \
  const int i1_ = min((ti_ + 1) * (P).tile_i, (P).g.nx);                                    \
  const int j = tj_ * kBTileJ + (int)threadIdx.x;                                           \
  if (j < (P).g.ny)                                                                         \
    for (int i = ti_ * (P).tile_i + (int)threadIdx.y; i < i1_; i += kBThreadsI)

#define B_TILE_EXT(P, tile, EI, EJ)                                                         \
  const int ti_ = (tile) / (P).tiles_j, tj_ = (tile) - ti_ * (P).tiles_j;                   \
  const int i1_ = (ti_ == (P).tiles_i - 1) ? (EI) : (ti_ + 1) * (P).tile_i;                  \
  const int j1_ = (tj_ == (P).tiles_j - 1) ? (EJ) : (tj_ + 1) * kBTileJ;                     \
  for (int i = ti_ * (P).tile_i + (int)threadIdx.y; i < i1_; i += kBThreadsI)                \
    for (int j = tj_ * kBTileJ + (int)threadIdx.x; j < j1_; j += kBTileJ)

// The tiles of chunk `chunk` of problem P (one block of a fine launch takes a
// chunk, so the per-block set-up -- map entry, record, flags -- is paid once
// for several tiles).
#define B_CHUNK_TILES(P, chunk)                                                             \
  for (int tile_ = (chunk) * (P).chunk_tiles, tend_ = min((P).tiles, tile_ + (P).chunk_tiles); \
       tile_ < tend_; ++tile_)

// Stage arrays: 0 the state, 1 the first stage buffer, 2 the second.
template <class T>
__device__ __forceinline__ double* b_arr_u(const BProb<T>& P, int code) {
  return code == 0 ? P.u : code == 1 ? P.us1 : P.us2;
}
template <class T>
__device__ __forceinline__ double* b_arr_v(const BProb<T>& P, int code) {
  return code == 0 ? P.v : code == 1 ? P.vs1 : P.vs2;
}

// Diagonal and weighted inverse diagonal of the fine operator at a cell: the
// set-up table (the same subtractions as fine_diag, in its order, so the same
// value), or fine_diag itself on an edge cell of a problem with Dirichlet walls.
template <class T>
__device__ __forceinline__ double b_diag(const BProb<T>& P, uint8_t f, int i, int j) {
  if (!(f & F_SOLV)) return 1.0;
  if (P.any_dir && (i == 0 || j == 0 || i == P.g.nx - 1 || j == P.g.ny - 1)) return fine_diag(f, i, j, P.g);
  return P.dtab[f & 15];
}
template <class T>
__device__ __forceinline__ double b_wdinv(const BProb<T>& P, uint8_t f, int i, int j) {
  if (!(f & F_SOLV)) return P.w0 * (1.0 / 1.0);
  if (P.any_dir && (i == 0 || j == 0 || i == P.g.nx - 1 || j == P.g.ny - 1))
    return P.w0 * (1.0 / fine_diag(f, i, j, P.g));
  return P.wtab[f & 15];
}

// (A x)_c in arithmetic type A: fine_apply's terms in its order, the diagonal
// from the table.  A = double for the FP64 kernels; the mixed form's inner
// solve uses A = float (FP32 accumulation, dot products stay FP64).
template <class A, class T, class X>
__device__ __forceinline__ A b_apply(const BProb<T>& P, uint8_t f, int i, int j, int c, X x) {
  const Geo& g = P.g;
  A acc = (A)b_diag(P, f, i, j) * x(c, i, j);
  if (f & F_W) { const int a = wrap_w(i, g); acc += (A)g.cx * x(a * g.ny + j, a, j); }
  if (f & F_E) { const int a = wrap_e(i, g); acc += (A)g.cx * x(a * g.ny + j, a, j); }
  if (f & F_S) { const int b = wrap_s(j, g); acc += (A)g.cy * x(i * g.ny + b, i, b); }
  if (f & F_N) { const int b = wrap_n(j, g); acc += (A)g.cy * x(i * g.ny + b, i, b); }
  return acc;
}

// A block's copy of what a fine cell loop reads from its problem's record: the
// geometry and strip shape in registers, the diagonal tables in shared memory.
// The record lives in global memory, and a loop that stores to the problem's
// vectors cannot keep record fields in registers by itself (the stores might
// alias it), so without the copy every cell would reload them.
struct BView {
  Geo g;
  int any_dir;
  double w0;
  const double* dtab;
  const double* wtab;
  int segs, items;   // warp strips: 32-column segments per row, strips x segments
  // FP32 copies for the vector strips, indexed by the flag's low five bits (a
  // cell without F_SOLV reads 1 and w0): the values (float)b_diag and
  // (float)b_wdinv give away from Dirichlet edges
  const float* df;
  const float* wf;
  float cxf, cyf;
};

// Declares `V` for problem record P; every thread of the block must reach it.
#define B_VIEW(V, P)                                                                           \
  __shared__ double V##_dt[16], V##_wt[16];                                                    \
  __shared__ float V##_df[32], V##_wf[32];                                                     \
  if (threadIdx.x < 16) {                                                                      \
    V##_dt[threadIdx.x] = (P).dtab[threadIdx.x];                                               \
    V##_wt[threadIdx.x] = (P).wtab[threadIdx.x];                                               \
  }                                                                                            \
  if (threadIdx.x < 32) {                                                                      \
    const bool sv_ = (threadIdx.x & F_SOLV) != 0;                                              \
    V##_df[threadIdx.x] = sv_ ? (float)(P).dtab[threadIdx.x & 15] : 1.0f;                      \
    V##_wf[threadIdx.x] = sv_ ? (float)(P).wtab[threadIdx.x & 15] : (float)((P).w0 * (1.0 / 1.0)); \
  }                                                                                            \
  __syncthreads();                                                                             \
  const BView V{(P).g, (P).any_dir, (P).w0, V##_dt, V##_wt, (P).s_segs, (P).s_items,          \
                V##_df, V##_wf, (float)(P).g.cx, (float)(P).g.cy}

__device__ __forceinline__ double b_diag(const BView& V, uint8_t f, int i, int j) {
  if (!(f & F_SOLV)) return 1.0;
  if (V.any_dir && (i == 0 || j == 0 || i == V.g.nx - 1 || j == V.g.ny - 1)) return fine_diag(f, i, j, V.g);
  return V.dtab[f & 15];
}
__device__ __forceinline__ double b_wdinv(const BView& V, uint8_t f, int i, int j) {
  if (!(f & F_SOLV)) return V.w0 * (1.0 / 1.0);
  if (V.any_dir && (i == 0 || j == 0 || i == V.g.nx - 1 || j == V.g.ny - 1))
    return V.w0 * (1.0 / fine_diag(f, i, j, V.g));
  return V.wtab[f & 15];
}
// (float)b_diag and (float)b_wdinv from the block's FP32 tables (one 32-bit
// shared load, no conversion, away from Dirichlet edges).
__device__ __forceinline__ float b_diag_f(const BView& V, uint8_t f, int i, int j) {
  if (V.any_dir && (f & F_SOLV) && (i == 0 || j == 0 || i == V.g.nx - 1 || j == V.g.ny - 1))
    return (float)fine_diag(f, i, j, V.g);
  return V.df[f & 31];
}
__device__ __forceinline__ float b_wdinv_f(const BView& V, uint8_t f, int i, int j) {
  if (V.any_dir && (f & F_SOLV) && (i == 0 || j == 0 || i == V.g.nx - 1 || j == V.g.ny - 1))
    return (float)(V.w0 * (1.0 / fine_diag(f, i, j, V.g)));
  return V.wf[f & 31];
}

// (A x) at a cell from its value and its four neighbours' values, fine_apply's
// terms in its order (diagonal, west, east, south, north), in arithmetic type A.
template <class A, class T>
__device__ __forceinline__ A b_apply5(const BView& V, uint8_t f, int i, int j, T c, T w, T e, T s, T n) {
  A acc = (A)b_diag(V, f, i, j) * (A)c;
  if (f & F_W) acc += (A)V.g.cx * (A)w;
  if (f & F_E) acc += (A)V.g.cx * (A)e;
  if (f & F_S) acc += (A)V.g.cy * (A)s;
  if (f & F_N) acc += (A)V.g.cy * (A)n;
  return acc;
}
// b_apply5<float> from the FP32 tables: the same value.
__device__ __forceinline__ float b_apply5f(const BView& V, uint8_t f, int i, int j, float c, float w, float e,
                                           float s, float n) {
  float acc = b_diag_f(V, f, i, j) * c;
  if (f & F_W) acc += V.cxf * w;
  if (f & F_E) acc += V.cxf * e;
  if (f & F_S) acc += V.cyf * s;
  if (f & F_N) acc += V.cyf * n;
  return acc;
}

// ---- warp strips -----------------------------------------------------------------
// The fine-level solver kernels (CG direction and operator, CG update, the
// level-0 multigrid sweeps) walk a problem's cells in warp strips: a warp takes
// one segment of y (lane = column, so each row of a vector is one coalesced
// access of 32 values) over kBStripRows rows of x.  The stencil operand of the
// strip and its two halo rows go to registers first, with every per-cell load
// of the strip, before any arithmetic; the y-neighbours then come from the
// adjacent lanes by shuffle.  The columns just west and east of the segment are
// lanes 0 and 31 themselves (a segment is the 30 columns of lanes 1..30): each
// lane forms one operand value per row, and no load sits under a lane-dependent
// branch.  (The alternative kept behind PCFD_BSTRIP_HALO_LANES=0, 32-column
// segments whose lanes all form the two edge columns' values as well, issues
// three operand loads per row instead of one.)  Off-grid rows and columns are
// read at a clamped (valid) index and the value dropped.
// No shared-memory staging and no block barrier until the block's reduction.
// A block (8 warps) takes kBStripItems consecutive (strip, segment) items of one
// problem, adjacent segments of the same rows first.
#ifndef PCFD_BSTRIP_ROWS
#define PCFD_BSTRIP_ROWS 8
#endif
constexpr int kBStripRows = PCFD_BSTRIP_ROWS;
#ifndef PCFD_BSTRIP_ITEMS
#define PCFD_BSTRIP_ITEMS 16
#endif
constexpr int kBStripItems = PCFD_BSTRIP_ITEMS;   // strips of kBStripRows rows per chunk (block)
// Halo lanes: 1 = a segment is 30 columns, lanes 1..30, and lanes 0 and 31 hold
// the columns just west and east of it (each lane forms one operand value per
// row); 0 = a segment is 32 columns and every lane also forms the two edge
// columns' values (three operand values per row).
#ifndef PCFD_BSTRIP_HALO_LANES
#define PCFD_BSTRIP_HALO_LANES 1
#endif
constexpr int kBSegCols = PCFD_BSTRIP_HALO_LANES ? 30 : 32;   // output columns per warp segment
static_assert(kBStripRows % 2 == 0, "the FP64-operand kernels take half-height strips");
// Strip height of a kernel whose per-cell values are of type T: FP64 values take
// twice the registers, so their kernels walk half-height strips.
template <class T>
__host__ __device__ constexpr int b_rs() { return sizeof(T) == 8 ? kBStripRows / 2 : kBStripRows; }
// Resident blocks per SM the strip kernels are compiled for (register bound
// 65536 / (256 x this)).  These kernels are latency-bound, and more resident
// blocks overlap one block's loads with another's reduction: on the 256-cavity
// batch, 2 blocks per SM (the compiler's own 128 registers) step in 27.1 ms,
// 4 blocks per SM (64 registers, small spills) in 26.5 ms with the coarse-level
// kernels unchanged.
#ifndef PCFD_BSTRIP_MINB
#define PCFD_BSTRIP_MINB 4
#endif
#define B_STRIP_KERNEL __global__ void __launch_bounds__(kBThreads, PCFD_BSTRIP_MINB)

// op(k, i, j): the operand at cell (i, j), k = i*ny + j (issues its loads; k is
// always a valid cell).  load(u, c): the per-cell loads of body row u (c valid;
// the values unused past the grid).  body(u, c, i, j, centre, west, east,
// south, north).  STENCIL = false: no operand (pointwise kernels); body gets
// zeros.
// RS: the strip height of the calling kernel (kBStripRows or a divisor of it).
// A chunk covers the same cells whatever RS is: kBStripItems strips of
// kBStripRows rows, that is kBStripItems * kBStripRows / RS strips of RS rows.
template <bool STENCIL, class T, int RS, class Op, class Load, class Body>
__device__ __forceinline__ void b_strips(const BView& V, int chunk, Op op, Load load, Body body) {
  static_assert(kBStripRows % RS == 0, "strip height must divide kBStripRows");
  constexpr int IPC = kBStripItems * (kBStripRows / RS);
  // pointwise kernels take aligned 32-column segments (no halo to hold); their
  // items then end no later than the stencil kernels' and fit the same chunks
  constexpr bool HALO = PCFD_BSTRIP_HALO_LANES && STENCIL;
  const int lane = (int)(threadIdx.x & 31), warp = (int)(threadIdx.x >> 5);
  const int nx = V.g.nx, ny = V.g.ny;
  const int segs = HALO ? V.segs : (ny + 31) / 32;
  const int items = segs * ((nx + RS - 1) / RS);
  const int it1 = min(items, (chunk + 1) * IPC);
  for (int it = chunk * IPC + warp; it < it1; it += kBThreads / 32) {
    const int strip = it / segs, seg = it - strip * segs;
    const int i0 = strip * RS;
    int j, jc;      // this lane's column and the (valid) column its loads use
    bool jv;        // the lane's cell is one of the segment's
    int jh = -1;    // HALO: the operand's column (wrapped), -1 off the grid
    int last = 31;  // !HALO: the segment's last valid lane
    if constexpr (HALO) {
      j = seg * kBSegCols - 1 + lane;   // lanes 0 and 31: the columns beside the segment
      jh = j;
      if (jh < 0) jh = V.g.periodic_y ? jh + ny : -1;
      else if (jh >= ny) jh = (V.g.periodic_y && jh == ny) ? 0 : -1;
      jc = jh >= 0 ? jh : (j < 0 ? 0 : ny - 1);
      jv = lane >= 1 && lane <= 30 && j < ny;
    } else {
      const int j0 = seg * 32;
      j = j0 + lane;
      jv = j < ny;
      jc = jv ? j : ny - 1;
      last = min(31, ny - 1 - j0);
    }
    T ov[STENCIL ? RS + 2 : 1];
    T ew[STENCIL && !HALO ? RS : 1], ee[STENCIL && !HALO ? RS : 1];
    if (STENCIL) {
#pragma unroll
      for (int u = 0; u < RS + 2; ++u) {
        const int r = strip_row(i0 - 1 + u, nx, V.g.periodic_x);
        const int rc = r >= 0 ? r : 0;
        const T val = op(rc * ny + jc, rc, jc);
        ov[u] = ((HALO ? jh >= 0 : jv) && r >= 0) ? val : (T)0;
      }
      if constexpr (!HALO) {
        int jw, je;
        strip_edges(seg * 32, last, ny, V.g.periodic_y, &jw, &je);
        const int jwc = jw >= 0 ? jw : 0, jec = je >= 0 ? je : 0;
#pragma unroll
        for (int u = 0; u < RS; ++u) {
          const int i = i0 + u, ic = i < nx ? i : nx - 1;
          const T vw = op(ic * ny + jwc, ic, jwc), ve = op(ic * ny + jec, ic, jec);
          ew[u] = (jw >= 0 && i < nx) ? vw : (T)0;
          ee[u] = (je >= 0 && i < nx) ? ve : (T)0;
        }
      }
    }
#pragma unroll
    for (int u = 0; u < RS; ++u) {
      const int i = i0 + u, ic = i < nx ? i : nx - 1;
      load(u, ic * ny + jc);
    }
#pragma unroll
    for (int u = 0; u < RS; ++u) {
      T c = (T)0, w = (T)0, e = (T)0, sv = (T)0, nv = (T)0;
      if (STENCIL) {
        c = ov[u + 1];
        w = ov[u];
        e = ov[u + 2];
        sv = __shfl_up_sync(0xffffffffu, c, 1);
        nv = __shfl_down_sync(0xffffffffu, c, 1);
        if constexpr (!HALO) {
          if (lane == 0) sv = ew[u];
          if (lane == last) nv = ee[u];
        }
      }
      const int i = i0 + u;
      if (jv && i < nx) body(u, i * ny + j, i, j, c, w, e, sv, nv);
    }
  }
}

// ---- vector strips (FP32 vectors, ny a multiple of 4) ------------------------------
// The FP32 kernels of the mixed form's inner solve walk a problem in vector
// strips when its rows are a multiple of 4 long: a lane holds four adjacent
// columns of y as one 16-byte float4 (every row starts 16-byte aligned), so a
// warp covers a 128-column segment of a row with ONE load instruction per array
// (the flags as one 32-bit word), against one per cell in the scalar strips,
// and the index arithmetic, clamps and per-row bookkeeping are paid once per
// four cells.  The operand's y-neighbours are the neighbouring elements, across
// lanes by shuffle; the two columns beside the segment come from one scalar
// operand value per row: lane 0 forms the column west of the segment, lane 31
// the one east of it (on a segment narrower than 128 columns, the first lane
// past the grid forms it and passes it down by the same shuffle).  A block
// takes kBVecRows rows of its problem, all segments.  Per cell the arithmetic
// is the scalar strips' (the same operand, stencil and update); only the order
// of the per-problem sums differs.
#ifndef PCFD_BVEC_ROWS
#define PCFD_BVEC_ROWS 32
#endif
constexpr int kBVecRows = PCFD_BVEC_ROWS;   // rows of one block of a vector-strip launch
constexpr int kBVecCols = 128;              // columns of a warp segment (32 lanes x float4)

__device__ __forceinline__ float4 b_ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void b_st4(float* p, const float (&v)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ uint32_t b_ldf4(const uint8_t* p) { return *reinterpret_cast<const uint32_t*>(p); }
__device__ __forceinline__ uint8_t b_fl(uint32_t w, int e) { return (uint8_t)(w >> (8 * e)); }
__device__ __forceinline__ float b_el(const float4& a, int e) {
  return e == 0 ? a.x : e == 1 ? a.y : e == 2 ? a.z : a.w;
}

// op4(k, i, j): the operand at cells k..k+3 of row i (k = i*ny + j, j a multiple
// of 4; issues its loads).  op1(k, i, j): the operand at one cell (the segment's
// edge columns).  load(u, k): the per-cell loads of body row u.  body(u, k, i,
// j, c, w, e, s, n): the four cells k..k+3 of row i, each argument a float[4]
// (centre, i-1, i+1, j-1, j+1).  STENCIL = false: no operand, no edges (the
// arguments are zeros).  RS: rows per warp item, a divisor of kBVecRows.
template <bool STENCIL, int RS, class Op4, class Op1, class Load, class Body>
__device__ __forceinline__ void b_vstrips(const BView& V, int chunk, Op4 op4, Op1 op1, Load load, Body body) {
  static_assert(kBVecRows % RS == 0, "rows per item must divide the block's rows");
  const int lane = (int)(threadIdx.x & 31), warp = (int)(threadIdx.x >> 5);
  const int nx = V.g.nx, ny = V.g.ny;
  const int segs = (ny + kBVecCols - 1) / kBVecCols;
  const int r0 = chunk * kBVecRows;
  const int items = segs * ((min(nx - r0, kBVecRows) + RS - 1) / RS);
  for (int it = warp; it < items; it += kBThreads / 32) {
    const int strip = it / segs, seg = it - strip * segs;
    const int i0 = r0 + strip * RS;
    const int j0 = seg * kBVecCols;
    const int nl = min(32, (ny - j0) >> 2);   // lanes over columns of the grid
    const int j = j0 + 4 * lane;
    const bool jv = lane < nl;
    const int jc = jv ? j : j0;               // an aligned valid column for the loads
    float ov[STENCIL ? RS + 2 : 1][4];
    float eg[STENCIL ? RS : 1];
    if constexpr (STENCIL) {
      // the edge column this lane forms: west of the segment (lane 0), east of it
      // (lane 31 on a full segment, else the first lane past the grid); -1 none
      const int le = nl < 32 ? nl : 31;
      int jh = -1;
      if (lane == 0) jh = j0 > 0 ? j0 - 1 : (V.g.periodic_y ? ny - 1 : -1);
      else if (lane == le) jh = j0 + 4 * nl < ny ? j0 + 4 * nl : (V.g.periodic_y ? 0 : -1);
      const int jhc = jh >= 0 ? jh : j0;
#pragma unroll
      for (int u = 0; u < RS + 2; ++u) {
        const int r = strip_row(i0 - 1 + u, nx, V.g.periodic_x);
        const int rc = r >= 0 ? r : 0;
        const float4 a = op4(rc * ny + jc, rc, jc);
        const bool ok = jv && r >= 0;
        ov[u][0] = ok ? a.x : 0.f;
        ov[u][1] = ok ? a.y : 0.f;
        ov[u][2] = ok ? a.z : 0.f;
        ov[u][3] = ok ? a.w : 0.f;
      }
#pragma unroll
      for (int u = 0; u < RS; ++u) {
        const int i = i0 + u, ic = i < nx ? i : nx - 1;
        const float h = op1(ic * ny + jhc, ic, jhc);
        eg[u] = (jh >= 0 && i < nx) ? h : 0.f;
      }
    }
#pragma unroll
    for (int u = 0; u < RS; ++u) {
      const int i = i0 + u, ic = i < nx ? i : nx - 1;
      load(u, ic * ny + jc);
    }
#pragma unroll
    for (int u = 0; u < RS; ++u) {
      float c[4] = {0.f, 0.f, 0.f, 0.f}, w[4] = {0.f, 0.f, 0.f, 0.f}, e[4] = {0.f, 0.f, 0.f, 0.f};
      float s[4] = {0.f, 0.f, 0.f, 0.f}, n[4] = {0.f, 0.f, 0.f, 0.f};
      if constexpr (STENCIL) {
        // j-1 of element 0 and j+1 of element 3 from the adjacent lanes (the
        // first lane past the grid carries the east edge in its element 0)
        const float up = __shfl_up_sync(0xffffffffu, ov[u + 1][3], 1);
        const float x0 = (nl < 32 && lane == nl) ? eg[u] : ov[u + 1][0];
        const float dn = __shfl_down_sync(0xffffffffu, x0, 1);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          c[q] = ov[u + 1][q];
          w[q] = ov[u][q];
          e[q] = ov[u + 2][q];
        }
        s[0] = lane == 0 ? eg[u] : up;
        s[1] = c[0];
        s[2] = c[1];
        s[3] = c[2];
        n[0] = c[1];
        n[1] = c[2];
        n[2] = c[3];
        n[3] = lane == 31 ? eg[u] : dn;
      }
      const int i = i0 + u;
      if (jv && i < nx) body(u, i * ny + j, i, j, c, w, e, s, n);
    }
  }
}

// ---- step bookkeeping -------------------------------------------------------
// max|u|, max|v| over the physical faces and the non-finite count of u, v, p:
// the inputs of the time-step control (pycfd/core/timestepper.py:94-142).
template <class T>
__global__ void __launch_bounds__(kBThreads) k_b_stats(const BProb<T>* __restrict__ probs,
                                                        const int2* __restrict__ map, BShared sh) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (b_frozen(sh, e.x)) return;
  const int nx = P.g.nx, ny = P.g.ny;
  const long W = ny + 2, WV = ny + 3;
  const double *u = P.u, *v = P.v, *p = P.p;
  double acc[3] = {0, 0, 0};
  {
    B_CHUNK_TILES(P, e.y) {
      B_TILE_EXT(P, tile_, nx + 3, ny + 3) {
        if (j < ny + 2) {
          const double a = u[(long)i * W + j];
          if (!isfinite(a)) acc[2] += 1.0;
          if (i >= 1 && i <= nx + 1 && j >= 1 && j <= ny) acc[0] = fmax(acc[0], fabs(a));
        }
        if (i < nx + 2) {
          const double a = v[(long)i * WV + j];
          if (!isfinite(a)) acc[2] += 1.0;
          if (i >= 1 && i <= nx && j >= 1 && j <= ny + 1) acc[1] = fmax(acc[1], fabs(a));
          if (j < ny + 2 && !isfinite(p[(long)i * W + j])) acc[2] += 1.0;
        }
      }
    }
  }
  b_reduce<3, 0x3u>(acc, sh.partials + (long)P.red_base * 8, P.counter, e.y, P.chunks, [&](double* t) {
    P.S[S_STAT0] = t[0];
    P.S[S_STAT0 + 1] = t[1];
    P.S[S_STAT0 + 7] = t[2];
  });
}

// Per-problem time step (one thread per problem): the single-problem control;
// a problem whose health flags trip, or whose end time or step count is
// reached, freezes.
template <class T>
__global__ void k_b_dt(const BProb<T>* __restrict__ probs, int nprob, BShared sh) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nprob) return;
  const BProb<T>& P = probs[k];
  if (P.I[I_FROZEN]) return;
  if (P.dtc.t_end - P.S[S_T] <= 0.0 || P.I[I_STEPS] >= P.max_steps) {
    P.I[I_FROZEN] = 2;
    sh.frozen[k] = 1;
    sh.solving[k] = 0;
    return;
  }
  adaptive_dt_update(P.S, P.I, P.dtc);
  if (P.I[I_HEALTH] != 0) {   // the step is not taken: state stays at the last good step
    P.I[I_FROZEN] = 1;
    sh.frozen[k] = 1;
    sh.solving[k] = 0;
    P.S[S_T] -= P.S[S_DT];
    P.I[I_STEPS] -= 1;
  }
}

// Fixed step parameters (initial projection: dt = 1; fixed-dt runs).
template <class T>
__global__ void k_b_set_dt(const BProb<T>* __restrict__ probs, int nprob, double dt) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nprob) return;
  const BProb<T>& P = probs[k];
  if (P.I[I_FROZEN]) return;
  P.S[S_DT] = dt;
  P.S[S_BLEND] = 0.0;
  P.I[I_TOTAL_IT] = 0;
}

// ---- stencils ----------------------------------------------------------------
// Predictor of one Runge-Kutta stage: out = U + dt*rhs on the solvable faces,
// U elsewhere, U = ca*a + cb*b (b absent: U = a) (pycfd/core/solver.py:619-622).
// Warp strips over the ghosted arrays: a warp loads 32 adjacent columns of
// kBStripRows + 2 rows of u and of v (the stage input formed on the fly) into
// registers and writes the 30 inner columns -- the outer two lanes only carry
// the halo, so every neighbour comes from a register or a shuffle.  The RHS is
// rhs_u_core / rhs_v_core, the single-problem predictor's arithmetic.
constexpr int kBPredCols = 30;   // output columns per warp segment (32 lanes, one halo lane each side)

template <class T>
B_STRIP_KERNEL k_b_predictor(const BProb<T>* __restrict__ probs,
                                                            const int2* __restrict__ map, int src_a,
                                                            int src_b, double ca, double cb, int dst,
                                                            BShared sh) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  constexpr int RS = kBStripRows;
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (b_frozen(sh, e.x)) return;
  const Geo g = P.g;
  const int nx = g.nx, ny = g.ny;
  const long W = ny + 2, WV = ny + 3;
  const StageIn u{b_arr_u(P, src_a), src_b >= 0 ? b_arr_u(P, src_b) : nullptr, ca, cb};
  const StageIn v{b_arr_v(P, src_a), src_b >= 0 ? b_arr_v(P, src_b) : nullptr, ca, cb};
  double* __restrict__ us = b_arr_u(P, dst);
  double* __restrict__ vs = b_arr_v(P, dst);
  const double dt = P.S[S_DT], blend = P.S[S_BLEND];
  const int lane = (int)(threadIdx.x & 31), warp = (int)(threadIdx.x >> 5);
  const int segs = (ny + 3 + kBPredCols - 1) / kBPredCols;
  const int items = segs * ((nx + 3 + RS - 1) / RS);
  const int it1 = min(items, (e.y + 1) * kBStripItems);
  for (int it = e.y * kBStripItems + warp; it < it1; it += kBThreads / 32) {
    const int strip = it / segs, seg = it - strip * segs;
    const int i0 = strip * RS, j = seg * kBPredCols - 1 + lane;
    const bool ju = j >= 0 && j < ny + 2, jv = j >= 0 && j < ny + 3;
    double U[RS + 2], V[RS + 2];
#pragma unroll
    for (int r = 0; r < RS + 2; ++r) {
      const int row = i0 - 1 + r;
      U[r] = (ju && row >= 0 && row < nx + 3) ? u[(long)row * W + j] : 0.0;
      V[r] = (jv && row >= 0 && row < nx + 2) ? v[(long)row * WV + j] : 0.0;
    }
    const bool out = lane >= 1 && lane <= kBPredCols;
#pragma unroll
    for (int q = 0; q < RS; ++q) {
      const int m = i0 + q;
      const double un = __shfl_down_sync(0xffffffffu, U[q + 1], 1);
      const double usv = __shfl_up_sync(0xffffffffu, U[q + 1], 1);
      const double us2 = __shfl_up_sync(0xffffffffu, U[q + 2], 1);
      const double vn0 = __shfl_down_sync(0xffffffffu, V[q], 1);
      const double vn1 = __shfl_down_sync(0xffffffffu, V[q + 1], 1);
      const double vsv = __shfl_up_sync(0xffffffffu, V[q + 1], 1);
      if (out && ju && m < nx + 3) {
        double val = U[q + 1];
        if (m >= g.u_lo && m < g.u_hi && j >= 1 && j <= ny)
          val = val + rmul(dt, rhs_u_core(U[q + 1], U[q + 2], U[q], un, usv, vn0, vn1, V[q], V[q + 1], g.dx,
                                          g.dy, g.nu, blend, g.fx));
        us[(long)m * W + j] = val;
      }
      if (out && jv && m < nx + 2) {
        double val = V[q + 1];
        if (m >= 1 && m <= nx && j >= g.v_lo && j < g.v_hi)
          val = val + rmul(dt, rhs_v_core(V[q + 1], vn1, vsv, V[q + 2], V[q], us2, U[q + 2], usv, U[q + 1],
                                          g.dx, g.dy, g.nu, blend, g.fy));
        vs[(long)m * WV + j] = val;
      }
    }
  }
}

// Boundary program of every problem, one block each; p_ghosts first rebuilds
// the ghost ring of p from the solution x (the single-problem path does this
// in the correction's last block).
template <class T>
__global__ void __launch_bounds__(kBThreads) k_b_boundary(const BProb<T>* __restrict__ probs, int arr,
                                                           BcProgram prog, int p_ghosts, BShared sh) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  const BProb<T>& P = probs[blockIdx.x];
  if (b_frozen(sh, blockIdx.x)) return;
  double* u = b_arr_u(P, arr);
  double* v = b_arr_v(P, arr);
  if (p_ghosts) {
    p_ghost_ring(P.p, P.x, P.g, P.bc_kind);
    __syncthreads();
  }
  for (int s = 0; s < 8 && prog.op[s] != OP_END; ++s) {
    switch (prog.op[s]) {
      case OP_VEL_PRED: bc_velocity(u, v, P.g, P.bc, true); break;
      case OP_VEL_CORR: bc_velocity(u, v, P.g, P.bc, false); break;
      case OP_MASS: if (P.bc.has_outlet) bc_mass_balance(u, v, P.g, P.bc); break;
      case OP_MASK_NONE:
      case OP_MASK_RESET:
      case OP_MASK_ACC: if (P.bc.n_mask_u + P.bc.n_mask_v > 0) bc_mask(u, v, P.bc, P.S, prog.op[s]); break;
      case OP_WRAP_FACES: bc_wrap_faces(u, v, P.g); break;
      default: break;
    }
  }
}

// Poisson right-hand side b = div(u*)/dt + Dirichlet terms on solvable rows and
// its fluid mean (pycfd/core/solver.py:659-661, pycfd/core/pressure.py:300-308).
// Warp strips: the four face values of each of a thread's cells loaded first.
template <class T>
B_STRIP_KERNEL k_b_div_rhs(const BProb<T>* __restrict__ probs,
                                                          const int2* __restrict__ map, int arr,
                                                          BShared sh) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  constexpr int RS = b_rs<double>();
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (b_frozen(sh, e.x)) return;
  B_VIEW(V, P);
  const Geo& g = V.g;
  const long W = g.ny + 2, WV = g.ny + 3;
  const double* __restrict__ u = b_arr_u(P, arr);
  const double* __restrict__ v = b_arr_v(P, arr);
  const uint8_t* __restrict__ flags = P.flags;
  double* __restrict__ b = P.b;
  const double dt = P.S[S_DT];
  double acc[1] = {0.0};
  uint8_t fv[RS];
  double ue[RS], uw[RS], vn[RS], vs[RS];
  b_strips<false, double, RS>(
      V, e.y, [](int, int, int) { return 0.0; },
      [&](int q, int c) {
        const int i = c / g.ny, j = c - i * g.ny;
        fv[q] = flags[c];
        ue[q] = u[(long)(i + 2) * W + j + 1];
        uw[q] = u[(long)(i + 1) * W + j + 1];
        vn[q] = v[(long)(i + 1) * WV + j + 2];
        vs[q] = v[(long)(i + 1) * WV + j + 1];
      },
      [&](int q, int c, int i, int j, double, double, double, double, double) {
        const uint8_t f = fv[q];
        double val = 0.0;
        if (f & F_SOLV) {
          const double div = (ue[q] - uw[q]) / g.dx + (vn[q] - vs[q]) / g.dy;   // cell_div's expression
          val = (div / dt) * 1.0 + fine_bc(f, i, j, g);
          acc[0] += val;
        }
        b[c] = val;
      });
  b_reduce<1>(acc, sh.partials + (long)P.red_base * 8, P.counter, e.y, P.s_chunks,
              [&](double* t) { P.S[S_MEAN_B] = g.n_fluid ? t[0] / g.n_fluid : 0.0; });
}

// Velocity correction on the solvable faces and the interior of p
// (pycfd/core/solver.py:665-682); the ghost ring follows in k_b_boundary.
template <class T>
__global__ void __launch_bounds__(kBThreads) k_b_correct(const BProb<T>* __restrict__ probs,
                                                          const int2* __restrict__ map, int arr,
                                                          BShared sh) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (b_frozen(sh, e.x)) return;
  const Geo& g = P.g;
  const int nx = g.nx, ny = g.ny;
  double* u = b_arr_u(P, arr);
  double* v = b_arr_v(P, arr);
  const double* x = P.x;
  double* p = P.p;
  const double dt = P.S[S_DT];
  B_CHUNK_TILES(P, e.y) {
    B_TILE_EXT(P, tile_, nx + 2, ny + 3) {
      if (i >= 1 && i <= nx && j >= 1 && j <= ny) p[(long)i * (ny + 2) + j] = x[(long)(i - 1) * ny + (j - 1)];
      if (i >= g.u_lo && i < g.u_hi && j >= 1 && j <= ny) {
        const long k = (long)i * (ny + 2) + j;
        u[k] = u[k] - dt * (p_at(x, i, j, g) - p_at(x, i - 1, j, g)) / g.dx;
      }
      if (i >= 1 && i <= nx && j >= g.v_lo && j < g.v_hi) {
        const long k = (long)i * (ny + 3) + j;
        v[k] = v[k] - dt * (p_at(x, i, j, g) - p_at(x, i, j - 1, g)) / g.dy;
      }
    }
  }
}

// u = ca*a + cb*b over whole ghosted arrays, in place into the state
// (pycfd/core/solver.py:705-721).
template <class T>
__global__ void __launch_bounds__(kBThreads) k_b_combine(const BProb<T>* __restrict__ probs,
                                                          const int2* __restrict__ map, int src_b,
                                                          double ca, double cb, BShared sh) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (b_frozen(sh, e.x)) return;
  const int nx = P.g.nx, ny = P.g.ny;
  const double* bu = b_arr_u(P, src_b);
  const double* bv = b_arr_v(P, src_b);
  B_CHUNK_TILES(P, e.y) {
    B_TILE_EXT(P, tile_, nx + 3, ny + 3) {
      if (j < ny + 2) {
        const long k = (long)i * (ny + 2) + j;
        P.u[k] = rmul(ca, P.u[k]) + rmul(cb, bu[k]);
      }
      if (i < nx + 2) {
        const long k = (long)i * (ny + 3) + j;
        P.v[k] = rmul(ca, P.v[k]) + rmul(cb, bv[k]);
      }
    }
  }
}

// ---- FP64 MG-PCG ---------------------------------------------------------------
// b <- b - mean (solvable rows), r = b - A x from the warm start x, norms and
// the convergence test before the first pass (scipy cg, pressure.py:300-308).
template <class T>
B_STRIP_KERNEL k_b_rhs_init(const BProb<T>* __restrict__ probs,
                                                           int nprob, const int2* __restrict__ map,
                                                           double tol, int maxiter, BShared sh,
                                                           LoopCtl loop) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  constexpr int RS = b_rs<double>();
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (!b_frozen(sh, e.x)) {
    B_VIEW(V, P);
    const Geo& g = V.g;
    const double mean = P.singular ? P.S[S_MEAN_B] : 0.0;
    const uint8_t* __restrict__ flags = P.flags;
    const T* __restrict__ xs = P.xs;
    double* __restrict__ b = P.b;
    T* __restrict__ r = P.r;
    double acc[3] = {0, 0, 0};
    uint8_t fv[RS];
    double bv[RS];
    b_strips<true, double, RS>(
        V, e.y, [&](int k, int, int) { return (double)xs[k]; },
        [&](int q, int c) {
          fv[q] = flags[c];
          bv[q] = b[c];
        },
        [&](int q, int c, int i, int j, double xc, double xw, double xe, double xsv, double xn) {
          const uint8_t f = fv[q];
          const double bc = (f & F_SOLV) ? bv[q] - mean : 0.0;
          b[c] = bc;
          const double ax = b_apply5<double>(V, f, i, j, xc, xw, xe, xsv, xn);
          const double rc = bc - ax;
          r[c] = (T)rc;
          acc[0] += bc * bc;
          acc[1] += rc * rc;
          if (f & F_SOLV) acc[2] += rc;
        });
    b_reduce<3>(acc, sh.partials + (long)P.red_base * 8, P.counter, e.y, P.s_chunks, [&](double* t) {
      double* S = P.S;
      int* I = P.I;
      S[S_BNORM2] = t[0];
      S[S_ATOL] = tol * sqrt(t[0]);
      S[S_RNORM2] = t[1];
      S[S_RHO_PREV] = 1.0;
      S[S_SUM_R] = t[2];
      S[S_MEAN_R] = g.n_fluid ? t[2] / g.n_fluid : 0.0;
      I[I_IT] = 0;
      I[I_ZERO_RHS] = (t[0] == 0.0);
      const bool conv = (t[0] == 0.0) || (sqrt(t[1]) < S[S_ATOL]);
      I[I_CONVERGED] = conv;
      I[I_DONE] = conv || maxiter <= 0;
      I[I_STATUS] = 0;
      sh.solving[e.x] = !I[I_DONE];
    });
  }
  b_loop_ticket(probs, nprob, sh, TK_CG, I_DONE, 1, maxiter + 1, loop);
}

// The CG direction of pass `it` lives in pa (it even) or pb (it odd), the
// previous one in the other buffer, so no pass copies p.
template <class T>
__device__ __forceinline__ T* b_pdir(const BProb<T>& P, int it) {
  return (it & 1) ? P.pb : P.pa;
}

// p = (z - mean z) + beta p_old on solvable rows, q = A p, p.q -> alpha.
template <class T>
B_STRIP_KERNEL k_b_cg_pq(const BProb<T>* __restrict__ probs,
                                                        const int2* __restrict__ map, BShared sh) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  constexpr int RS = b_rs<T>();
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (!b_solving(sh, e.x)) return;
  B_VIEW(V, P);
  const int it = P.I[I_IT];
  const bool first = it == 0;
  const double beta = first ? 0.0 : P.S[S_RHO] / P.S[S_RHO_PREV];
  const double mz = P.S[S_MEAN_Z];
  const uint8_t* __restrict__ flags = P.flags;
  const T* __restrict__ zraw = P.z;
  const T* __restrict__ p_old = b_pdir(P, it + 1);
  T* __restrict__ pn = b_pdir(P, it);
  T* __restrict__ q = P.q;
  // arithmetic in T (FP32 in the mixed form's inner solve), p.q summed in FP64
  const T tb = (T)beta, tm = (T)mz;
  auto pval = [&](int k, int, int) -> T {   // all loads issued, then selected
    const uint8_t fk = flags[k];
    const T zk = zraw[k];
    const T pk = p_old[k];                   // unused (and possibly unset) on the first pass
    const T z = (fk & F_SOLV) ? zk - tm : (T)0;
    if (first) return z;
    return pk * tb + z;
  };
  double acc[1] = {0.0};
  bool walked = false;
  if constexpr (sizeof(T) == 4) {
    if (P.vec) {
      constexpr int RSV = 2;
      auto pval4 = [&](int k, int, int) -> float4 {   // all loads issued, then selected
        const uint32_t fk = b_ldf4(flags + k);
        const float4 zk = b_ld4(zraw + k);
        const float4 pk = b_ld4(p_old + k);
        float o[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) {
          const float z = (b_fl(fk, s) & F_SOLV) ? b_el(zk, s) - tm : 0.f;
          o[s] = first ? z : b_el(pk, s) * tb + z;
        }
        return make_float4(o[0], o[1], o[2], o[3]);
      };
      uint32_t fw[RSV];
      b_vstrips<true, RSV>(V, e.y, pval4, pval, [&](int u, int k) { fw[u] = b_ldf4(flags + k); },
                           [&](int u, int k, int i, int j, const float(&pc)[4], const float(&pw)[4],
                               const float(&pe)[4], const float(&ps)[4], const float(&pnb)[4]) {
                             float qc[4];
#pragma unroll
                             for (int s = 0; s < 4; ++s) {
                               qc[s] = b_apply5f(V, b_fl(fw[u], s), i, j + s, pc[s], pw[s], pe[s], ps[s],
                                                       pnb[s]);
                               acc[0] += (double)pc[s] * (double)qc[s];
                             }
                             b_st4(pn + k, pc);
                             b_st4(q + k, qc);
                           });
      walked = true;
    }
  }
  if (!walked) {
    uint8_t fv[RS];
    b_strips<true, T, RS>(V, e.y, pval, [&](int u, int c) { fv[u] = flags[c]; },
                      [&](int u, int c, int i, int j, T pc, T pw, T pe, T ps, T pnn) {
                        const T qc = b_apply5<T>(V, fv[u], i, j, pc, pw, pe, ps, pnn);
                        pn[c] = pc;
                        q[c] = qc;
                        acc[0] += (double)pc * (double)qc;
                      });
  }
  b_reduce<1>(acc, sh.partials + (long)P.red_base * 8, P.counter, e.y, b_nchunks(P), [&](double* t) {
    P.S[S_PQ] = t[0];
    P.S[S_ALPHA] = P.S[S_RHO] / t[0];
  });
}

// x += alpha p, r -= alpha q; ||r||^2 and sum(r); the next pass's convergence
// test; launch-wide loop decision.
template <class T>
B_STRIP_KERNEL k_b_cg_xr(const BProb<T>* __restrict__ probs, int nprob,
                                                        const int2* __restrict__ map, int maxiter,
                                                        BShared sh, LoopCtl loop) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  constexpr int RS = b_rs<T>();
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (b_solving(sh, e.x)) {
    const Geo& g = P.g;
    B_VIEW(V, P);
    const double alpha = P.S[S_ALPHA];
    const uint8_t* __restrict__ flags = P.flags;
    const T* __restrict__ pn = b_pdir(P, P.I[I_IT]);
    const T* __restrict__ q = P.q;
    T* __restrict__ xs = P.xs;
    T* __restrict__ r = P.r;
    double acc[2] = {0, 0};
    bool walked = false;
    if constexpr (sizeof(T) == 4) {
      if (P.vec) {
        constexpr int RSV = 2;
        float4 pw[RSV], xw[RSV], rw[RSV], qw[RSV];
        uint32_t fw[RSV];
        b_vstrips<false, RSV>(
            V, e.y, [](int, int, int) { return make_float4(0.f, 0.f, 0.f, 0.f); },
            [](int, int, int) { return 0.f; },
            [&](int u, int k) {
              pw[u] = b_ld4(pn + k);
              xw[u] = b_ld4(xs + k);
              rw[u] = b_ld4(r + k);
              qw[u] = b_ld4(q + k);
              fw[u] = b_ldf4(flags + k);
            },
            [&](int u, int k, int, int, const float(&)[4], const float(&)[4], const float(&)[4],
                const float(&)[4], const float(&)[4]) {
              float xo[4], ro[4];
#pragma unroll
              for (int s = 0; s < 4; ++s) {
                const double xc = (double)b_el(xw[u], s) + alpha * (double)b_el(pw[u], s);
                const double rc = (double)(float)((double)b_el(rw[u], s) - alpha * (double)b_el(qw[u], s));
                xo[s] = (float)xc;
                ro[s] = (float)rc;
                acc[0] += rc * rc;
                if (b_fl(fw[u], s) & F_SOLV) acc[1] += rc;
              }
              b_st4(xs + k, xo);
              b_st4(r + k, ro);
            });
        walked = true;
      }
    }
    if (!walked) {
      T pv[RS], xv[RS], rv[RS], qv[RS];
      uint8_t fv[RS];
      b_strips<false, T, RS>(
          V, e.y, [](int, int, int) { return (T)0; },
          [&](int u, int c) {
            pv[u] = pn[c];
            xv[u] = xs[c];
            rv[u] = r[c];
            qv[u] = q[c];
            fv[u] = flags[c];
          },
          [&](int u, int c, int, int, T, T, T, T, T) {
            const double xc = (double)xv[u] + alpha * (double)pv[u];
            const double rc = (double)(T)((double)rv[u] - alpha * (double)qv[u]);
            xs[c] = (T)xc;
            r[c] = (T)rc;
            acc[0] += rc * rc;
            if (fv[u] & F_SOLV) acc[1] += rc;
          });
    }
    b_reduce<2>(acc, sh.partials + (long)P.red_base * 8, P.counter, e.y, b_nchunks(P), [&](double* t) {
      double* S = P.S;
      int* I = P.I;
      const int it = I[I_IT] + 1;
      I[I_IT] = it;
      I[I_TOTAL_IT] += 1;
      S[S_RNORM2] = t[0];
      S[S_SUM_R] = t[1];
      S[S_MEAN_R] = g.n_fluid ? t[1] / g.n_fluid : 0.0;
      const bool conv = sqrt(t[0]) < S[S_ATOL];
      I[I_CONVERGED] = conv;
      I[I_DONE] = conv || it >= maxiter;
      sh.solving[e.x] = !I[I_DONE];
    });
  }
  b_loop_ticket(probs, nprob, sh, TK_CG, I_DONE, 0, maxiter + 1, loop);
}

// ||b - A x||/||b|| and the fluid mean of x (pycfd/core/pressure.py:310-322).
template <class T>
B_STRIP_KERNEL k_b_finish_stats(const BProb<T>* __restrict__ probs,
                                                               const int2* __restrict__ map, double tol,
                                                               BShared sh) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  constexpr int RS = b_rs<double>();
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (b_frozen(sh, e.x)) return;
  B_VIEW(V, P);
  const Geo& g = V.g;
  const bool zero = P.I[I_ZERO_RHS] != 0;
  const double* __restrict__ x = P.x;
  const double* __restrict__ b = P.b;
  const uint8_t* __restrict__ flags = P.flags;
  double acc[2] = {0, 0};
  uint8_t fv[RS];
  double bv[RS];
  b_strips<true, double, RS>(
      V, e.y, [&](int k, int, int) { return zero ? 0.0 : x[k]; },
      [&](int q, int c) {
        fv[q] = flags[c];
        bv[q] = b[c];
      },
      [&](int q, int, int i, int j, double xc, double xw, double xe, double xsv, double xn) {
        const uint8_t f = fv[q];
        const double rc = bv[q] - b_apply5<double>(V, f, i, j, xc, xw, xe, xsv, xn);
        acc[0] += rc * rc;
        if (f & F_SOLV) acc[1] += xc;
      });
  b_reduce<2>(acc, sh.partials + (long)P.red_base * 8, P.counter, e.y, P.s_chunks, [&](double* t) {
    double* S = P.S;
    const double nb = sqrt(S[S_BNORM2]);
    S[S_RESID] = sqrt(t[0]) / (nb > 1e-300 ? nb : 1.0);
    if (!P.I[I_CONVERGED] && S[S_RESID] > fmax(tol * 10.0, 1e-8)) P.I[I_STATUS] = -3;
    S[S_MEAN_X] = (P.singular && g.n_fluid) ? t[1] / g.n_fluid : 0.0;
  });
}

// x <- x - mean on solvable rows, 0 elsewhere.
template <class T>
B_STRIP_KERNEL k_b_finish_apply(const BProb<T>* __restrict__ probs,
                                                               const int2* __restrict__ map, BShared sh) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  constexpr int RS = b_rs<double>();
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (b_frozen(sh, e.x)) return;
  B_VIEW(V, P);
  const bool zero = P.I[I_ZERO_RHS] != 0;
  const double m = P.S[S_MEAN_X];
  double* __restrict__ x = P.x;
  const uint8_t* __restrict__ flags = P.flags;
  uint8_t fv[RS];
  double xv[RS];
  b_strips<false, double, RS>(
      V, e.y, [](int, int, int) { return 0.0; },
      [&](int q, int c) {
        fv[q] = flags[c];
        xv[q] = x[c];
      },
      [&](int q, int c, int, int, double, double, double, double, double) {
        x[c] = (!zero && (fv[q] & F_SOLV)) ? xv[q] - m : 0.0;
      });
}

// ---- mixed form: FP64 iterative refinement around the FP32 MG-PCG -----------
// One refinement pass per problem (see k_ir_residual): r = b - A x in FP64, the
// outer test ||r|| < tol ||b||, and the inner solve A e = r set up from e = 0.
template <class T>
B_STRIP_KERNEL k_b_ir_residual(const BProb<T>* __restrict__ probs,
                                                              int nprob, const int2* __restrict__ map,
                                                              double tol, double inner_tol,
                                                              int max_passes, int first, BShared sh,
                                                              LoopCtl outer) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  constexpr int RS = b_rs<double>();
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (!b_frozen(sh, e.x) && (first || !P.I[I_IR_DONE])) {
    B_VIEW(V, P);
    const Geo& g = V.g;
    const double mean = (first && P.singular) ? P.S[S_MEAN_B] : 0.0;
    const uint8_t* __restrict__ flags = P.flags;
    const double* __restrict__ x = P.x;
    double* __restrict__ b = P.b;
    T* __restrict__ r = P.r;
    T* __restrict__ xs = P.xs;
    double acc[3] = {0, 0, 0};
    uint8_t fv[RS];
    double bv[RS];
    b_strips<true, double, RS>(
        V, e.y, [&](int k, int, int) { return x[k]; },
        [&](int q, int c) {
          fv[q] = flags[c];
          bv[q] = b[c];
        },
        [&](int q, int c, int i, int j, double xc, double xw, double xe, double xsv, double xn) {
          const uint8_t f = fv[q];
          double bc = bv[q];
          if (first) {
            bc = (f & F_SOLV) ? bc - mean : 0.0;
            b[c] = bc;
          }
          const double rc = bc - b_apply5<double>(V, f, i, j, xc, xw, xe, xsv, xn);
          r[c] = (T)rc;
          xs[c] = (T)0;
          acc[0] += rc * rc;
          if (f & F_SOLV) acc[1] += (double)(T)rc;
          if (first) acc[2] += bc * bc;
        });
    b_reduce<3>(acc, sh.partials + (long)P.red_base * 8, P.counter, e.y, P.s_chunks, [&](double* t) {
      double* S = P.S;
      int* I = P.I;
      if (first) {
        S[S_IR_BNORM] = sqrt(t[2]);
        S[S_BNORM2] = t[2];
        I[I_IR_IT] = 0;
        I[I_ZERO_RHS] = (t[2] == 0.0);
        I[I_STATUS] = 0;
      }
      const double nb = S[S_IR_BNORM];
      S[S_IR_RNORM2] = t[0];
      const bool conv = (nb == 0.0) || (sqrt(t[0]) < tol * nb);
      const bool done = conv || I[I_IR_IT] >= max_passes;
      I[I_CONVERGED] = conv;
      I[I_IR_DONE] = done;
      S[S_ATOL] = fmax(inner_tol * sqrt(t[0]), kIrLastFraction * tol * nb);   // as k_ir_residual
      S[S_RNORM2] = t[0];
      S[S_RHO_PREV] = 1.0;
      S[S_SUM_R] = t[1];
      S[S_MEAN_R] = g.n_fluid ? t[1] / g.n_fluid : 0.0;
      I[I_IT] = 0;
      I[I_DONE] = done;
      sh.solving[e.x] = !done;
    });
  }
  b_loop_ticket(probs, nprob, sh, TK_IR, I_IR_DONE, first, max_passes + 1, outer);
}

// Arm the inner loop: does any problem run an inner solve in this pass?
template <class T>
__global__ void k_b_ir_arm(const BProb<T>* __restrict__ probs, int nprob, BShared sh, LoopCtl inner) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  int any = 0;
  for (int p = threadIdx.x; p < nprob; p += blockDim.x)
    if (b_solving(sh, p)) any = 1;
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) {
    sh.any[TK_ARM] = any;
    sh.iters[TK_CG] = 0u;   // the inner loop's passes count from here
    inner.set(any != 0);
    if (any) sh.passes[TK_ARM] += 1;
  }
}

// x += e on solvable rows for the problems that ran this pass; count the pass.
template <class T>
B_STRIP_KERNEL k_b_ir_update(const BProb<T>* __restrict__ probs,
                                                            const int2* __restrict__ map, BShared sh) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  constexpr int RS = b_rs<double>();
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (b_frozen(sh, e.x) || P.I[I_IR_DONE]) return;
  B_VIEW(V, P);
  double* __restrict__ x = P.x;
  const T* __restrict__ xs = P.xs;
  const uint8_t* __restrict__ flags = P.flags;
  uint8_t fv[RS];
  double xv[RS];
  T ev[RS];
  b_strips<false, double, RS>(
      V, e.y, [](int, int, int) { return 0.0; },
      [&](int q, int c) {
        fv[q] = flags[c];
        xv[q] = x[c];
        ev[q] = xs[c];
      },
      [&](int q, int c, int, int, double, double, double, double, double) {
        if (fv[q] & F_SOLV) x[c] = xv[q] + (double)ev[q];
      });
  if (e.y == 0 && threadIdx.x == 0) P.I[I_IR_IT] += 1;
}

// ---- V-cycle ---------------------------------------------------------------------
// Level-0 (matrix-free) phases.  The right-hand side is the CG residual r
// projected onto the active set (r - mean r on solvable rows,
// pycfd/core/multigrid.py:453-458).  Buffers: 0 level-0 xa, 1 level-0 xb, 2 z.
enum BFineMode { FM_PRE = 0, FM_WDB, FM_SMOOTH, FM_RESID, FM_LAST };

template <class T>
__device__ __forceinline__ T* b_fine_buf(const BProb<T>& P, int sel) {
  return sel == 0 ? P.lxa[0] : sel == 1 ? P.lxb[0] : P.z;
}

// Level d's iterate in buffer sel (0: xa, 1: xb).
template <class T>
__device__ __forceinline__ T* b_lvl_x(const BProb<T>& P, int d, int sel) {
  if (d == P.nlev - 1 || d == P.tail) return P.lxa[d];   // coarsest and tail results are in xa
  return sel == 0 ? P.lxa[d] : P.lxb[d];
}

// Closes the last sweep of a cycle from its sums (t[0] = sum z over the
// solvable cells, t[1] = r.z): the fluid mean of z and rho = r.(z - mean z).
template <class T>
__device__ __forceinline__ void b_last_close(const BProb<T>& P, const double* t) {
  double* S = P.S;
  const double m = (P.singular && P.g.n_fluid) ? t[0] / P.g.n_fluid : 0.0;
  S[S_MEAN_Z] = m;
  S[S_RHO_PREV] = S[S_RHO];
  S[S_RHO] = t[1] - m * S[S_SUM_R];
}

template <class T, int MODE>
B_STRIP_KERNEL k_b_fine(const BProb<T>* __restrict__ probs,
                                                       const BHier<T>* __restrict__ hiers,
                                                       const int2* __restrict__ map, int src, int dst,
                                                       BShared sh) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  constexpr int RS = b_rs<T>();
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (!b_solving(sh, e.x)) return;
  B_VIEW(V, P);
  // arithmetic in T (FP32 in the mixed form's inner solve), sums in FP64
  const uint8_t* __restrict__ flags = P.flags;
  const T* __restrict__ r = P.r;
  const T mr = (T)(P.singular ? P.S[S_MEAN_R] : 0.0);
  const T* __restrict__ x = b_fine_buf(P, src);
  T* __restrict__ xo = b_fine_buf(P, dst);
  T* __restrict__ lres0 = P.lres[0];
  double acc[2] = {0, 0};
  if constexpr (sizeof(T) == 4) {
    if (P.vec) {
      constexpr int RSV = 2;
      uint32_t fw[RSV];
      float4 rw[RSV];
      auto vload = [&](int u, int k) {
        fw[u] = b_ldf4(flags + k);
        rw[u] = b_ld4(r + k);
      };
      auto vb = [&](int u, int s) -> float { return (b_fl(fw[u], s) & F_SOLV) ? b_el(rw[u], s) - mr : 0.f; };
      if (MODE == FM_WDB) {
        b_vstrips<false, RSV>(V, e.y, [](int, int, int) { return make_float4(0.f, 0.f, 0.f, 0.f); },
                              [](int, int, int) { return 0.f; }, vload,
                              [&](int u, int k, int i, int j, const float(&)[4], const float(&)[4],
                                  const float(&)[4], const float(&)[4], const float(&)[4]) {
                                float o[4];
#pragma unroll
                                for (int s = 0; s < 4; ++s) o[s] = b_wdinv_f(V, b_fl(fw[u], s), i, j + s) * vb(u, s);
                                b_st4(xo + k, o);
                              });
      } else if (MODE == FM_PRE) {
        // first sweep from zero, x = W b, and the residual b - A W b
        auto xw1 = [&](int k, int ii, int jj) -> float {
          const uint8_t fk = flags[k];
          const float rk = r[k];
          const float bk = (fk & F_SOLV) ? rk - mr : 0.f;
          return b_wdinv_f(V, fk, ii, jj) * bk;
        };
        auto xw4 = [&](int k, int ii, int jj) -> float4 {   // all loads issued, then selected
          const uint32_t fk = b_ldf4(flags + k);
          const float4 rk = b_ld4(r + k);
          float o[4];
#pragma unroll
          for (int s = 0; s < 4; ++s) {
            const uint8_t f = b_fl(fk, s);
            const float bk = (f & F_SOLV) ? b_el(rk, s) - mr : 0.f;
            o[s] = b_wdinv_f(V, f, ii, jj + s) * bk;
          }
          return make_float4(o[0], o[1], o[2], o[3]);
        };
        b_vstrips<true, RSV>(V, e.y, xw4, xw1, vload,
                             [&](int u, int k, int i, int j, const float(&xc)[4], const float(&xwe)[4],
                                 const float(&xe)[4], const float(&xsv)[4], const float(&xn)[4]) {
                               float o[4];
#pragma unroll
                               for (int s = 0; s < 4; ++s)
                                 o[s] = vb(u, s) - b_apply5f(V, b_fl(fw[u], s), i, j + s, xc[s], xwe[s], xe[s],
                                                                   xsv[s], xn[s]);
                               b_st4(xo + k, xc);
                               b_st4(lres0 + k, o);
                             });
      } else {
        b_vstrips<true, RSV>(V, e.y, [&](int k, int, int) { return b_ld4(x + k); },
                             [&](int k, int, int) -> float { return x[k]; }, vload,
                             [&](int u, int k, int i, int j, const float(&xc)[4], const float(&xwe)[4],
                                 const float(&xe)[4], const float(&xsv)[4], const float(&xn)[4]) {
                               float o[4];
#pragma unroll
                               for (int s = 0; s < 4; ++s) {
                                 const uint8_t f = b_fl(fw[u], s);
                                 const float ax = b_apply5f(V, f, i, j + s, xc[s], xwe[s], xe[s], xsv[s], xn[s]);
                                 if (MODE == FM_RESID) {
                                   o[s] = vb(u, s) - ax;
                                 } else {
                                   const float xnew = xc[s] + b_wdinv_f(V, f, i, j + s) * (vb(u, s) - ax);
                                   o[s] = xnew;
                                   if (MODE == FM_LAST && (f & F_SOLV)) {
                                     acc[0] += (double)xnew;
                                     acc[1] += (double)b_el(rw[u], s) * (double)xnew;
                                   }
                                 }
                               }
                               b_st4(MODE == FM_RESID ? lres0 + k : xo + k, o);
                             });
      }
      if (MODE != FM_LAST) return;
      b_reduce<2>(acc, sh.partials + (long)P.red_base * 8, P.counter, e.y, P.v_chunks, [&](double* t) {
        b_last_close(P, t);
      });
      return;
    }
  }
  uint8_t fv[RS];
  T rv[RS];
  auto load = [&](int u, int c) {
    fv[u] = flags[c];
    rv[u] = r[c];
  };
  auto bfv = [&](int u) -> T { return (fv[u] & F_SOLV) ? rv[u] - mr : (T)0; };   // right-hand side at the cell
  if (MODE == FM_WDB) {
    b_strips<false, T, RS>(V, e.y, [](int, int, int) { return (T)0; }, load,
                       [&](int u, int c, int i, int j, T, T, T, T, T) {
                         xo[c] = (T)b_wdinv(V, fv[u], i, j) * bfv(u);
                       });
  } else if (MODE == FM_PRE) {
    // first sweep from zero, x = W b, and the residual b - A W b
    auto xw = [&](int k, int ii, int jj) -> T {   // both loads issued, then selected
      const uint8_t fk = flags[k];
      const T rk = r[k];
      const T bk = (fk & F_SOLV) ? rk - mr : (T)0;
      return (T)b_wdinv(V, fk, ii, jj) * bk;
    };
    b_strips<true, T, RS>(V, e.y, xw, load, [&](int u, int c, int i, int j, T xc, T xw_, T xe, T xs_, T xn) {
      xo[c] = xc;
      lres0[c] = bfv(u) - b_apply5<T>(V, fv[u], i, j, xc, xw_, xe, xs_, xn);
    });
  } else {
    auto xv = [&](int k, int, int) -> T { return x[k]; };
    b_strips<true, T, RS>(V, e.y, xv, load, [&](int u, int c, int i, int j, T xc, T xw_, T xe, T xs_, T xn) {
      const uint8_t f = fv[u];
      if (MODE == FM_RESID) {
        lres0[c] = bfv(u) - b_apply5<T>(V, f, i, j, xc, xw_, xe, xs_, xn);
      } else {
        const T xnew = xc + (T)b_wdinv(V, f, i, j) * (bfv(u) - b_apply5<T>(V, f, i, j, xc, xw_, xe, xs_, xn));
        xo[c] = xnew;
        if (MODE == FM_LAST && (f & F_SOLV)) {
          acc[0] += (double)xnew;
          acc[1] += (double)rv[u] * (double)xnew;
        }
      }
    });
  }
  if (MODE != FM_LAST) return;
  b_reduce<2>(acc, sh.partials + (long)P.red_base * 8, P.counter, e.y, P.s_chunks, [&](double* t) {
    b_last_close(P, t);
  });
}

// ---- level-0 transfers as stencils -------------------------------------------------
// On a structure whose level 1 aggregates 2 x 2 fine cells (T: the 0/1 map of a
// solvable cell (i, j) to aggregate (i/2, j/2)), the smoothed prolongation and
// the fused restriction of the hierarchy are
//   P_1 = (I - W A) T,   M_1 = P_1^T (I - A W) = T^T (I - A W)^2,
// A the fine operator, W its damped inverse diagonal (A symmetric, W diagonal).
// Both then run as stencils over the fine cells instead of row gathers through
// the stored matrices: the aggregate map is index arithmetic and A the flag
// stencil, so a fine cell costs its flags, its residual and one level-1 value.
// Each needs values two cells away, so a block takes a tile of output cells
// (h_tr rows of x, 28 columns of y) and stages the tile with two halo cells on
// each side (h_tr + 4 rows x 32 columns: lane = column) in shared memory: every
// thread issues its loads of the tile at once, then the stages run on shared
// memory between block barriers.  The arithmetic is the matrices' definition in
// the storage type, so the results equal the matrix products to rounding (not
// bit for bit).
constexpr int kBHaloTC = 28;   // output columns of a tile (input: 32, two halo columns each side)
// Most output rows of a tile (FP32 60, FP64 28: the staged arrays stay within
// 48 KB); a problem's tiles take ceil(nx / ceil(nx / most)) rows, rounded up to even.
template <class T>
__host__ __device__ constexpr int b_halo_tr_max() { return sizeof(T) == 8 ? 28 : 60; }
#ifndef PCFD_BHALO_MINB
#define PCFD_BHALO_MINB 4
#endif
#define B_HALO_KERNEL __global__ void __launch_bounds__(kBThreads, PCFD_BHALO_MINB)

// Cell index of a line of n cells at offset r (at most two past either end):
// wrapped on a periodic axis, -1 off the grid.
__device__ __forceinline__ int b_wrap2(int r, int n, int periodic) {
  if (r < 0) r = periodic ? r + n : -1;
  else if (r >= n) r = periodic ? r - n : -1;
  return (r >= 0 && r < n) ? r : -1;
}

// A tile's staged arrays: input rows x 32 columns.
template <class T>
struct BHaloTile {
  static constexpr int R = b_halo_tr_max<T>() + 4;
  uint8_t f[R][32];                          // flags (0 off the grid)
  T dg[R][32], wd[R][32];                    // diagonal, damped inverse diagonal
  T a[R][32], b[R][32], c[R][32];            // the stages' vectors
};

// Stage 0 of a tile with first output cell (i0, j0): thread (warp w, lane)
// loads input rows w, w + 8, ... of column j0 - 2 + lane -- the flags and
// get(k) (cell index k; read at a valid index, dropped off the grid), all
// loads first -- and stores the flags, the diagonal and weighted inverse
// diagonal (b_diag and b_wdinv) and put(row, lane, f, wd, value).
template <class T, class Get, class Put>
__device__ __forceinline__ void b_tile_load(const BView& V, BHaloTile<T>& S, int rows, int i0, int j0,
                                            const uint8_t* __restrict__ flags, Get get, Put put) {
  constexpr int K = BHaloTile<T>::R / 8;
  const int lane = (int)(threadIdx.x & 31), w = (int)(threadIdx.x >> 5);
  const int nx = V.g.nx, ny = V.g.ny;
  const int col = b_wrap2(j0 - 2 + lane, ny, V.g.periodic_y), cc = col >= 0 ? col : 0;
  uint8_t fr[K];
  T vr[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int row = b_wrap2(i0 - 2 + w + 8 * k, nx, V.g.periodic_x), rc = row >= 0 ? row : 0;
    const int idx = rc * ny + cc;
    const uint8_t fk = flags[idx];
    const T vk = get(idx, rc, cc);
    const bool ok = row >= 0 && col >= 0 && w + 8 * k < rows;
    fr[k] = ok ? fk : (uint8_t)0;
    vr[k] = ok ? vk : (T)0;
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int ii = w + 8 * k;
    if (ii >= rows) break;
    const uint8_t fu = fr[k];
    double d = 1.0, wv = V.w0 * (1.0 / 1.0);   // b_diag, b_wdinv off the solvable cells
    if (fu & F_SOLV) {
      const int i = b_wrap2(i0 - 2 + ii, nx, V.g.periodic_x);
      if (V.any_dir && (i == 0 || col == 0 || i == nx - 1 || col == ny - 1)) {
        d = fine_diag(fu, i, col, V.g);
        wv = V.w0 * (1.0 / d);
      } else {
        d = V.dtab[fu & 15];
        wv = V.wtab[fu & 15];
      }
    }
    S.f[ii][lane] = fu;
    S.dg[ii][lane] = (T)d;
    S.wd[ii][lane] = (T)wv;
    put(ii, lane, fu, (T)wv, vr[k]);
  }
}

// (A x) at staged cell (ii, jl), b_apply5's terms in its order.
template <class T>
__device__ __forceinline__ T b_tile_apply(const BView& V, const BHaloTile<T>& S, const T (*x)[32], int ii, int jl) {
  const uint8_t f = S.f[ii][jl];
  T acc = S.dg[ii][jl] * x[ii][jl];
  if (f & F_W) acc += (T)V.g.cx * x[ii - 1][jl];
  if (f & F_E) acc += (T)V.g.cx * x[ii + 1][jl];
  if (f & F_S) acc += (T)V.g.cy * x[ii][jl - 1];
  if (f & F_N) acc += (T)V.g.cy * x[ii][jl + 1];
  return acc;
}

// b_1 = T^T (I - A W)^2 b, b the projected CG residual (the fused restriction
// from the fine level; pycfd/core/multigrid.py:436-447 with the sweep from zero).
// One block per tile (map entries (problem, tile)).
template <class T>
B_HALO_KERNEL k_b_frestrict0(const BProb<T>* __restrict__ probs, const int2* __restrict__ map, BShared sh) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  constexpr int K = BHaloTile<T>::R / 8, AC = kBHaloTC / 2;
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (!b_solving(sh, e.x)) return;
  B_VIEW(V, P);
  __shared__ BHaloTile<T> S;
  const T* __restrict__ r = P.r;
  T* __restrict__ b1 = P.lb[1];
  const T mr = (T)(P.singular ? P.S[S_MEAN_R] : 0.0);
  const int nx = V.g.nx, ny = V.g.ny, ncy = (ny + 1) >> 1;
  const int tr = P.h_tr, rows = tr + 4;
  const int ti = e.y / P.h_tiles_j, tj = e.y - ti * P.h_tiles_j;
  const int i0 = ti * tr, j0 = tj * kBHaloTC;
  const int lane = (int)(threadIdx.x & 31), w = (int)(threadIdx.x >> 5);
  // b (0 off the solvable cells) and y = W b
  b_tile_load<T>(V, S, rows, i0, j0, P.flags, [&](int k, int, int) { return r[k]; },
                 [&](int ii, int jl, uint8_t f, T wd, T rv) {
                   const T bv = (f & F_SOLV) ? rv - mr : (T)0;
                   S.b[ii][jl] = bv;
                   S.a[ii][jl] = wd * bv;
                 });
  __syncthreads();
  const bool inner_c = lane >= 1 && lane < 31;
#pragma unroll
  for (int k = 0; k < K; ++k) {   // z = (I - A W) b in place of b, one cell in from the tile's edge
    const int ii = w + 8 * k;
    if (ii >= 1 && ii < rows - 1 && inner_c) S.b[ii][lane] -= b_tile_apply<T>(V, S, S.a, ii, lane);
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) {   // y = W z
    const int ii = w + 8 * k;
    if (ii >= 1 && ii < rows - 1 && inner_c) S.a[ii][lane] = S.wd[ii][lane] * S.b[ii][lane];
  }
  __syncthreads();
  // (I - A W) z on the output cells, summed over each aggregate (rows, then columns)
  for (int ag = (int)threadIdx.x; ag < (tr / 2) * AC; ag += kBThreads) {
    const int ar = ag / AC, ac = ag - ar * AC;
    const int gi = i0 + 2 * ar, gj = j0 + 2 * ac;
    if (gi >= nx || gj >= ny) continue;
    T zq[2][2];
#pragma unroll
    for (int di = 0; di < 2; ++di)
#pragma unroll
      for (int dj = 0; dj < 2; ++dj) {
        const int ii = 2 + 2 * ar + di, jl = 2 + 2 * ac + dj;
        const T z2 = S.b[ii][jl] - b_tile_apply<T>(V, S, S.a, ii, jl);
        zq[di][dj] = ((S.f[ii][jl] & F_SOLV) && gi + di < nx && gj + dj < ny) ? z2 : (T)0;
      }
    b1[(gi >> 1) * ncy + (gj >> 1)] = (zq[0][0] + zq[1][0]) + (zq[0][1] + zq[1][1]);
  }
}

// The last two phases of the cycle in one pass: the prolongation onto the fine
// level with its first sweep formed again, x_0 = W b + (I - W A) T x_1, and the
// last sweep z = x_0 + W (b - A x_0), with sum(z) and r.z (k_b_fine FM_LAST).
template <class T>
B_HALO_KERNEL k_b_prolong_last(const BProb<T>* __restrict__ probs, const int2* __restrict__ map, BShared sh) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  constexpr int K = BHaloTile<T>::R / 8;
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (!b_solving(sh, e.x)) return;
  B_VIEW(V, P);
  __shared__ BHaloTile<T> S;
  const T* __restrict__ r = P.r;
  const T* __restrict__ x1 = b_lvl_x(P, 1, 1);
  T* __restrict__ zo = P.z;
  const T mr = (T)(P.singular ? P.S[S_MEAN_R] : 0.0);
  const int nx = V.g.nx, ny = V.g.ny, ncy = (ny + 1) >> 1;
  const int tr = P.h_tr, rows = tr + 4;
  const int ti = e.y / P.h_tiles_j, tj = e.y - ti * P.h_tiles_j;
  const int i0 = ti * tr, j0 = tj * kBHaloTC;
  const int lane = (int)(threadIdx.x & 31), w = (int)(threadIdx.x >> 5);
  // b (0 off the solvable cells) in b, T x_1 (the cell's aggregate value) in a;
  // the residual itself in c for r.z
  b_tile_load<T>(V, S, rows, i0, j0, P.flags, [&](int k, int rc, int cc) { return r[k]; },
                 [&](int ii, int jl, uint8_t f, T, T rv) {
                   S.b[ii][jl] = (f & F_SOLV) ? rv - mr : (T)0;
                   S.c[ii][jl] = rv;
                 });
  {
    const int col = b_wrap2(j0 - 2 + lane, ny, V.g.periodic_y), cc = col >= 0 ? col : 0;
    T xg[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int row = b_wrap2(i0 - 2 + w + 8 * k, nx, V.g.periodic_x), rc = row >= 0 ? row : 0;
      xg[k] = x1[(rc >> 1) * ncy + (cc >> 1)];
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int ii = w + 8 * k;
      if (ii < rows) S.a[ii][lane] = (S.f[ii][lane] & F_SOLV) ? xg[k] : (T)0;   // this thread's own flags
    }
  }
  __syncthreads();
  const bool inner_c = lane >= 1 && lane < 31;
  T x0[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {   // x_0 = W b + (t - W A t), one cell in from the tile's edge
    const int ii = w + 8 * k;
    x0[k] = (T)0;
    if (ii >= 1 && ii < rows - 1 && inner_c) {
      const T wd = S.wd[ii][lane];
      const T s = S.a[ii][lane] - wd * b_tile_apply<T>(V, S, S.a, ii, lane);   // (P_1 x_1) at the cell
      x0[k] = wd * S.b[ii][lane] + s;
    }
  }
  __syncthreads();   // every read of t done: x_0 goes in its place
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int ii = w + 8 * k;
    if (ii >= 1 && ii < rows - 1 && inner_c) S.a[ii][lane] = x0[k];
  }
  __syncthreads();
  double acc[2] = {0, 0};
  const int gj = j0 - 2 + lane;
  if (lane >= 2 && lane < 30 && gj < ny) {
#pragma unroll
    for (int k = 0; k < K; ++k) {   // z = x_0 + W (b - A x_0) on the output cells
      const int ii = w + 8 * k, gi = i0 - 2 + ii;
      if (ii < 2 || ii >= rows - 2 || gi >= nx) continue;
      const T xnew = S.a[ii][lane] + S.wd[ii][lane] * (S.b[ii][lane] - b_tile_apply<T>(V, S, S.a, ii, lane));
      zo[gi * ny + gj] = xnew;
      if (S.f[ii][lane] & F_SOLV) {
        acc[0] += (double)xnew;
        acc[1] += (double)S.c[ii][lane] * (double)xnew;
      }
    }
  }
  b_reduce<2>(acc, sh.partials + (long)P.red_base * 8, P.counter, e.y, P.h_tiles, [&](double* t) {
    b_last_close(P, t);
  });
}

// ELL phases of coarse level d (and prolongation into level 0), applied to
// groups of a structure's problems (k_b_ellg below); one launch covers every
// structure, whatever its hierarchy.
// EO_FRESTRICT: b_d = M_d b_{d-1} (first sweep on d-1 and restriction of its
// residual in one product; from level 0 the right-hand side is the projected CG
// residual).  EO_PROLONGW: prolongation onto a level whose first-sweep iterate
// W b was not stored -- it is formed again, with the same T roundings.
enum BEllOp { EO_RESTRICT = 0, EO_PRE, EO_SMOOTH, EO_RESID, EO_PROLONG, EO_FRESTRICT, EO_PROLONGW };

// Row dot product of E by L lanes (L a power of two, runtime), rows past the
// end contribute nothing; every lane of the warp calls it.
template <class T, class X>
__device__ __forceinline__ T b_ell_row(const Ell<T>& E, int L, int row, int lane, X x) {
  T acc = (T)0;
  if (row < E.n) {
    if (E.rowmajor) {
      const long base = (long)row * E.K;
#pragma unroll 4
      for (int k = lane; k < E.K; k += L) acc += E.val[base + k] * x(E.col[base + k]);
    } else {
#pragma unroll 4
      for (int k = lane; k < E.K; k += L) {
        const long at = (long)k * E.n + row;
        acc += E.val[at] * x(E.col[at]);
      }
    }
  }
  for (int o = L >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o, L);
  return acc;
}

// ---- grouped ELL phases ------------------------------------------------------------
// The problems of one structure share its hierarchy, so a block of a coarse-
// level launch applies one row block of a structure's matrix to a GROUP of up
// to GS of its problems: each lane loads an entry (value, column) once and
// multiplies it into every problem's gathered vector with its own accumulator.
// GS = 8: the shared matrices cross from L2 once per group instead of once per
// problem, and the per-entry index arithmetic is paid once per group.  GS = 1:
// one problem per block, more blocks and eight rows per lane group in flight
// (the per-problem form).  Each problem's row sum keeps the per-problem order
// (lane-strided entries, then the lane tree) in both.
constexpr int kBGroup = 8;         // problems per block of the grouped form
#ifndef PCFD_BELL_ROUNDS
#define PCFD_BELL_ROUNDS 2
#endif
template <int GS>
__host__ __device__ constexpr int b_ell_rounds() { return GS == 1 ? 8 : PCFD_BELL_ROUNDS; }   // rounds of kBThreads / L rows

// What the fine level's weighted inverse diagonal (b_wdinv) needs, held by a
// coarse-level block: the structure's geometry scalars in registers and its
// weight table in shared memory.
struct BFineW {
  int nx, ny, any_dir;
  double w0;
  const double* wtab;
};

// The group's vectors for one op, filled from the problem records by the first
// GS threads; a null output marks a member that is absent or not solving.
template <class T, int GS>
struct BGroup {
  const T* src[GS];   // gathered vector
  const T* b[GS];     // the level's right-hand side (or r on level 0)
  T* out[GS];
  T* out2[GS];
  T mr[GS];           // fluid mean of r (projected level-0 right-hand side)
};

// Fill member g (thread g of the block) for op OP at depth d.
template <class T, int OP, int GS>
__device__ __forceinline__ void b_group_fill(BGroup<T, GS>& G, int g, const BProb<T>* P, int d, int src, int dst) {
  G.src[g] = nullptr;
  G.b[g] = nullptr;
  G.out[g] = nullptr;
  G.out2[g] = nullptr;
  G.mr[g] = (T)0;
  if (!P) return;
  if ((OP == EO_PROLONGW && d == 0) || (OP == EO_FRESTRICT && d == 1)) {
    G.b[g] = P->r;
    G.mr[g] = (T)(P->singular ? P->S[S_MEAN_R] : 0.0);
  }
  switch (OP) {
    case EO_PROLONG:
    case EO_PROLONGW:
      G.src[g] = b_lvl_x(*P, d + 1, src);
      G.out[g] = d == 0 ? b_fine_buf(*P, dst) : b_lvl_x(*P, d, dst);
      if (OP == EO_PROLONGW && d > 0) G.b[g] = P->lb[d];
      break;
    case EO_FRESTRICT:
      G.out[g] = P->lb[d];
      if (d > 1) G.src[g] = P->lb[d - 1];
      break;
    case EO_RESTRICT:
      G.out[g] = P->lb[d];
      G.src[g] = P->lres[d - 1];
      break;
    case EO_PRE:
      G.b[g] = P->lb[d];
      G.out[g] = P->lxa[d];
      G.out2[g] = P->lres[d];
      break;
    case EO_SMOOTH:
      G.src[g] = b_lvl_x(*P, d, src);
      G.b[g] = P->lb[d];
      G.out[g] = b_lvl_x(*P, d, dst);
      break;
    default:   // EO_RESID
      G.src[g] = b_lvl_x(*P, d, src);
      G.b[g] = P->lb[d];
      G.out[g] = P->lres[d];
      break;
  }
}

// b_ell_rounds<GS>() rounds of kBThreads / L rows of row block rb of matrix E,
// for every member of the group.  L lanes per row fixed at compile time (L > 1:
// row-major entries, L = 1: column-major).  All rounds gather first and store
// after: the group's vectors are reached through pointers the compiler cannot
// prove disjoint from the outputs, so a store between rounds would hold back
// the next round's loads.  A lane takes its entries four at a time, the four
// (value, column) pairs loaded together and then every member's four gathers,
// so a row costs one dependent load pair per four entries per lane.
template <int L, int OP, int GS, class T>
__device__ __forceinline__ void b_ellg_rows(const BProb<T>& P0, const BFineW& fw, const uint8_t* __restrict__ flags,
                                            const BGroup<T, GS>& G, const Ell<T>& E,
                                            const T* __restrict__ wd, int d, int rb) {
  constexpr int per = kBThreads / L;
  constexpr int ROUNDS = b_ell_rounds<GS>();
  const int lane = (int)threadIdx.x & (L - 1);
  const bool fr1 = OP == EO_FRESTRICT && d == 1;   // gathers the projected fine CG residual
  const T* src[GS];
  T mr[GS];
#pragma unroll
  for (int g = 0; g < GS; ++g) {
    const bool on = G.out[g] != nullptr;
    src[g] = on ? (OP == EO_PRE || fr1 ? G.b[g] : G.src[g]) : nullptr;
    mr[g] = G.mr[g];
  }
  const int K = E.K, n = E.n;
  T acc[ROUNDS][GS];
#pragma unroll
  for (int rd = 0; rd < ROUNDS; ++rd) {
    const int row = (rb * ROUNDS + rd) * per + (int)threadIdx.x / L;
#pragma unroll
    for (int g = 0; g < GS; ++g) acc[rd][g] = (T)0;
    if (row >= n) continue;
    for (int k0 = L > 1 ? lane : 0; k0 < K; k0 += 4 * L) {
      T vv[4];
      int cc[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int k = k0 + q * L;
        const bool ok = k < K;
        const long at = L > 1 ? (long)row * K + k : (long)k * n + row;
        vv[q] = ok ? E.val[at] : (T)0;
        cc[q] = ok ? E.col[at] : 0;
      }
      T sc[4];   // the per-column factor shared by the group (W on a coarse level)
      bool sv[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        sc[q] = OP == EO_PRE ? wd[cc[q]] : (T)1;
        sv[q] = fr1 ? (flags[cc[q]] & F_SOLV) != 0 : true;
      }
#pragma unroll
      for (int g = 0; g < GS; ++g) {
        if (!src[g]) continue;
        T gv[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) gv[q] = src[g][cc[q]];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          T x = gv[q];
          if (OP == EO_PRE) x = sc[q] * x;
          if (fr1) x = sv[q] ? x - mr[g] : (T)0;
          acc[rd][g] += vv[q] * x;
        }
      }
    }
  }
#pragma unroll
  for (int rd = 0; rd < ROUNDS; ++rd)
#pragma unroll
    for (int g = 0; g < GS; ++g)
#pragma unroll
      for (int o = L / 2; o > 0; o >>= 1) acc[rd][g] += __shfl_xor_sync(0xffffffffu, acc[rd][g], o, L);
  if (lane != 0) return;
#pragma unroll
  for (int rd = 0; rd < ROUNDS; ++rd) {
    const int row = (rb * ROUNDS + rd) * per + (int)threadIdx.x / L;
    if (row >= n) continue;
    // the row's W (fine level: b_wdinv of the cell, from the block's copy of the
    // weight table) and solvable flag, formed once for the group
    T wrow = (T)0;
    bool srow = true;
    if (OP == EO_PROLONGW && d == 0) {
      const uint8_t f = flags[row];
      srow = (f & F_SOLV) != 0;
      double w = fw.w0 * (1.0 / 1.0);
      if (srow) {
        const int i = row / fw.ny, j = row - i * fw.ny;
        if (fw.any_dir && (i == 0 || j == 0 || i == fw.nx - 1 || j == fw.ny - 1))
          w = fw.w0 * (1.0 / fine_diag(f, i, j, P0.g));
        else
          w = fw.wtab[f & 15];
      }
      wrow = (T)w;
    } else if (OP == EO_PROLONGW) {
      wrow = wd[row];
    }
#pragma unroll
    for (int g = 0; g < GS; ++g) {
      T* __restrict__ o = G.out[g];
      if (!o) continue;
      const T s = acc[rd][g];
      switch (OP) {
        case EO_PROLONG: o[row] = o[row] + s; break;
        case EO_PROLONGW: {
          T wb;
          if (d == 0) {
            const T bfr = srow ? G.b[g][row] - mr[g] : (T)0;
            wb = wrow * bfr;
          } else {
            wb = wrow * G.b[g][row];
          }
          o[row] = wb + s;
          break;
        }
        case EO_FRESTRICT:
        case EO_RESTRICT: o[row] = s; break;
        case EO_PRE: {
          const T bx = G.b[g][row];
          o[row] = wd[row] * bx;
          G.out2[g][row] = bx - s;
          break;
        }
        case EO_SMOOTH: {
          const T xr = G.src[g][row];
          o[row] = xr + wd[row] * (G.b[g][row] - s);
          break;
        }
        default: o[row] = G.b[g][row] - s; break;   // EO_RESID
      }
    }
  }
}

// One ELL op at depth d over the map's (structure, row block x 1024 + group)
// entries.  Members: sprobs[H.sp0 + group * GS + g], g < GS.
// Resident blocks per SM of the coarse-level ELL kernels: the same latency
// argument; 2 / 4 / 5 / 6 / 8 blocks per SM step the batch in 26.5 / 21.2 /
// 19.8 / 20.1 / 20.1 ms (strip kernels at 4).
#ifndef PCFD_BELL_MINB
#define PCFD_BELL_MINB 5
#endif
template <class T, int OP, int GS>
__global__ void __launch_bounds__(kBThreads, PCFD_BELL_MINB) k_b_ellg(const BProb<T>* __restrict__ probs,
                                                       const BHier<T>* __restrict__ hiers,
                                                       const int2* __restrict__ map,
                                                       const int* __restrict__ sprobs, int d, int src,
                                                       int dst, BShared sh) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  const int2 e = map[blockIdx.x];
  const BHier<T>& H = hiers[e.x];
  const int rb = e.y >> 10, grp = e.y & 1023;
  __shared__ BGroup<T, GS> G;
  __shared__ int any;
  // The level's matrix (copied by value), its weights and the structure's leader
  // record (geometry and flags) are loaded by every thread before the barrier, in
  // parallel with warp 0 gathering the group's members.
  const bool pl = OP == EO_PROLONG || OP == EO_PROLONGW;
  const BLevel<T>& Lm = pl ? H.lv[d + 1] : H.lv[d];
  const Ell<T> E = pl ? Lm.P : OP == EO_RESTRICT ? Lm.R : OP == EO_FRESTRICT ? Lm.M : Lm.A;
  const int Lop = pl ? Lm.lp : OP == EO_RESTRICT ? Lm.lr : OP == EO_FRESTRICT ? Lm.lm : Lm.la;
  const T* wd = d > 0 ? H.lv[d].wd : nullptr;
  const BProb<T>& P0 = probs[sprobs[H.sp0 + grp * GS]];   // the structure's geometry and flags
  const uint8_t* flags0 = P0.flags;
  __shared__ double wt0[16];
  if (OP == EO_PROLONGW && d == 0 && threadIdx.x >= 32 && threadIdx.x < 48) wt0[threadIdx.x - 32] = P0.wtab[threadIdx.x - 32];
  const BFineW fw{P0.g.nx, P0.g.ny, P0.any_dir, P0.w0, wt0};
  if (threadIdx.x < 32) {   // GS <= 32: the members are lanes of warp 0
    const int k = grp * GS + (int)threadIdx.x;
    const BProb<T>* P = nullptr;
    if ((int)threadIdx.x < GS && k < H.spn) {
      const int pi = sprobs[H.sp0 + k];
      if (b_solving(sh, pi)) P = probs + pi;
    }
    if ((int)threadIdx.x < GS) b_group_fill<T, OP, GS>(G, (int)threadIdx.x, P, d, src, dst);
    const unsigned on = __ballot_sync(0xffffffffu, P != nullptr);
    if (threadIdx.x == 0) any = on != 0u;
  }
  __syncthreads();
  if (!any) return;
  switch (Lop) {
    case 1: b_ellg_rows<1, OP, GS>(P0, fw, flags0, G, E, wd, d, rb); break;
    case 4: b_ellg_rows<4, OP, GS>(P0, fw, flags0, G, E, wd, d, rb); break;
    case 8: b_ellg_rows<8, OP, GS>(P0, fw, flags0, G, E, wd, d, rb); break;
    case 16: b_ellg_rows<16, OP, GS>(P0, fw, flags0, G, E, wd, d, rb); break;
    default: b_ellg_rows<32, OP, GS>(P0, fw, flags0, G, E, wd, d, rb); break;
  }
}

// Coarsest level d of the problems whose structure has no dense tail: the
// restriction from level d - 1 and the dense pseudo-inverse, one block per problem.
template <class T>
__global__ void __launch_bounds__(kBThreads) k_b_coarsest(const BProb<T>* __restrict__ probs,
                                                           const int2* __restrict__ map, int d, BShared sh) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  extern __shared__ double sb[];
  const int2 e = map[blockIdx.x];
  if (!b_solving(sh, e.x)) return;
  const BProb<T>& P = probs[e.x];
  const BLevel<T>& Lc = P.lv[d];
  const T* res = P.lres[d - 1];
  const int L = Lc.lr, lane = threadIdx.x & (L - 1);
  const int per = kBThreads / L;
  for (int base = 0; base < Lc.R.n; base += per) {
    const int row = base + (int)threadIdx.x / L;
    const T s = b_ell_row(Lc.R, L, row, lane, [&](int c) { return res[c]; });
    if (lane == 0 && row < Lc.R.n) {
      sb[row] = (double)s;
      P.lb[d][row] = s;
    }
  }
  __syncthreads();
  const int wl = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = kBThreads >> 5;
  const int n = Lc.R.n;
  for (int row = warp; row < n; row += nw) {
    double acc = 0.0;
    for (int k = wl; k < n; k += 32) acc += (double)P.C[(long)row * n + k] * sb[k];
    acc = warp_sum(acc);
    if (wl == 0) P.lxa[d][row] = (T)acc;
  }
}

// Dense close of the V-cycle on the tensor cores: X_t = M B_t for every tailed
// structure, where M (n x n, row-major) is the structure's operator of the cycle
// at and below its tail depth t and the columns of B_t are the level-t
// right-hand sides of its problems -- a matrix product with the problems as the
// N dimension.  One launch after the down sweep covers every structure.  A block
// takes a kTailBM = 16-row tile of M against a kTailBN = 32-problem column tile;
// its 8 warps split K (warp w takes the K chunks w, w + 8, ...) and load their
// MMA fragments straight from global memory (M and the vectors sit in L2; each
// chunk's loads are all issued before its MMAs, and no barrier is taken inside
// the K loop), then the eight partial tiles are summed through shared memory in
// warp order, so the result is deterministic.  FP64 form: DMMA (mma m8n8k4 f64,
// FP64 products and sums).  Mixed form: three TF32 MMAs per product (m16n8k8;
// each FP32 operand split into a TF32 head and a TF32 remainder,
// head*head + head*rem + rem*head) so the result keeps FP32 accuracy and the
// preconditioner its FP32 behaviour.
constexpr int kTailBM = 16, kTailBN = 32, kTailThreads = 256;
constexpr int kBTailGroup = kTailBN;   // problems per column tile of the tail launch

template <class T> struct TailK;
template <> struct TailK<float> { static constexpr int KW = 32; };    // K per warp chunk: 4 m16n8k8 steps
template <> struct TailK<double> { static constexpr int KW = 16; };   // 4 m8n8k4 steps

__device__ __forceinline__ uint32_t b_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void b_mma_tf32(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void b_mma_f64(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

template <class T>
__device__ __forceinline__ T b_ld_or0(const T* p, bool ok) {
  return ok ? __ldg(p) : (T)0;
}

template <class T>
__global__ void __launch_bounds__(kTailThreads) k_b_tail(const BProb<T>* __restrict__ probs,
                                                          const BHier<T>* __restrict__ hiers,
                                                          const int2* __restrict__ map,
                                                          const int* __restrict__ sprobs, BShared sh) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  constexpr int KW = TailK<T>::KW;
  constexpr int NW = kTailThreads / 32;
  const int2 e = map[blockIdx.x];   // (structure, row tile * 64 + column tile)
  const BHier<T>& H = hiers[e.x];
  const int d = H.tail_level;
  const int n = H.tail_n;
  const int r0 = (e.y >> 6) * kTailBM, ct = e.y & 63;
  __shared__ const T* sb[kTailBN];
  __shared__ T* sx[kTailBN];
  __shared__ int any;
  __shared__ __align__(16) T red[NW][16 * 32];   // each warp's partial 16 x 32 tile, fragment order
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  if (threadIdx.x < kTailBN) {
    const int k = ct * kTailBN + (int)threadIdx.x;
    const T* b = nullptr;
    T* x = nullptr;
    if (k < H.spn) {
      const int pi = sprobs[H.sp0 + k];
      if (b_solving(sh, pi)) {
        b = probs[pi].lb[d];
        x = probs[pi].lxa[d];
        any = 1;
      }
    }
    sb[threadIdx.x] = b;
    sx[threadIdx.x] = x;
  }
  __syncthreads();
  if (!any) return;   // block-uniform
  const int warp = (int)(threadIdx.x >> 5), lane = (int)(threadIdx.x & 31);
  const int g = lane >> 2, t = lane & 3;
  const T* __restrict__ M = H.tail;
  const bool ok0 = r0 + g < n, ok1 = r0 + g + 8 < n;
  const T* m0 = M + (long)(ok0 ? r0 + g : 0) * n;
  const T* m1 = M + (long)(ok1 ? r0 + g + 8 : 0) * n;
  const T* bq[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) bq[q] = sb[q * 8 + g];
  T* out = &red[warp][0];
  if constexpr (sizeof(T) == 4) {
    float acc[4][4];   // [n tile][fragment]
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[q][i] = 0.f;
    for (int k0 = warp * KW; k0 < n; k0 += NW * KW) {
      float av[4][4], bv[4][4][2];
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int ka = k0 + s * 8 + t, kb = ka + 4;
        av[s][0] = b_ld_or0(m0 + ka, ok0 && ka < n);
        av[s][1] = b_ld_or0(m1 + ka, ok1 && ka < n);
        av[s][2] = b_ld_or0(m0 + kb, ok0 && kb < n);
        av[s][3] = b_ld_or0(m1 + kb, ok1 && kb < n);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          bv[s][q][0] = b_ld_or0(bq[q] + ka, bq[q] && ka < n);
          bv[s][q][1] = b_ld_or0(bq[q] + kb, bq[q] && kb < n);
        }
      }
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        uint32_t ah[4], al[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          ah[i] = b_tf32(av[s][i]);
          al[i] = b_tf32(av[s][i] - __uint_as_float(ah[i]));
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const uint32_t bh0 = b_tf32(bv[s][q][0]), bh1 = b_tf32(bv[s][q][1]);
          const uint32_t bl0 = b_tf32(bv[s][q][0] - __uint_as_float(bh0));
          const uint32_t bl1 = b_tf32(bv[s][q][1] - __uint_as_float(bh1));
          b_mma_tf32(acc[q], al, bh0, bh1);
          b_mma_tf32(acc[q], ah, bl0, bl1);
          b_mma_tf32(acc[q], ah, bh0, bh1);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int i = 0; i < 4; ++i) out[(q * 4 + i) * 32 + lane] = acc[q][i];
  } else {
    double acc[2][4][2];   // [m tile][n tile][fragment]
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[m][q][0] = acc[m][q][1] = 0.0;
    for (int k0 = warp * KW; k0 < n; k0 += NW * KW) {
      double av[4][2], bv[4][4];
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int k = k0 + s * 4 + t;
        av[s][0] = b_ld_or0(m0 + k, ok0 && k < n);
        av[s][1] = b_ld_or0(m1 + k, ok1 && k < n);
#pragma unroll
        for (int q = 0; q < 4; ++q) bv[s][q] = b_ld_or0(bq[q] + k, bq[q] && k < n);
      }
#pragma unroll
      for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          b_mma_f64(acc[0][q], av[s][0], bv[s][q]);
          b_mma_f64(acc[1][q], av[s][1], bv[s][q]);
        }
    }
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int i = 0; i < 2; ++i) out[((m * 4 + q) * 2 + i) * 32 + lane] = acc[m][q][i];
  }
  __syncthreads();
  // the partial tiles summed in warp order; slot -> (lane, fragment) -> (row, problem)
  for (int idx = threadIdx.x; idx < 16 * 32; idx += kTailThreads) {
    T v = red[0][idx];
#pragma unroll
    for (int w = 1; w < NW; ++w) v += red[w][idx];
    const int f = idx >> 5, l = idx & 31, lg = l >> 2, lt = l & 3;
    int row, col;
    if constexpr (sizeof(T) == 4) {   // f = q * 4 + i: rows g, g + 8; columns 2t, 2t + 1 of n tile q
      const int q = f >> 2, i = f & 3;
      row = lg + ((i & 2) ? 8 : 0);
      col = q * 8 + 2 * lt + (i & 1);
    } else {                          // f = (m * 4 + q) * 2 + i: row 8m + g; columns 2t, 2t + 1 of n tile q
      const int m = f >> 3, q = (f >> 1) & 3, i = f & 1;
      row = 8 * m + lg;
      col = q * 8 + 2 * lt + i;
    }
    T* x = sx[col];
    if (x && r0 + row < n) x[r0 + row] = v;
  }
}

// Coarse levels of the V-cycle, one thread block per problem: levels
// d0 = min(dc, coarsest) .. coarsest of every solving problem run inside one
// block, phases separated by __syncthreads -- restriction from the residual of
// level d0 - 1, first sweep + residual (more sweeps if asked), down to the
// coarsest dense solve, then prolongation and smoothing back up to d0.  These
// levels hold few rows, so one launch for all problems replaces a launch per
// phase and level; their vectors and the shared matrices stay in L2.  The
// result at d0 lands in the buffer the per-level path would leave it in
// (b_coarse_final), so the prolongation into d0 - 1 is unchanged.  Measured on
// the 256-cavity batch this form is slower than per-level launches (one SM
// carries a problem's whole coarse cycle, and the largest problems set the
// launch's length), so it is an option, not the default.
constexpr int kBCoarseThreads = 512;

__host__ __device__ inline int b_coarse_final(int sweeps) {
  // down: the first sweep writes xa, each further one swaps; up: every sweep swaps
  return (((sweeps - 1) & 1) + sweeps) & 1;
}

template <class T, class X, class W>
__device__ __forceinline__ void b_blk_ell(const Ell<T>& E, int L, X x, W write) {
  const int lane = threadIdx.x & (L - 1), per = blockDim.x / L;
  for (int base = 0; base < E.n; base += per) {
    const int row = base + (int)threadIdx.x / L;
    const T s = b_ell_row(E, L, row, lane, x);
    if (lane == 0 && row < E.n) write(row, s);
  }
}

template <class T>
__global__ void __launch_bounds__(kBCoarseThreads) k_b_coarse(const BProb<T>* __restrict__ probs,
                                                               const int* __restrict__ order, int dc,
                                                               int sweeps, BShared sh) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  extern __shared__ double sb[];
  const int p = order[blockIdx.x];
  if (!b_solving(sh, p)) return;
  const BProb<T>& P = probs[p];
  const int c = P.nlev - 1;
  const int d0 = min(dc, c);
  int cur[kBMaxLevels];
  // ---- down ----
  for (int l = d0; l <= c; ++l) {
    const BLevel<T>& Lv = P.lv[l];
    const T* __restrict__ src = P.lres[l - 1];
    T* __restrict__ bl = P.lb[l];
    const bool coarsest = l == c;
    b_blk_ell(Lv.R, Lv.lr, [&](int k) { return src[k]; }, [&](int row, T s) {
      bl[row] = s;
      if (coarsest) sb[row] = (double)s;
    });
    __syncthreads();
    if (coarsest) {
      const int wl = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
      const int n = Lv.R.n;
      T* __restrict__ xo = P.lxa[l];
      for (int row = warp; row < n; row += nw) {
        double acc = 0.0;
        for (int k = wl; k < n; k += 32) acc += (double)P.C[(long)row * n + k] * sb[k];
        acc = warp_sum(acc);
        if (wl == 0) xo[row] = (T)acc;
      }
      __syncthreads();
      cur[l] = 0;
      break;
    }
    const T* __restrict__ wd = Lv.wd;
    T* __restrict__ xa = P.lxa[l];
    T* __restrict__ xb = P.lxb[l];
    T* __restrict__ rs = P.lres[l];
    b_blk_ell(Lv.A, Lv.la, [&](int k) { return wd[k] * bl[k]; }, [&](int row, T s) {
      const T bx = bl[row];
      xa[row] = wd[row] * bx;
      rs[row] = bx - s;
    });
    __syncthreads();
    int a = 0;
    if (sweeps > 1) {
      for (int k = 1; k < sweeps; ++k) {
        const T* xi = a == 0 ? xa : xb;
        T* xn = a == 0 ? xb : xa;
        b_blk_ell(Lv.A, Lv.la, [&](int q) { return xi[q]; }, [&](int row, T s) {
          xn[row] = xi[row] + wd[row] * (bl[row] - s);
        });
        __syncthreads();
        a ^= 1;
      }
      const T* xi = a == 0 ? xa : xb;
      b_blk_ell(Lv.A, Lv.la, [&](int q) { return xi[q]; },
                [&](int row, T s) { rs[row] = bl[row] - s; });
      __syncthreads();
    }
    cur[l] = a;
  }
  // ---- up ----
  for (int l = c - 1; l >= d0; --l) {
    const BLevel<T>& Lv = P.lv[l];
    const BLevel<T>& Lc = P.lv[l + 1];
    const T* __restrict__ xc = (l + 1 == c || cur[l + 1] == 0) ? P.lxa[l + 1] : P.lxb[l + 1];
    T* xa = P.lxa[l];
    T* xb = P.lxb[l];
    int a = cur[l];
    {
      T* __restrict__ xf = a == 0 ? xa : xb;
      b_blk_ell(Lc.P, Lc.lp, [&](int k) { return xc[k]; },
                [&](int row, T s) { xf[row] = xf[row] + s; });
      __syncthreads();
    }
    const T* __restrict__ wd = Lv.wd;
    const T* __restrict__ bl = P.lb[l];
    for (int k = 1; k <= sweeps; ++k) {
      const T* xi = a == 0 ? xa : xb;
      T* xn = a == 0 ? xb : xa;
      b_blk_ell(Lv.A, Lv.la, [&](int q) { return xi[q]; }, [&](int row, T s) {
        xn[row] = xi[row] + wd[row] * (bl[row] - s);
      });
      __syncthreads();
      a ^= 1;
    }
    cur[l] = a;
  }
}

// Per-problem status for the host: frozen flag, steps, solver iterations of
// the last step, status, clock and dt.
template <class T>
__global__ void k_b_gather(const BProb<T>* __restrict__ probs, int nprob, int* __restrict__ iout,
                           double* __restrict__ dout) {
  pdl_begin();   // programmatic dependent launch: the predecessor's results first
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nprob) return;
  const BProb<T>& P = probs[k];
  iout[4 * k + 0] = P.I[I_FROZEN];
  iout[4 * k + 1] = P.I[I_STEPS];
  iout[4 * k + 2] = P.I[I_TOTAL_IT];
  iout[4 * k + 3] = P.I[I_STATUS];
  dout[2 * k + 0] = P.S[S_T];
  dout[2 * k + 1] = P.S[S_DT];
}

}  // namespace pcfd
