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
constexpr int kBEllRounds = 8;   // ELL blocks: rounds of kBThreads / L rows each

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
  // Per-problem flags indexed by problem, mirrored from the scalar block by the
  // kernels that change them: a block learns whether its problem takes part
  // from one load beside its map entry instead of a chain through the record.
  uint8_t* frozen;       // I_FROZEN != 0
  uint8_t* solving;      // not frozen and the current solve not done
};

enum BTicket { TK_CG = 0, TK_IR = 1, TK_ARM = 2, TK_COUNT = 4 };

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
// and at `cap` passes the loop ends whatever the flags say (each problem's
// own iteration limit ends it first; the cap only bounds the device loop).
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
    if (any && it >= (unsigned)cap) {
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
// geometry and tile shape in registers, the diagonal tables in shared memory.
// The record lives in global memory, and a loop that stores to the problem's
// vectors cannot keep record fields in registers by itself (the stores might
// alias it), so without the copy every cell would reload them.
struct BView {
  Geo g;
  int any_dir;
  double w0;
  const double* dtab;
  const double* wtab;
  int tile_i, tiles_i, tiles_j, tiles, chunk_tiles;
};

// Declares `V` for problem record P; every thread of the block must reach it.
#define B_VIEW(V, P)                                                                           \
  __shared__ double V##_dt[16], V##_wt[16];                                                    \
  if (threadIdx.y == 0 && threadIdx.x < 16) {                                                  \
    V##_dt[threadIdx.x] = (P).dtab[threadIdx.x];                                               \
    V##_wt[threadIdx.x] = (P).wtab[threadIdx.x];                                               \
  }                                                                                            \
  __syncthreads();                                                                             \
  const BView V{(P).g, (P).any_dir, (P).w0, V##_dt, V##_wt, (P).tile_i, (P).tiles_i, (P).tiles_j, \
                (P).tiles, (P).chunk_tiles}

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
template <class A, class X>
__device__ __forceinline__ A b_apply(const BView& V, uint8_t f, int i, int j, int c, X x) {
  const Geo& g = V.g;
  A acc = (A)b_diag(V, f, i, j) * x(c, i, j);
  if (f & F_W) { const int a = wrap_w(i, g); acc += (A)g.cx * x(a * g.ny + j, a, j); }
  if (f & F_E) { const int a = wrap_e(i, g); acc += (A)g.cx * x(a * g.ny + j, a, j); }
  if (f & F_S) { const int b = wrap_s(j, g); acc += (A)g.cy * x(i * g.ny + b, i, b); }
  if (f & F_N) { const int b = wrap_n(j, g); acc += (A)g.cy * x(i * g.ny + b, i, b); }
  return acc;
}

// ---- staged fine tiles --------------------------------------------------------
// The stencil kernels stage a tile's values once in shared memory, with a one-
// cell halo, instead of rebuilding every neighbour's value per cell: sm[li][lj]
// holds v at cell (i0 + li - 1, j0 + lj - 1).  Outside the domain the halo
// wraps where the axis is periodic; elsewhere it holds 0 -- a face flag is
// clear there, so the value is never read.
constexpr int kBHaloJ = kBTileJ + 2;
constexpr int kBHaloRows = 64 + 2;   // the largest tile height, plus the halo

template <class T, class F>
__device__ __forceinline__ void b_stage(T (*sm)[kBHaloJ], const BView& V, int i0, int j0, int rows, F v) {
  const int nx = V.g.nx, ny = V.g.ny;
  const int total = (rows + 2) * kBHaloJ;
#pragma unroll 4
  for (int idx = (int)(threadIdx.y * kBTileJ + threadIdx.x); idx < total; idx += kBThreads) {
    const int li = idx / kBHaloJ, lj = idx - li * kBHaloJ;
    int i = i0 + li - 1, j = j0 + lj - 1;
    bool ok = true;
    if (i < 0) {
      ok = V.g.periodic_x != 0;
      i = nx - 1;
    } else if (i >= nx) {
      ok = V.g.periodic_x && i == nx;
      i = 0;
    }
    if (j < 0) {
      ok = ok && V.g.periodic_y;
      j = ny - 1;
    } else if (j >= ny) {
      ok = ok && V.g.periodic_y && j == ny;
      j = 0;
    }
    sm[li][lj] = ok ? v(i * ny + j, i, j) : (T)0;
  }
}

// (A x)_c from a staged tile, fine_apply's terms in its order.
template <class A, class T>
__device__ __forceinline__ A b_apply_sm(const BView& V, uint8_t f, int i, int j, const T (*sm)[kBHaloJ], int li,
                                        int lj) {
  A acc = (A)b_diag(V, f, i, j) * (A)sm[li][lj];
  if (f & F_W) acc += (A)V.g.cx * (A)sm[li - 1][lj];
  if (f & F_E) acc += (A)V.g.cx * (A)sm[li + 1][lj];
  if (f & F_S) acc += (A)V.g.cy * (A)sm[li][lj - 1];
  if (f & F_N) acc += (A)V.g.cy * (A)sm[li][lj + 1];
  return acc;
}

// A thread's cells of a tile in batches of kBCellBatch rows: load(u, c) for
// every cell of the batch first (independent loads in flight), then body(u, c,
// i, j, li, lj) in row order -- the order a plain row loop visits them.
constexpr int kBCellBatch = 4;

template <class Load, class Body>
__device__ __forceinline__ void b_tile_cells(const BView& V, int i0, int j0, int rows, Load load, Body body) {
  const int j = j0 + (int)threadIdx.x, lj = (int)threadIdx.x + 1;
  if (j >= V.g.ny) return;
  for (int l0 = 1 + (int)threadIdx.y; l0 <= rows; l0 += kBCellBatch * kBThreadsI) {
    int c[kBCellBatch];
#pragma unroll
    for (int u = 0; u < kBCellBatch; ++u) {
      const int li = l0 + u * kBThreadsI;
      c[u] = (i0 + li - 1) * V.g.ny + j;
      if (li <= rows) load(u, c[u]);
    }
#pragma unroll
    for (int u = 0; u < kBCellBatch; ++u) {
      const int li = l0 + u * kBThreadsI;
      if (li <= rows) body(u, c[u], i0 + li - 1, j, li, lj);
    }
  }
}

// The tiles of a chunk (block-uniform), optionally staged: with a value
// function `val`, each tile's values and halo go to `sm` first.  Every thread
// of the block runs the same tiles (the barriers need them all).
template <bool STAGE, class T, class Val, class Load, class Body>
__device__ __forceinline__ void b_chunk_cells(const BView& V, int chunk, T (*sm)[kBHaloJ], Val val, Load load,
                                              Body body) {
  for (int tile = chunk * V.chunk_tiles, tend = min(V.tiles, tile + V.chunk_tiles); tile < tend; ++tile) {
    const int ti = tile / V.tiles_j, tj = tile - ti * V.tiles_j;
    const int i0 = ti * V.tile_i, j0 = tj * kBTileJ;
    const int rows = min(V.tile_i, V.g.nx - i0);
    if (STAGE) {
      __syncthreads();
      b_stage(sm, V, i0, j0, rows, val);
      __syncthreads();
    }
    b_tile_cells(V, i0, j0, rows, load, body);
  }
}

// ---- step bookkeeping -------------------------------------------------------
// max|u|, max|v| over the physical faces and the non-finite count of u, v, p:
// the inputs of the time-step control (pycfd/core/timestepper.py:94-142).
template <class T>
__global__ void __launch_bounds__(kBThreads) k_b_stats(const BProb<T>* __restrict__ probs,
                                                        const int2* __restrict__ map, BShared sh) {
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
template <class T>
__global__ void __launch_bounds__(kBThreads) k_b_predictor(const BProb<T>* __restrict__ probs,
                                                            const int2* __restrict__ map, int src_a,
                                                            int src_b, double ca, double cb, int dst,
                                                            BShared sh) {
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (b_frozen(sh, e.x)) return;
  const Geo& g = P.g;
  const int nx = g.nx, ny = g.ny;
  const StageIn u{b_arr_u(P, src_a), src_b >= 0 ? b_arr_u(P, src_b) : nullptr, ca, cb};
  const StageIn v{b_arr_v(P, src_a), src_b >= 0 ? b_arr_v(P, src_b) : nullptr, ca, cb};
  double* us = b_arr_u(P, dst);
  double* vs = b_arr_v(P, dst);
  const double dt = P.S[S_DT], blend = P.S[S_BLEND];
  B_CHUNK_TILES(P, e.y) {
    B_TILE_EXT(P, tile_, nx + 3, ny + 3) {
      if (j < ny + 2) {
        const long k = (long)i * (ny + 2) + j;
        double val = u[k];
        if (i >= g.u_lo && i < g.u_hi && j >= 1 && j <= ny)
          val = val + dt * rhs_u_at(u, v, i, j, ny, g.dx, g.dy, g.nu, blend, g.fx);
        us[k] = val;
      }
      if (i < nx + 2) {
        const long k = (long)i * (ny + 3) + j;
        double val = v[k];
        if (i >= 1 && i <= nx && j >= g.v_lo && j < g.v_hi)
          val = val + dt * rhs_v_at(u, v, i, j, ny, g.dx, g.dy, g.nu, blend, g.fy);
        vs[k] = val;
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
template <class T>
__global__ void __launch_bounds__(kBThreads) k_b_div_rhs(const BProb<T>* __restrict__ probs,
                                                          const int2* __restrict__ map, int arr,
                                                          BShared sh) {
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (b_frozen(sh, e.x)) return;
  const Geo& g = P.g;
  const double* u = b_arr_u(P, arr);
  const double* v = b_arr_v(P, arr);
  const double dt = P.S[S_DT];
  double acc[1] = {0.0};
  {
    B_CHUNK_TILES(P, e.y) {
      B_TILE_CELLS(P, tile_) {
        const int c = i * g.ny + j;
        const uint8_t f = P.flags[c];
        double val = 0.0;
        if (f & F_SOLV) {
          val = (cell_div(u, v, i, j, g.ny, g.dx, g.dy) / dt) * 1.0 + fine_bc(f, i, j, g);
          acc[0] += val;
        }
        P.b[c] = val;
      }
    }
  }
  b_reduce<1>(acc, sh.partials + (long)P.red_base * 8, P.counter, e.y, P.chunks,
              [&](double* t) { P.S[S_MEAN_B] = g.n_fluid ? t[0] / g.n_fluid : 0.0; });
}

// Velocity correction on the solvable faces and the interior of p
// (pycfd/core/solver.py:665-682); the ghost ring follows in k_b_boundary.
template <class T>
__global__ void __launch_bounds__(kBThreads) k_b_correct(const BProb<T>* __restrict__ probs,
                                                          const int2* __restrict__ map, int arr,
                                                          BShared sh) {
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
        P.u[k] = ca * P.u[k] + cb * bu[k];
      }
      if (i < nx + 2) {
        const long k = (long)i * (ny + 3) + j;
        P.v[k] = ca * P.v[k] + cb * bv[k];
      }
    }
  }
}

// ---- FP64 MG-PCG ---------------------------------------------------------------
// b <- b - mean (solvable rows), r = b - A x from the warm start x, norms and
// the convergence test before the first pass (scipy cg, pressure.py:300-308).
template <class T>
__global__ void __launch_bounds__(kBThreads) k_b_rhs_init(const BProb<T>* __restrict__ probs,
                                                           int nprob, const int2* __restrict__ map,
                                                           double tol, int maxiter, BShared sh,
                                                           LoopCtl loop) {
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (!b_frozen(sh, e.x)) {
    const Geo& g = P.g;
    const double mean = P.singular ? P.S[S_MEAN_B] : 0.0;
    double acc[3] = {0, 0, 0};
    {
      B_CHUNK_TILES(P, e.y) {
        B_TILE_CELLS(P, tile_) {
          const int c = i * g.ny + j;
          const uint8_t f = P.flags[c];
          const double bc = (f & F_SOLV) ? P.b[c] - mean : 0.0;
          P.b[c] = bc;
          const double ax = b_apply<double>(P, f, i, j, c, [&](int k, int, int) { return (double)P.xs[k]; });
          const double rc = bc - ax;
          P.r[c] = (T)rc;
          acc[0] += bc * bc;
          acc[1] += rc * rc;
          if (f & F_SOLV) acc[2] += rc;
        }
      }
    }
    b_reduce<3>(acc, sh.partials + (long)P.red_base * 8, P.counter, e.y, P.chunks, [&](double* t) {
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

// p = (z - mean z) + beta p_old on solvable rows, q = A p, p.q -> alpha.
template <class T>
__global__ void __launch_bounds__(kBThreads) k_b_cg_pq(const BProb<T>* __restrict__ probs,
                                                        const int2* __restrict__ map, BShared sh) {
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (!b_solving(sh, e.x)) return;
  B_VIEW(V, P);
  const int ny = V.g.ny;
  const bool first = P.I[I_IT] == 0;
  const double beta = first ? 0.0 : P.S[S_RHO] / P.S[S_RHO_PREV];
  const double mz = P.S[S_MEAN_Z];
  const uint8_t* __restrict__ flags = P.flags;
  const T* __restrict__ zraw = P.z;
  const T* __restrict__ p_old = P.pa;
  T* __restrict__ pn = P.pb;
  T* __restrict__ q = P.q;
  // arithmetic in T (FP32 in the mixed form's inner solve), p.q summed in FP64
  const T tb = (T)beta, tm = (T)mz;
  auto pval = [&](int k, int, int) -> T {   // all loads issued, then selected
    const uint8_t fk = flags[k];
    const T zk = zraw[k];
    const T pk = first ? (T)0 : p_old[k];
    const T z = (fk & F_SOLV) ? zk - tm : (T)0;
    if (first) return z;
    return pk * tb + z;
  };
  double acc[1] = {0.0};
  __shared__ T sm[kBHaloRows][kBHaloJ];
  uint8_t fv[kBCellBatch];
  b_chunk_cells<true>(V, e.y, sm, pval, [&](int u, int c) { fv[u] = flags[c]; },
                      [&](int u, int c, int i, int j, int li, int lj) {
                        const T pc = sm[li][lj];
                        const T qc = b_apply_sm<T>(V, fv[u], i, j, sm, li, lj);
                        pn[c] = pc;
                        q[c] = qc;
                        acc[0] += (double)pc * (double)qc;
                      });
  (void)ny;
  b_reduce<1>(acc, sh.partials + (long)P.red_base * 8, P.counter, e.y, P.chunks, [&](double* t) {
    P.S[S_PQ] = t[0];
    P.S[S_ALPHA] = P.S[S_RHO] / t[0];
  });
}

// x += alpha p, r -= alpha q, p kept for the next pass; ||r||^2 and sum(r);
// the next pass's convergence test; launch-wide loop decision.
template <class T>
__global__ void __launch_bounds__(kBThreads) k_b_cg_xr(const BProb<T>* __restrict__ probs, int nprob,
                                                        const int2* __restrict__ map, int maxiter,
                                                        BShared sh, LoopCtl loop) {
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (b_solving(sh, e.x)) {
    const Geo& g = P.g;
    B_VIEW(V, P);
    const int ny = V.g.ny;
    const double alpha = P.S[S_ALPHA];
    const uint8_t* __restrict__ flags = P.flags;
    const T* __restrict__ pn = P.pb;
    const T* __restrict__ q = P.q;
    T* __restrict__ pa = P.pa;
    T* __restrict__ xs = P.xs;
    T* __restrict__ r = P.r;
    double acc[2] = {0, 0};
    T pv[kBCellBatch], xv[kBCellBatch], rv[kBCellBatch], qv[kBCellBatch];
    uint8_t fv[kBCellBatch];
    b_chunk_cells<false, T>(
        V, e.y, nullptr, [](int, int, int) { return (T)0; },
        [&](int u, int c) {
          pv[u] = pn[c];
          xv[u] = xs[c];
          rv[u] = r[c];
          qv[u] = q[c];
          fv[u] = flags[c];
        },
        [&](int u, int c, int, int, int, int) {
          const T pc = pv[u];
          const double xc = (double)xv[u] + alpha * (double)pc;
          const double rc = (double)(T)((double)rv[u] - alpha * (double)qv[u]);
          pa[c] = pc;
          xs[c] = (T)xc;
          r[c] = (T)rc;
          acc[0] += rc * rc;
          if (fv[u] & F_SOLV) acc[1] += rc;
        });
    (void)ny;
    b_reduce<2>(acc, sh.partials + (long)P.red_base * 8, P.counter, e.y, P.chunks, [&](double* t) {
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
__global__ void __launch_bounds__(kBThreads) k_b_finish_stats(const BProb<T>* __restrict__ probs,
                                                               const int2* __restrict__ map, double tol,
                                                               BShared sh) {
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (b_frozen(sh, e.x)) return;
  const Geo& g = P.g;
  const bool zero = P.I[I_ZERO_RHS] != 0;
  const double* x = P.x;
  auto xv = [&](int k, int, int) -> double { return zero ? 0.0 : x[k]; };
  double acc[2] = {0, 0};
  {
    B_CHUNK_TILES(P, e.y) {
      B_TILE_CELLS(P, tile_) {
        const int c = i * g.ny + j;
        const uint8_t f = P.flags[c];
        const double rc = P.b[c] - b_apply<double>(P, f, i, j, c, xv);
        acc[0] += rc * rc;
        if (f & F_SOLV) acc[1] += xv(c, i, j);
      }
    }
  }
  b_reduce<2>(acc, sh.partials + (long)P.red_base * 8, P.counter, e.y, P.chunks, [&](double* t) {
    double* S = P.S;
    const double nb = sqrt(S[S_BNORM2]);
    S[S_RESID] = sqrt(t[0]) / (nb > 1e-300 ? nb : 1.0);
    if (!P.I[I_CONVERGED] && S[S_RESID] > fmax(tol * 10.0, 1e-8)) P.I[I_STATUS] = -3;
    S[S_MEAN_X] = (P.singular && g.n_fluid) ? t[1] / g.n_fluid : 0.0;
  });
}

// x <- x - mean on solvable rows, 0 elsewhere.
template <class T>
__global__ void __launch_bounds__(kBThreads) k_b_finish_apply(const BProb<T>* __restrict__ probs,
                                                               const int2* __restrict__ map, BShared sh) {
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (b_frozen(sh, e.x)) return;
  const bool zero = P.I[I_ZERO_RHS] != 0;
  const double m = P.S[S_MEAN_X];
  B_CHUNK_TILES(P, e.y) {
    B_TILE_CELLS(P, tile_) {
      const int c = i * P.g.ny + j;
      P.x[c] = (!zero && (P.flags[c] & F_SOLV)) ? P.x[c] - m : 0.0;
    }
  }
}

// ---- mixed form: FP64 iterative refinement around the FP32 MG-PCG -----------
// One refinement pass per problem (see k_ir_residual): r = b - A x in FP64, the
// outer test ||r|| < tol ||b||, and the inner solve A e = r set up from e = 0.
template <class T>
__global__ void __launch_bounds__(kBThreads) k_b_ir_residual(const BProb<T>* __restrict__ probs,
                                                              int nprob, const int2* __restrict__ map,
                                                              double tol, double inner_tol,
                                                              int max_passes, int first, BShared sh,
                                                              LoopCtl outer) {
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (!b_frozen(sh, e.x) && (first || !P.I[I_IR_DONE])) {
    const Geo& g = P.g;
    const double mean = (first && P.singular) ? P.S[S_MEAN_B] : 0.0;
    double acc[3] = {0, 0, 0};
    {
      B_CHUNK_TILES(P, e.y) {
        B_TILE_CELLS(P, tile_) {
          const int c = i * g.ny + j;
          const uint8_t f = P.flags[c];
          double bc = P.b[c];
          if (first) {
            bc = (f & F_SOLV) ? bc - mean : 0.0;
            P.b[c] = bc;
          }
          const double rc = bc - b_apply<double>(P, f, i, j, c, [&](int k, int, int) { return P.x[k]; });
          P.r[c] = (T)rc;
          P.xs[c] = (T)0;
          acc[0] += rc * rc;
          if (f & F_SOLV) acc[1] += (double)(T)rc;
          if (first) acc[2] += bc * bc;
        }
      }
    }
    b_reduce<3>(acc, sh.partials + (long)P.red_base * 8, P.counter, e.y, P.chunks, [&](double* t) {
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
__global__ void __launch_bounds__(kBThreads) k_b_ir_update(const BProb<T>* __restrict__ probs,
                                                            const int2* __restrict__ map, BShared sh) {
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (b_frozen(sh, e.x) || P.I[I_IR_DONE]) return;
  {
    B_CHUNK_TILES(P, e.y) {
      B_TILE_CELLS(P, tile_) {
        const int c = i * P.g.ny + j;
        if (P.flags[c] & F_SOLV) P.x[c] = P.x[c] + (double)P.xs[c];
      }
    }
  }
  if (e.y == 0 && threadIdx.x == 0 && threadIdx.y == 0) P.I[I_IR_IT] += 1;
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

template <class T, int MODE>
__global__ void __launch_bounds__(kBThreads) k_b_fine(const BProb<T>* __restrict__ probs,
                                                       const BHier<T>* __restrict__ hiers,
                                                       const int2* __restrict__ map, int src, int dst,
                                                       BShared sh) {
  const int2 e = map[blockIdx.x];
  const BProb<T>& P = probs[e.x];
  if (!b_solving(sh, e.x)) return;
  const Geo& g = P.g;
  B_VIEW(V, P);
  const int ny = V.g.ny;
  // arithmetic in T (FP32 in the mixed form's inner solve), sums in FP64
  const uint8_t* __restrict__ flags = P.flags;
  const T* __restrict__ r = P.r;
  const T mr = (T)(P.singular ? P.S[S_MEAN_R] : 0.0);
  auto bf = [&](int k) -> T {   // both loads issued, then selected
    const uint8_t fk = flags[k];
    const T rk = r[k];
    return (fk & F_SOLV) ? rk - mr : (T)0;
  };
  const T* __restrict__ x = b_fine_buf(P, src);
  T* __restrict__ xo = b_fine_buf(P, dst);
  T* __restrict__ lres0 = P.lres[0];
  double acc[2] = {0, 0};
  __shared__ T sm[kBHaloRows][kBHaloJ];
  if (MODE == FM_WDB) {
    B_CHUNK_TILES(V, e.y) {
      B_TILE_CELLS(V, tile_) {
        const int c = i * ny + j;
        xo[c] = (T)b_wdinv(V, flags[c], i, j) * bf(c);
      }
    }
  } else {
    uint8_t fv[kBCellBatch];
    T rv[kBCellBatch];
    auto load = [&](int u, int c) {
      fv[u] = flags[c];
      rv[u] = r[c];
    };
    auto bfv = [&](int u) -> T { return (fv[u] & F_SOLV) ? rv[u] - mr : (T)0; };   // bf at the cell
    if (MODE == FM_PRE) {
      auto xw = [&](int k, int ii, int jj) -> T {
        const uint8_t fk = flags[k];
        const T bk = bf(k);
        return (T)b_wdinv(V, fk, ii, jj) * bk;
      };
      b_chunk_cells<true>(V, e.y, sm, xw, load, [&](int u, int c, int i, int j, int li, int lj) {
        xo[c] = sm[li][lj];
        lres0[c] = bfv(u) - b_apply_sm<T>(V, fv[u], i, j, sm, li, lj);
      });
    } else {
      auto xw = [&](int k, int, int) -> T { return x[k]; };
      b_chunk_cells<true>(V, e.y, sm, xw, load, [&](int u, int c, int i, int j, int li, int lj) {
        const uint8_t f = fv[u];
        if (MODE == FM_RESID) {
          lres0[c] = bfv(u) - b_apply_sm<T>(V, f, i, j, sm, li, lj);
        } else {
          const T xn = sm[li][lj] + (T)b_wdinv(V, f, i, j) * (bfv(u) - b_apply_sm<T>(V, f, i, j, sm, li, lj));
          xo[c] = xn;
          if (MODE == FM_LAST && (f & F_SOLV)) {
            acc[0] += (double)xn;
            acc[1] += (double)rv[u] * (double)xn;
          }
        }
      });
    }
  }
  if (MODE != FM_LAST) return;
  b_reduce<2>(acc, sh.partials + (long)P.red_base * 8, P.counter, e.y, P.chunks, [&](double* t) {
    double* S = P.S;
    const double m = (P.singular && g.n_fluid) ? t[0] / g.n_fluid : 0.0;
    S[S_MEAN_Z] = m;
    S[S_RHO_PREV] = S[S_RHO];
    S[S_RHO] = t[1] - m * S[S_SUM_R];
  });
}

// ELL phases of coarse level d (and prolongation into level 0).  A block takes
// kBEllRounds x kBThreads / L rows, L lanes per row from the problem's
// hierarchy (runtime), so problems of different structures share one launch
// and wide rows spread over many blocks.
// EO_FRESTRICT: b_d = M_d b_{d-1} (first sweep on d-1 and restriction of its
// residual in one product; from level 0 the right-hand side is the projected CG
// residual).  EO_PROLONGW: prolongation onto a level whose first-sweep iterate
// W b was not stored -- it is formed again, with the same T roundings.
enum BEllOp { EO_RESTRICT = 0, EO_PRE, EO_SMOOTH, EO_RESID, EO_PROLONG, EO_FRESTRICT, EO_PROLONGW };

template <class T>
__device__ __forceinline__ T* b_lvl_x(const BProb<T>& P, int d, int sel) {
  if (d == P.nlev - 1 || d == P.tail) return P.lxa[d];   // coarsest and tail results are in xa
  return sel == 0 ? P.lxa[d] : P.lxb[d];
}

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

// Row dot product of E with L lanes fixed at compile time (L > 1: row-major
// entries, L = 1: column-major), the same summation order as b_ell_row.
template <int L, class T, class X>
__device__ __forceinline__ T b_ell_row_c(const Ell<T>& E, int row, int lane, X x) {
  T acc = (T)0;
  if (row < E.n) {
    if (L > 1) {
      const long base = (long)row * E.K;
#pragma unroll 4
      for (int k = lane; k < E.K; k += L) acc += E.val[base + k] * x(E.col[base + k]);
    } else {
#pragma unroll 4
      for (int k = 0; k < E.K; ++k) {
        const long at = (long)k * E.n + row;
        acc += E.val[at] * x(E.col[at]);
      }
    }
  }
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o, L);
  return acc;
}

// Rows [r0, r1) of level d for one ELL op: kBEllRounds rounds of kBThreads / L
// rows, the rounds unrolled so their loads overlap.
template <int L, int OP, class T>
__device__ __forceinline__ void b_ell_rows(const BProb<T>& P, int d, int src, int dst, int blk) {
  constexpr int per = kBThreads / L;
  const int n = (d == 0) ? P.g.nx * P.g.ny : P.lv[d].n;
  const int r0 = blk * per * kBEllRounds;
  const int r1 = min(n, r0 + per * kBEllRounds);
  const int lane = threadIdx.x & (L - 1);
  if (OP == EO_PROLONG) {
    // x_d += P_{d+1} x_{d+1}
    const Ell<T> Pm = P.lv[d + 1].P;
    const T* __restrict__ xc = b_lvl_x(P, d + 1, src);
    T* __restrict__ xf = (d == 0) ? b_fine_buf(P, dst) : b_lvl_x(P, d, dst);
#pragma unroll
    for (int rd = 0; rd < kBEllRounds; ++rd) {
      const int row = r0 + rd * per + (int)threadIdx.x / L;
      const T s = b_ell_row_c<L>(Pm, row < r1 ? row : Pm.n, lane, [&](int c) { return xc[c]; });
      if (lane == 0 && row < r1) xf[row] = xf[row] + s;
    }
    return;
  }
  if (OP == EO_PROLONGW) {
    // x_d = W b_d + P_{d+1} x_{d+1}; on level 0 W b is fine_wdinv * (projected residual)
    const Ell<T> Pm = P.lv[d + 1].P;
    const T* __restrict__ xc = b_lvl_x(P, d + 1, src);
    T* __restrict__ xf = (d == 0) ? b_fine_buf(P, dst) : b_lvl_x(P, d, dst);
    const T* __restrict__ b = P.lb[d];
    const T* __restrict__ wd = P.lv[d].wd;
    const uint8_t* __restrict__ flags = P.flags;
    const T* __restrict__ r = P.r;
    const T mr = (T)(d == 0 && P.singular ? P.S[S_MEAN_R] : 0.0);
    const int ny = P.g.ny;
#pragma unroll
    for (int rd = 0; rd < kBEllRounds; ++rd) {
      const int row = r0 + rd * per + (int)threadIdx.x / L;
      const T s = b_ell_row_c<L>(Pm, row < r1 ? row : Pm.n, lane, [&](int c) { return xc[c]; });
      if (lane == 0 && row < r1) {
        T wb;
        if (d == 0) {
          const uint8_t f = flags[row];
          const int i = row / ny, j = row - i * ny;
          const T bfr = (f & F_SOLV) ? r[row] - mr : (T)0;
          wb = (T)b_wdinv(P, f, i, j) * bfr;
        } else {
          wb = wd[row] * b[row];
        }
        xf[row] = wb + s;
      }
    }
    return;
  }
  if (OP == EO_FRESTRICT) {
    // b_d = M_d b_{d-1}, from level 0 the projected CG residual
    const Ell<T> M = P.lv[d].M;
    T* __restrict__ bo = P.lb[d];
    if (d == 1) {
      const uint8_t* __restrict__ flags = P.flags;
      const T* __restrict__ r = P.r;
      const T mr = (T)(P.singular ? P.S[S_MEAN_R] : 0.0);
#pragma unroll
      for (int rd = 0; rd < kBEllRounds; ++rd) {
        const int row = r0 + rd * per + (int)threadIdx.x / L;
        const T s = b_ell_row_c<L>(M, row < r1 ? row : M.n, lane, [&](int c) {
          const uint8_t fc = flags[c];
          const T rc = r[c];
          return (fc & F_SOLV) ? rc - mr : (T)0;
        });
        if (lane == 0 && row < r1) bo[row] = s;
      }
    } else {
      const T* __restrict__ bi = P.lb[d - 1];
#pragma unroll
      for (int rd = 0; rd < kBEllRounds; ++rd) {
        const int row = r0 + rd * per + (int)threadIdx.x / L;
        const T s = b_ell_row_c<L>(M, row < r1 ? row : M.n, lane, [&](int c) { return bi[c]; });
        if (lane == 0 && row < r1) bo[row] = s;
      }
    }
    return;
  }
  if (OP == EO_RESTRICT) {
    const Ell<T> R = P.lv[d].R;
    const T* __restrict__ res = P.lres[d - 1];
    T* __restrict__ bo = P.lb[d];
#pragma unroll
    for (int rd = 0; rd < kBEllRounds; ++rd) {
      const int row = r0 + rd * per + (int)threadIdx.x / L;
      const T s = b_ell_row_c<L>(R, row < r1 ? row : R.n, lane, [&](int c) { return res[c]; });
      if (lane == 0 && row < r1) bo[row] = s;
    }
    return;
  }
  const Ell<T> A = P.lv[d].A;
  const T* __restrict__ b = P.lb[d];
  const T* __restrict__ wd = P.lv[d].wd;
  const T* __restrict__ x = b_lvl_x(P, d, src);
  T* __restrict__ xo = b_lvl_x(P, d, dst);
  T* __restrict__ xa = P.lxa[d];
  T* __restrict__ ro = P.lres[d];
#pragma unroll
  for (int rd = 0; rd < kBEllRounds; ++rd) {
    const int row = r0 + rd * per + (int)threadIdx.x / L;
    const int rr = row < r1 ? row : A.n;
    if (OP == EO_PRE) {
      const T s = b_ell_row_c<L>(A, rr, lane, [&](int c) { return wd[c] * b[c]; });
      if (lane == 0 && row < r1) {
        const T bx = b[row];
        xa[row] = wd[row] * bx;
        ro[row] = bx - s;
      }
    } else if (OP == EO_SMOOTH) {
      const T s = b_ell_row_c<L>(A, rr, lane, [&](int c) { return x[c]; });
      if (lane == 0 && row < r1) xo[row] = x[row] + wd[row] * (b[row] - s);
    } else {   // EO_RESID
      const T s = b_ell_row_c<L>(A, rr, lane, [&](int c) { return x[c]; });
      if (lane == 0 && row < r1) ro[row] = b[row] - s;
    }
  }
}

template <class T, int OP>
__global__ void __launch_bounds__(kBThreads) k_b_ell(const BProb<T>* __restrict__ probs,
                                                      const int2* __restrict__ map, int d, int src,
                                                      int dst, BShared sh) {
  extern __shared__ double sb[];
  const int2 e = map[blockIdx.x];
  if (!b_solving(sh, e.x)) return;
  const BProb<T>& P = probs[e.x];
  if (OP == EO_RESTRICT && e.y < 0) {
    // coarsest level d: restriction and dense solve in this block
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
    return;
  }
  // the rows of this block, with the lane count of its matrix fixed at compile time
  const int Lop = (OP == EO_PROLONG || OP == EO_PROLONGW) ? P.lv[d + 1].lp
                  : OP == EO_RESTRICT                    ? P.lv[d].lr
                  : OP == EO_FRESTRICT                   ? P.lv[d].lm
                                                         : P.lv[d].la;
  switch (Lop) {
    case 1: b_ell_rows<1, OP>(P, d, src, dst, e.y); break;
    case 4: b_ell_rows<4, OP>(P, d, src, dst, e.y); break;
    case 8: b_ell_rows<8, OP>(P, d, src, dst, e.y); break;
    case 16: b_ell_rows<16, OP>(P, d, src, dst, e.y); break;
    default: b_ell_rows<32, OP>(P, d, src, dst, e.y); break;
  }
}

// Dense close of the V-cycle: x_t = M b_t for every problem whose structure has
// a tail, t the structure's tail depth and M its operator (n x n, row-major; the
// cycle at and below t as one linear map).  One launch after the down sweep
// covers every structure, whatever its tail depth.  A block takes kBTailRows rows of M
// (one warp each) for a group of kBTailGroup problems of one structure: each
// lane loads its entries of M once and applies them to every problem of the
// group (independent accumulators), so M crosses from L2 once per group and a
// row's sum is a fixed lane-strided order plus the warp tree.
constexpr int kBTailRows = kBThreads / 32;
constexpr int kBTailGroup = 8;

template <class T>
__device__ __forceinline__ T b_warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <class T>
__global__ void __launch_bounds__(kBThreads) k_b_tail(const BProb<T>* __restrict__ probs,
                                                       const BHier<T>* __restrict__ hiers,
                                                       const int2* __restrict__ map,
                                                       const int* __restrict__ sprobs, BShared sh) {
  const int2 e = map[blockIdx.x];   // (structure, row block * 64 + problem group)
  const BHier<T>& H = hiers[e.x];
  const int d = H.tail_level;
  const int n = H.tail_n;
  const int rb = e.y >> 6, grp = e.y & 63;
  __shared__ const T* sb[kBTailGroup];
  __shared__ T* sx[kBTailGroup];
  if (threadIdx.x < kBTailGroup) {
    const int k = grp * kBTailGroup + (int)threadIdx.x;
    const T* b = nullptr;
    T* x = nullptr;
    if (k < H.spn) {
      const int pi = sprobs[H.sp0 + k];
      if (b_solving(sh, pi)) {
        b = probs[pi].lb[d];
        x = probs[pi].lxa[d];
      }
    }
    sb[threadIdx.x] = b;
    sx[threadIdx.x] = x;
  }
  __syncthreads();
  const int warp = (int)(threadIdx.x >> 5), lane = (int)(threadIdx.x & 31);
  const int row = rb * kBTailRows + warp;
  if (row >= n) return;   // warp-uniform, no block barrier follows
  const T* m = H.tail + (long)row * n;
  T acc[kBTailGroup];
#pragma unroll
  for (int g = 0; g < kBTailGroup; ++g) acc[g] = (T)0;
  for (int c = lane; c < n; c += 32) {
    const T mv = __ldg(m + c);
#pragma unroll
    for (int g = 0; g < kBTailGroup; ++g)
      if (sb[g]) acc[g] += mv * sb[g][c];
  }
#pragma unroll
  for (int g = 0; g < kBTailGroup; ++g) {
    const T t = b_warp_sum(acc[g]);
    if (lane == 0 && sx[g]) sx[g][row] = t;
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
