// Shared device helpers: geometry, scalar slots and deterministic grid reductions.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pcfd {

// A product rounded on its own: never fused with the add or subtract it feeds.
// The library is compiled with FMA contraction on (the solver kernels gain from
// it); the momentum stencil, the stage combinations, the boundary sums and the
// rasteriser form their products through rmul so that every product rounds
// before it is summed, as the reference's array arithmetic does, and stay
// bit-identical to it.  Products by 0.5, 2 or 4 are exact and need no guard.
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }

#define PCFD_MAX_BODIES_DEV 8

// Wall order of every boundary pass (pycfd/core/boundary.py:375-379).
enum { W_LEFT = 0, W_RIGHT = 1, W_BOTTOM = 2, W_TOP = 3 };
enum { BC_NO_SLIP = 0, BC_MOVING_WALL = 1, BC_INLET = 2, BC_OUTLET = 3,
       BC_PRESSURE_OUTLET = 4, BC_PERIODIC = 5, BC_SYMMETRY = 6 };

// Cell flags of the fine Poisson operator: which of the four faces carry a
// 1/h^2 coupling (both cells fluid and joined inside the domain or across a
// periodic wrap) and whether the row is a solvable unknown
// (pycfd/core/pressure.py:209-247).
enum : uint8_t { F_W = 1, F_E = 2, F_S = 4, F_N = 8, F_SOLV = 16 };

// Device scalar slots (doubles) shared by the kernels of one solver.
enum Slot {
  S_DT = 0, S_BLEND,
  S_BNORM2, S_ATOL, S_RNORM2, S_RHO, S_RHO_PREV, S_ALPHA, S_BETA, S_PQ,
  S_MEAN_B, S_MEAN_R, S_MEAN_X, S_RESID, S_RES_PREV, S_SUM_R, S_TOL,
  S_BNORM2_0, S_IR_RNORM2, S_MEAN_Z, S_IR_BNORM, S_T,
  S_FX, S_FY,
  S_BODY_FX,                      // PCFD_MAX_BODIES slots
  S_BODY_FY = S_BODY_FX + 8,
  S_MASS_IN = S_BODY_FY + 8, S_MASS_OUT,
  S_STAT0,                        // field stats block (8 slots)
  S_COUNT = S_STAT0 + 8 + 8
};

// Device int slots.
enum ISlot {
  I_IT = 0, I_DONE, I_CONVERGED, I_STATUS, I_STALLED, I_TOTAL_IT, I_ZERO_RHS, I_MAXITER,
  I_IR_IT, I_IR_DONE, I_FINITE, I_HEALTH, I_STEPS,
  I_FROZEN,        // 1 stopped by a health flag, 2 reached its end time, 3 steady (device loops)
  I_HIST,          // rows appended to the device history since it was last read
  I_COUNT = 16
};

struct Geo {
  int nx, ny;
  double dx, dy, nu, fx, fy;
  int u_lo, u_hi, v_lo, v_hi;   // solvable face ranges (pycfd/core/solver.py:235-263)
  int periodic_x, periodic_y;
  int dir_w, dir_e, dir_s, dir_n;  // Dirichlet (pressure outlet) walls
  double pref_w, pref_e, pref_s, pref_n;
  double cx, cy;                // 1/dx^2, 1/dy^2
  int n_fluid;                  // number of solvable cells
  const double* met;            // stretched mesh: packed metrics (Metrics below); nullptr when uniform
};

// The spacings of a stretched mesh (pycfd/core/mesh.py:122-218), packed in this
// order by MeshMetrics.device_block: hx[nx], hy[ny] (cell widths / heights),
// hxu[nx+1], hyv[ny+1] (centre-to-centre distance across each face, ghost
// mirroring its neighbour), hx_ext[nx+2], hy_ext[ny+2] (widths with that ghost),
// wx[nx+1], wy[ny+1] (upper-node weight of a corner interpolant), the Poisson
// face denominators hxu*vbar[nx+1], hyv*vbar[ny+1] and vbar, the mean cell area
// (pycfd/core/pressure.py:193-207).
struct Metrics {
  const double* p;
  int nx, ny;
  __host__ __device__ __forceinline__ Metrics(const Geo& g) : p(g.met), nx(g.nx), ny(g.ny) {}
  __device__ __forceinline__ double hx(int i) const { return p[i]; }
  __device__ __forceinline__ double hy(int j) const { return p[nx + j]; }
  __device__ __forceinline__ double hxu(int f) const { return p[nx + ny + f]; }
  __device__ __forceinline__ double hyv(int f) const { return p[2 * nx + ny + 1 + f]; }
  __device__ __forceinline__ double hx_ext(int k) const { return p[2 * nx + 2 * ny + 2 + k]; }
  __device__ __forceinline__ double hy_ext(int k) const { return p[3 * nx + 2 * ny + 4 + k]; }
  __device__ __forceinline__ double wx(int f) const { return p[3 * nx + 3 * ny + 6 + f]; }
  __device__ __forceinline__ double wy(int f) const { return p[4 * nx + 3 * ny + 7 + f]; }
  __device__ __forceinline__ double axv(int f) const { return p[4 * nx + 4 * ny + 8 + f]; }
  __device__ __forceinline__ double ayv(int f) const { return p[5 * nx + 4 * ny + 9 + f]; }
  __device__ __forceinline__ double vbar() const { return p[5 * nx + 5 * ny + 10]; }
  // Poisson coefficients of the faces around cell (i, j): face area over the
  // centre distance and the mean cell area, the reference's expressions.
  __device__ __forceinline__ double cw(int i, int j) const { return hy(j) / axv(i); }
  __device__ __forceinline__ double ce(int i, int j) const { return hy(j) / axv(i + 1); }
  __device__ __forceinline__ double cs(int i, int j) const { return hx(i) / ayv(j); }
  __device__ __forceinline__ double cn(int i, int j) const { return hx(i) / ayv(j + 1); }
  // Row scale of the Poisson system: cell area over the mean cell area.
  __device__ __forceinline__ double row_scale(int i, int j) const { return __dmul_rn(hx(i), hy(j)) / vbar(); }
};
inline int metrics_count(int nx, int ny) { return 5 * nx + 5 * ny + 11; }

// Reduction workspace: one row of NV partials per block plus a ticket counter.
struct RedBuf {
  double* partials;
  unsigned int* counter;
};

constexpr int kMaxRedBlocks = 1184;   // 148 SMs x 8 resident blocks (partials buffer size)
// Streaming grids are sized to one wave: 148 SMs x 4 resident 256-thread
// blocks (every streaming kernel here stays at <= 64 registers per thread),
// with grid-stride loops, so no kernel pays a partial second wave.
constexpr int kWaveBlocks = 592;
constexpr int kRedThreads = 256;

// Programmatic dependent launch (sm_90+): a kernel launched with the
// programmatic-serialization attribute may be scheduled while its predecessor
// is still running.  Every kernel therefore first waits for the predecessor's
// completion and memory (a no-op without the attribute), then allows its own
// successor to be scheduled, so the launch latency between dependent kernels
// overlaps execution.
__device__ __forceinline__ void pdl_begin() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide reduction of NV values (sum, or max where bit k of MAXMASK is set).
// Result valid in thread 0.  Fixed tree: deterministic for a fixed block size.
template <int NV, unsigned MAXMASK = 0u>
__device__ __forceinline__ void block_reduce(double (&v)[NV]) {
  __shared__ double sm[NV][32];
  const int t = threadIdx.x + threadIdx.y * blockDim.x;
  const int lane = t & 31, wid = t >> 5;
  const int nw = (blockDim.x * blockDim.y + 31) >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    v[k] = ((MAXMASK >> k) & 1u) ? warp_max(v[k]) : warp_sum(v[k]);
    if (lane == 0) sm[k][wid] = v[k];
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = (lane < nw) ? sm[k][lane] : (((MAXMASK >> k) & 1u) ? -INFINITY : 0.0);
      v[k] = ((MAXMASK >> k) & 1u) ? warp_max(t) : warp_sum(t);
    }
  }
  __syncthreads();
}

// The last block's pass over every block's NV partials (row b at b*NV): L2
// loads (ld.global.cg, coherent with the other blocks' fenced writes), several
// blocks' rows in flight per thread; each thread adds its rows in block order,
// so the totals are those of a plain strided loop.
template <int NV, unsigned MAXMASK = 0u>
__device__ __forceinline__ void sum_partials(const double* __restrict__ partials, int n, int tid, int nthr,
                                             double (&acc)[NV]) {
  constexpr int U = NV <= 2 ? 4 : (NV <= 4 ? 2 : 1);
#pragma unroll
  for (int k = 0; k < NV; ++k) acc[k] = ((MAXMASK >> k) & 1u) ? -INFINITY : 0.0;
  for (int b0 = tid; b0 < n; b0 += U * nthr) {
    double p[U][NV];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int b = b0 + u * nthr;
#pragma unroll
      for (int k = 0; k < NV; ++k) p[u][k] = b < n ? __ldcg(partials + (long)b * NV + k) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (b0 + u * nthr < n) {
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[k] = ((MAXMASK >> k) & 1u) ? fmax(acc[k], p[u][k]) : acc[k] + p[u][k];
      }
    }
  }
}

// Grid-wide reduction.  Every block contributes NV values; the last block to
// arrive (ticket counter) combines the partials in block order and calls
// fin(totals) on its thread 0.  Returns true in that thread.
template <int NV, unsigned MAXMASK = 0u, class Fin>
__device__ __forceinline__ void grid_reduce(double (&v)[NV], RedBuf rb, Fin fin) {
  block_reduce<NV, MAXMASK>(v);
  __shared__ bool last;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  const int nthr = blockDim.x * blockDim.y;
  const int bid = blockIdx.x + blockIdx.y * gridDim.x;
  const int nblk = gridDim.x * gridDim.y;
  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) rb.partials[bid * NV + k] = v[k];
    __threadfence();
    unsigned t = atomicAdd(rb.counter, 1u);
    last = (t == (unsigned)nblk - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double acc[NV];
  sum_partials<NV, MAXMASK>(rb.partials, nblk, tid, nthr, acc);
  block_reduce<NV, MAXMASK>(acc);
  if (tid == 0) {
    fin(acc);
    *rb.counter = 0u;
  }
}

// Fine-level diagonal, accumulated face by face in the reference's order
// (left, [left Dirichlet], right, [right Dirichlet], bottom, ..., top), so it is
// bit-identical to the assembled matrix (pycfd/core/pressure.py:229-247).
__device__ __forceinline__ double fine_diag(uint8_t f, int i, int j, const Geo& g) {
  if (!(f & F_SOLV)) return 1.0;
  double d = 0.0;
  if (g.met) {   // stretched: per-face coefficients, the same order
    const Metrics M(g);
    const double cw = M.cw(i, j), ce = M.ce(i, j), cs = M.cs(i, j), cn = M.cn(i, j);
    if (f & F_W) d -= cw;
    if (g.dir_w && i == 0) d -= 2.0 * cw;
    if (f & F_E) d -= ce;
    if (g.dir_e && i == g.nx - 1) d -= 2.0 * ce;
    if (f & F_S) d -= cs;
    if (g.dir_s && j == 0) d -= 2.0 * cs;
    if (f & F_N) d -= cn;
    if (g.dir_n && j == g.ny - 1) d -= 2.0 * cn;
    return d;
  }
  if (f & F_W) d -= g.cx;
  if (g.dir_w && i == 0) d -= 2.0 * g.cx;
  if (f & F_E) d -= g.cx;
  if (g.dir_e && i == g.nx - 1) d -= 2.0 * g.cx;
  if (f & F_S) d -= g.cy;
  if (g.dir_s && j == 0) d -= 2.0 * g.cy;
  if (f & F_N) d -= g.cy;
  if (g.dir_n && j == g.ny - 1) d -= 2.0 * g.cy;
  return d;
}

// Dirichlet right-hand-side contribution -2 c p_ref per Dirichlet wall the
// cell touches, in wall order (pycfd/core/pressure.py:240-247).
__device__ __forceinline__ double fine_bc(uint8_t f, int i, int j, const Geo& g) {
  if (!(f & F_SOLV)) return 0.0;
  double b = 0.0;
  if (g.met) {
    const Metrics M(g);
    if (g.dir_w && i == 0) b -= rmul(2.0 * M.cw(i, j), g.pref_w);
    if (g.dir_e && i == g.nx - 1) b -= rmul(2.0 * M.ce(i, j), g.pref_e);
    if (g.dir_s && j == 0) b -= rmul(2.0 * M.cs(i, j), g.pref_s);
    if (g.dir_n && j == g.ny - 1) b -= rmul(2.0 * M.cn(i, j), g.pref_n);
    return b;
  }
  if (g.dir_w && i == 0) b -= rmul(2.0 * g.cx, g.pref_w);
  if (g.dir_e && i == g.nx - 1) b -= rmul(2.0 * g.cx, g.pref_e);
  if (g.dir_s && j == 0) b -= rmul(2.0 * g.cy, g.pref_s);
  if (g.dir_n && j == g.ny - 1) b -= rmul(2.0 * g.cy, g.pref_n);
  return b;
}

// Neighbour coordinates across the four faces (periodic wrap applied; only
// used where the face flag is set).
__device__ __forceinline__ int wrap_w(int i, const Geo& g) { return i > 0 ? i - 1 : g.nx - 1; }
__device__ __forceinline__ int wrap_e(int i, const Geo& g) { return i < g.nx - 1 ? i + 1 : 0; }
__device__ __forceinline__ int wrap_s(int j, const Geo& g) { return j > 0 ? j - 1 : g.ny - 1; }
__device__ __forceinline__ int wrap_n(int j, const Geo& g) { return j < g.ny - 1 ? j + 1 : 0; }
__device__ __forceinline__ int nb_w(int i, int j, const Geo& g) { return wrap_w(i, g) * g.ny + j; }
__device__ __forceinline__ int nb_e(int i, int j, const Geo& g) { return wrap_e(i, g) * g.ny + j; }
__device__ __forceinline__ int nb_s(int i, int j, const Geo& g) { return i * g.ny + wrap_s(j, g); }
__device__ __forceinline__ int nb_n(int i, int j, const Geo& g) { return i * g.ny + wrap_n(j, g); }

// (A x)_c for the fine operator; the functor x(k, i, j) supplies the value at
// flat index k = i*ny + j (so neighbour values can be formed on the fly).
template <class T, class X>
__device__ __forceinline__ T fine_apply(uint8_t f, int i, int j, int c, const Geo& g, X x) {
  if (g.met) {
    const Metrics M(g);
    T acc = (T)fine_diag(f, i, j, g) * x(c, i, j);
    if (f & F_W) { const int a = wrap_w(i, g); acc += (T)M.cw(i, j) * x(a * g.ny + j, a, j); }
    if (f & F_E) { const int a = wrap_e(i, g); acc += (T)M.ce(i, j) * x(a * g.ny + j, a, j); }
    if (f & F_S) { const int b = wrap_s(j, g); acc += (T)M.cs(i, j) * x(i * g.ny + b, i, b); }
    if (f & F_N) { const int b = wrap_n(j, g); acc += (T)M.cn(i, j) * x(i * g.ny + b, i, b); }
    return acc;
  }
  T acc = (T)fine_diag(f, i, j, g) * x(c, i, j);
  if (f & F_W) { const int a = wrap_w(i, g); acc += (T)g.cx * x(a * g.ny + j, a, j); }
  if (f & F_E) { const int a = wrap_e(i, g); acc += (T)g.cx * x(a * g.ny + j, a, j); }
  if (f & F_S) { const int b = wrap_s(j, g); acc += (T)g.cy * x(i * g.ny + b, i, b); }
  if (f & F_N) { const int b = wrap_n(j, g); acc += (T)g.cy * x(i * g.ny + b, i, b); }
  return acc;
}

// Cells of the fine grid for a 2D launch (threads along y, blocks striding x):
// no integer division anywhere in the fine-level kernels.
#define FOR_CELLS(g)                                                                    \
  for (int i = blockIdx.y * blockDim.y + threadIdx.y; i < (g).nx; i += gridDim.y * blockDim.y) \
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < (g).ny; j += gridDim.x * blockDim.x)

// ---- warp strips of one grid ------------------------------------------------
// The fine-level solver kernels walk the grid in warp strips: a warp takes one
// segment of y (lane = column: every row load is one coalesced access) over
// kStripRows rows of x.  The stencil operand of the strip and its two halo rows
// are formed once, into registers, before any arithmetic; the y-neighbours come
// from the adjacent lanes by shuffle.  A stencil kernel's segment is 30 columns,
// lanes 1..30, and lanes 0 and 31 hold the columns just west and east of it, so
// each lane forms one operand value per row, no load sits under a lane-dependent
// branch and the whole strip's loads are in flight at once; a pointwise kernel
// takes aligned 32-column segments.  Off-grid rows and columns are read at a
// clamped (valid) index and the value dropped.
// Blocks of 256 threads (8 warps) stride over the items (strip x segment).
#ifndef PCFD_STRIP_ROWS
#define PCFD_STRIP_ROWS 4
#endif
constexpr int kStripRows = PCFD_STRIP_ROWS;
constexpr int kStripThreads = 256;

constexpr int kStripSegCols = 30;   // output columns of a stencil kernel's segment (lanes 1..30)
// items of the stencil kernels (the pointwise kernels' 32-column segments are no more)
inline int strip_items(const Geo& g) {
  return ((g.ny + kStripSegCols - 1) / kStripSegCols) * ((g.nx + kStripRows - 1) / kStripRows);
}
inline int strip_grid(const Geo& g) {
  const int b = (strip_items(g) + kStripThreads / 32 - 1) / (kStripThreads / 32);
  return b < kMaxRedBlocks ? (b < 1 ? 1 : b) : kMaxRedBlocks;
}

// Row of the operand at strip row r (halo rows included): wrapped on a periodic
// x axis, -1 off the grid.
__device__ __forceinline__ int strip_row(int r, int nx, int periodic_x) {
  if (r < 0) return periodic_x ? nx - 1 : -1;
  if (r >= nx) return (r == nx && periodic_x) ? 0 : -1;
  return r;
}

// The columns west and east of segment [j0, j0 + last]: wrapped on a periodic y
// axis, -1 off the grid.
__device__ __forceinline__ void strip_edges(int j0, int last, int ny, int periodic_y, int* jw, int* je) {
  *jw = j0 > 0 ? j0 - 1 : (periodic_y ? ny - 1 : -1);
  *je = j0 + last + 1 < ny ? j0 + last + 1 : (periodic_y ? 0 : -1);
}

// op(k, i, j): the operand at cell (i, j) (issues its loads; k always a valid
// cell, the value dropped where the cell is off the grid); load(u, c): the
// per-cell loads of body row u (c valid; the values unused past the grid);
// body(u, c, i, j, centre, west, east, south, north).  STENCIL = false: no
// operand (pointwise kernels).  Neighbours off the grid are wrapped on periodic
// axes and 0 otherwise (their face flags are clear).
template <bool STENCIL, class Op, class Load, class Body>
__device__ __forceinline__ void strip_cells(const Geo& g, Op op, Load load, Body body) {
  constexpr int RS = kStripRows;
  const int lane = (int)(threadIdx.x & 31), warp = (int)(threadIdx.x >> 5);
  const int nx = g.nx, ny = g.ny;
  const int segs = STENCIL ? (ny + kStripSegCols - 1) / kStripSegCols : (ny + 31) / 32;
  const int items = segs * ((nx + RS - 1) / RS);
  const int wpb = (int)(blockDim.x >> 5);
  for (int it = (int)blockIdx.x * wpb + warp; it < items; it += (int)gridDim.x * wpb) {
    const int strip = it / segs, seg = it - strip * segs;
    const int i0 = strip * RS;
    int j, jc;
    bool jv;
    int jh = -1;   // STENCIL: the operand's column (wrapped), -1 off the grid
    if (STENCIL) {
      j = seg * kStripSegCols - 1 + lane;   // lanes 0 and 31: the columns beside the segment
      jh = j;
      if (jh < 0) jh = g.periodic_y ? jh + ny : -1;
      else if (jh >= ny) jh = (g.periodic_y && jh == ny) ? 0 : -1;
      jc = jh >= 0 ? jh : (j < 0 ? 0 : ny - 1);
      jv = lane >= 1 && lane <= 30 && j < ny;
    } else {
      j = seg * 32 + lane;
      jv = j < ny;
      jc = jv ? j : ny - 1;
    }
    double ov[STENCIL ? RS + 2 : 1];
    if (STENCIL) {
#pragma unroll
      for (int u = 0; u < RS + 2; ++u) {
        const int r = strip_row(i0 - 1 + u, nx, g.periodic_x);
        const int rc = r >= 0 ? r : 0;
        const double val = op(rc * ny + jc, rc, jc);
        ov[u] = (jh >= 0 && r >= 0) ? val : 0.0;
      }
    }
#pragma unroll
    for (int u = 0; u < RS; ++u) {
      const int i = i0 + u, ic = i < nx ? i : nx - 1;
      load(u, ic * ny + jc);
    }
#pragma unroll
    for (int u = 0; u < RS; ++u) {
      double c = 0.0, w = 0.0, e = 0.0, sv = 0.0, nv = 0.0;
      if (STENCIL) {
        c = ov[u + 1];
        w = ov[u];
        e = ov[u + 2];
        sv = __shfl_up_sync(0xffffffffu, c, 1);
        nv = __shfl_down_sync(0xffffffffu, c, 1);
      }
      const int i = i0 + u;
      if (jv && i < nx) body(u, i * ny + j, i, j, c, w, e, sv, nv);
    }
  }
}

// (A x) at a cell from its value and its neighbours', fine_apply's terms in its
// order (diagonal, west, east, south, north).
__device__ __forceinline__ double fine_apply5(uint8_t f, int i, int j, const Geo& g, double c, double w, double e,
                                              double s, double n) {
  if (g.met) {
    const Metrics M(g);
    double acc = fine_diag(f, i, j, g) * c;
    if (f & F_W) acc += M.cw(i, j) * w;
    if (f & F_E) acc += M.ce(i, j) * e;
    if (f & F_S) acc += M.cs(i, j) * s;
    if (f & F_N) acc += M.cn(i, j) * n;
    return acc;
  }
  double acc = fine_diag(f, i, j, g) * c;
  if (f & F_W) acc += g.cx * w;
  if (f & F_E) acc += g.cx * e;
  if (f & F_S) acc += g.cy * s;
  if (f & F_N) acc += g.cy * n;
  return acc;
}

constexpr int kCellTJ = 32, kCellTI = 8;

// 2D launch shape over nx x ny cells with at most kMaxRedBlocks blocks.
inline void cell_launch(int nx, int ny, dim3* grid, dim3* block) {
  *block = dim3(kCellTJ, kCellTI);
  int gx = (ny + kCellTJ - 1) / kCellTJ;
  if (gx > kWaveBlocks) gx = kWaveBlocks;
  int gy = (nx + kCellTI - 1) / kCellTI;
  const int cap = kWaveBlocks / gx > 0 ? kWaveBlocks / gx : 1;
  if (gy > cap) gy = cap;
  *grid = dim3(gx, gy);
}

inline int grid_for(long n, int threads, int max_blocks = kMaxRedBlocks) {
  long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > max_blocks) b = max_blocks;
  return (int)b;
}

}  // namespace pcfd
