// A whole conjugate-gradient Poisson solve (Jacobi- or multigrid-
// preconditioned) as ONE cooperative launch.
//
// The separate-kernel form launches ~26 kernels per MG-PCG pass on a 512^2
// grid, each carrying under two cells per thread, so a pass costs the sum of
// 26 kernel start/drain latencies more than its bytes.  Here the grid is
// launched cooperatively (every CTA is resident at once, or the launch fails
// with an error instead of starting) and the phases of a pass -- the V-cycle
// levels, p/q and x/r -- are separated by grid barriers: one fenced atomic
// arrival per CTA on a counter that only grows, its thread 0 polling the
// counter until every CTA has arrived.  Dot products are all-reduced
// redundantly: each CTA writes its block sum, and after the barrier every CTA
// sums all of them in CTA order with the same tree, so every CTA holds the same
// scalars (alpha, beta, the convergence test) without another round trip, and
// results are run-to-run deterministic.  Every wait is bounded by a wall-clock
// limit: a CTA that gives up raises the error word, every other wait then
// returns at once, the solve loop ends and the solve reports status -6.
//
// Per row and per cell the arithmetic is that of the separate kernels
// (poisson.cuh, multigrid.cuh): the same expressions, the same ELL lane split
// and per-lane summation order, the same coarsest dense product; the fine
// diagonal comes from a 32-entry table of fine_diag's own sums (cells beside a
// Dirichlet wall use fine_diag itself).  Only the CTA partition of the dot
// products differs.  Vectors written inside the kernel are read through L2
// (ld.global.cg); matrices, flags and weights are read-only for its lifetime.
#pragma once
#include "multigrid.cuh"
#include "poisson.cuh"

namespace pcfd {

constexpr int kPThreads = 512;
constexpr int kPMaxLevels = 12;
constexpr int kPDenseMax = 1024;                            // coarsest rows solved in CTA 0
constexpr int kPMaxNV = 4;                                  // sums per all-reduce
constexpr unsigned long long kPWaitLimitNs = 2000000000ull;  // default limit of one barrier wait: 2 s
constexpr int kPStatusTimeout = -6;
constexpr int kPTraceCap = 8192;                            // words of the phase trace

// Phase tags of the trace (low byte; the level in the next byte).
enum PTag { PT_INIT = 1, PT_FINE_PRE, PT_RESTRICT, PT_PRE, PT_COARSEST, PT_PROLONG, PT_SMOOTH,
            PT_FINE_SMOOTH, PT_PQ, PT_XR, PT_FINISH, PT_DENSE_RHS, PT_TAIL };

template <class T>
struct PLevel {
  Ell<T> A, R, P;   // A, R: rows of this level; P: rows of the next finer level
  int la, lr, lp;   // lanes per row of each block
  const T* wd;
  T *b, *xa, *xb, *res;
};

template <class T>
struct PSolve {
  PLevel<T> lv[kPMaxLevels];   // lv[0] is the matrix-free fine level (buffers only)
  int nlev;
  const T* C;                  // coarsest pseudo-inverse, row-major nc x nc
  int nc;
  const T* tail;               // dense cycle operator of level tail_level (0: none)
  int tail_level;
  const uint8_t* flags;
  Geo g;
  double w0;                   // weight of the fine damped-Jacobi sweep
  int sweeps;
  SolveCfg cfg;
  int has_x0;
  double* b;                   // right-hand side, conditioned in place
  T *x, *r, *z, *pa, *pb, *q;
  double* S;
  int* I;
  double* partials;            // 2 x kPMaxNV x gridDim.x (alternating slots)
  unsigned* bar;               // [0] arrivals, [32] error word; zeroed before every launch
  unsigned long long* trace;   // optional: [0] count, then (globaltimer, tag) pairs
  unsigned long long wait_ns;  // limit of one barrier wait (kPWaitLimitNs unless set)
};

__device__ __forceinline__ unsigned p_ld_relaxed(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long p_clock_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Barrier and all-reduce state of one CTA.
struct PBar {
  unsigned* bar;
  unsigned target;             // arrivals that end the current barrier (thread 0)
  unsigned red;                // all-reduces so far (selects the partials slot)
  unsigned long long* trace;   // CTA 0 only
  int ntr;
  unsigned long long wait_ns;  // limit of one barrier wait
};

__device__ __forceinline__ bool p_failed(const PBar& pb) { return p_ld_relaxed(pb.bar + 32) != 0u; }

// Grid barrier.  Thread 0 of every CTA arrives once (its CTA's writes ordered
// before by the block barrier and the fence) and polls until all have arrived.
__device__ __forceinline__ void p_sync(PBar& pb, int tag) {
  __syncthreads();
  if (threadIdx.x == 0) {
    pb.target += gridDim.x;
    __threadfence();
    atomicAdd(pb.bar, 1u);
    const unsigned long long t0 = p_clock_ns();
    int k = 0;
    while (p_ld_relaxed(pb.bar) < pb.target) {
      if (p_clock_ns() - t0 > pb.wait_ns) {           // checked on every poll
        atomicExch(pb.bar + 32, 1u);
        break;
      }
      if ((++k & 63) == 0 && p_failed(pb)) break;     // another CTA gave up
    }
    __threadfence();
    if (pb.trace && blockIdx.x == 0 && 2 * pb.ntr + 2 < kPTraceCap) {
      pb.trace[1 + 2 * pb.ntr] = p_clock_ns();
      pb.trace[2 + 2 * pb.ntr] = (unsigned long long)tag;
      ++pb.ntr;
    }
  }
  __syncthreads();
}

// All-reduce of NV sums over the grid: block sums to this reduction's slot,
// barrier, then every CTA sums the slot in CTA order with the same tree.
// Thread 0 gets the totals in tot and runs fin(tot) before the threads of the
// CTA are released (fin writes the CTA's shared scalars).
template <int NV, class Fin>
__device__ __forceinline__ void p_allreduce(PBar& pb, double* partials, double (&v)[NV], int tag, Fin fin) {
  block_reduce<NV>(v);
  double* slot = partials + (size_t)(pb.red & 1u) * kPMaxNV * gridDim.x;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) slot[k * gridDim.x + blockIdx.x] = v[k];
  }
  p_sync(pb, tag);
  double acc[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    acc[k] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) acc[k] += __ldcg(slot + k * gridDim.x + b);
  }
  block_reduce<NV>(acc);
  if (threadIdx.x == 0) fin(acc);
  __syncthreads();
  pb.red += 1u;
}

// Fine cells, flat over the whole grid (y contiguous), coordinates stepped
// without a division per cell.
template <class F>
__device__ __forceinline__ void p_cells(const Geo& g, F f) {
  const int n = g.nx * g.ny;
  const int nthr = (int)(gridDim.x * blockDim.x);
  int c = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (c >= n) return;
  int i = c / g.ny, j = c - i * g.ny;
  const int di = nthr / g.ny, dj = nthr - di * g.ny;
  for (; c < n; c += nthr) {
    f(c, i, j);
    i += di;
    j += dj;
    if (j >= g.ny) {
      j -= g.ny;
      ++i;
    }
  }
}

template <class T>
__device__ __forceinline__ double p_ld(const T* p) { return (double)__ldcg(p); }

// Fine diagonal: a table of fine_diag over the 32 flag patterns (no Dirichlet
// term), fine_diag itself beside a Dirichlet wall.
__device__ __forceinline__ bool p_edge(int i, int j, const Geo& g) {
  return (g.dir_w && i == 0) || (g.dir_e && i == g.nx - 1) || (g.dir_s && j == 0) || (g.dir_n && j == g.ny - 1);
}
// (A stretched mesh has no per-flag table: every cell forms its own coefficients.)
__device__ __forceinline__ double p_diag(const double* dtab, uint8_t f, int i, int j, const Geo& g) {
  return (g.met || p_edge(i, j, g)) ? fine_diag(f, i, j, g) : dtab[f & 31];
}
__device__ __forceinline__ double p_wdinv(const double* wtab, uint8_t f, int i, int j, const Geo& g, double w) {
  return (g.met || p_edge(i, j, g)) ? fine_wdinv(f, i, j, g, w) : wtab[f & 31];
}
// fine_apply<double> with the tabled diagonal.
template <class X>
__device__ __forceinline__ double p_apply(const double* dtab, uint8_t f, int i, int j, int c, const Geo& g, X x) {
  if (g.met) return fine_apply<double>(f, i, j, c, g, x);
  double acc = p_diag(dtab, f, i, j, g) * x(c, i, j);
  if (f & F_W) { const int a = wrap_w(i, g); acc += g.cx * x(a * g.ny + j, a, j); }
  if (f & F_E) { const int a = wrap_e(i, g); acc += g.cx * x(a * g.ny + j, a, j); }
  if (f & F_S) { const int b = wrap_s(j, g); acc += g.cy * x(i * g.ny + b, i, b); }
  if (f & F_N) { const int b = wrap_n(j, g); acc += g.cy * x(i * g.ny + b, i, b); }
  return acc;
}

// One ELL pass over all rows, L lanes per row, every thread the same number
// of rounds.  A lane's entries are gathered four at a time -- indices and
// values first, then the vector values, then the products added in entry
// order -- so the sums are those of a lane's plain loop with four gathers in flight.
constexpr int kPGather = 4;
template <class T, class X, class W>
__device__ __forceinline__ void p_ell(const Ell<T>& E, int L, int gtid, int nthr, X x, W write) {
  const int per = nthr / L;
  const int lane = gtid % L, r0 = gtid / L;
  for (int base = 0; base < E.n; base += per) {
    const int row = base + r0;
    double acc = 0.0;
    if (row < E.n) {
      for (int k0 = lane; k0 < E.K; k0 += kPGather * L) {
        int cc[kPGather];
        T vv[kPGather];
#pragma unroll
        for (int u = 0; u < kPGather; ++u) {
          const int k = k0 + u * L;
          cc[u] = 0;
          vv[u] = (T)0;
          if (k < E.K) {
            const long e = E.rowmajor ? (long)row * E.K + k : (long)k * E.n + row;
            cc[u] = __ldg(E.col + e);
            vv[u] = __ldg(E.val + e);
          }
        }
        double xx[kPGather];
#pragma unroll
        for (int u = 0; u < kPGather; ++u) xx[u] = (k0 + u * L < E.K) ? x(cc[u]) : 0.0;
#pragma unroll
        for (int u = 0; u < kPGather; ++u)
          if (k0 + u * L < E.K) acc += (double)vv[u] * xx[u];
      }
    }
    for (int s = L >> 1; s > 0; s >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, s, L);
    if (lane == 0 && row < E.n) write(row, acc);
  }
}

// x = M b over the grid (k_tail's split: four warps per row, their sums added
// in warp order); every CTA runs the same number of rounds.
template <class T>
__device__ __forceinline__ void p_tail(const T* M, int n, const T* b, T* x) {
  __shared__ double part[kPThreads / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int rows_per_cta = kPThreads / 32 / kTailWarps;
  for (int r0 = blockIdx.x * rows_per_cta; r0 < n; r0 += gridDim.x * rows_per_cta) {
    const int row = r0 + warp / kTailWarps;
    const int w = warp % kTailWarps;
    double acc = 0.0;
    if (row < n) {
      const T* m = M + (long)row * n;
      constexpr int stride = 32 * kTailWarps;
      for (int k0 = w * 32 + lane; k0 < n; k0 += 8 * stride) {
        T mm[8];
        double bb[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int k = k0 + u * stride;
          mm[u] = k < n ? __ldg(m + k) : (T)0;
          bb[u] = k < n ? p_ld(b + k) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) acc += (double)mm[u] * bb[u];
      }
    }
    acc = warp_sum(acc);
    if (lane == 0) part[warp] = acc;
    __syncthreads();
    if (row < n && w == 0 && lane == 0) {
      double t = 0.0;
      for (int k = 0; k < kTailWarps; ++k) t += part[warp + k];
      x[row] = (T)t;
    }
    __syncthreads();
  }
}

// Scalars of the solve, identical in every CTA.
struct PScal {
  double rho, rho_prev, alpha, atol, mean_r, mean_z, sum_r, bnorm2, rnorm2, pq, resid, mean_x;
  int it, done, conv, zero, status, total0;
};

// ---- V-cycle from zero on the CG residual r (vcycle_pcg's phases) ----------
// Leaves z_out, and mean(z), rho_prev, rho in the CTA's scalars.
template <class T>
__device__ void p_vcycle(const PSolve<T>& t, PBar& pb, PScal& sc, const double* dtab, const double* wtab,
                         const T* r, T* z_out) {
  const Geo& g = t.g;
  const uint8_t* fl = t.flags;
  const int gtid = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int nthr = (int)(gridDim.x * blockDim.x);
  const double mean_r = t.cfg.singular ? sc.mean_r : 0.0;
  // projected fine right-hand side of the preconditioner (BFromRS)
  auto bf = [&](int k) -> double { return (fl[k] & F_SOLV) ? p_ld(r + k) - mean_r : 0.0; };
  const double w = t.w0;
  const int Lv = t.nlev;
  const int sw = t.sweeps;
  const int singular = t.cfg.singular, nf = g.n_fluid;
  auto fin_z = [&](double* tt) {   // mean(z), rho = r.z - mean(z) sum(r)
    const double m = (singular && nf) ? tt[0] / nf : 0.0;
    sc.mean_z = m;
    sc.rho_prev = sc.rho;
    sc.rho = tt[1] - m * sc.sum_r;
  };
  const PLevel<T>& B0 = t.lv[0];
  if (Lv == 1) {   // single level: z = C (projected r)
    p_cells(g, [&](int c, int, int) { B0.b[c] = (T)bf(c); });
    p_sync(pb, PT_DENSE_RHS);
    const int lane = gtid & 31;
    for (int row = gtid >> 5; row < t.nc; row += nthr >> 5) {
      double acc = 0.0;
      for (int k = lane; k < t.nc; k += 32) acc += (double)t.C[(long)row * t.nc + k] * p_ld(B0.b + k);
      acc = warp_sum(acc);
      if (lane == 0) z_out[row] = (T)acc;
    }
    double s2[2] = {0.0, 0.0};
    p_sync(pb, PT_COARSEST);
    p_cells(g, [&](int c, int, int) {
      if (fl[c] & F_SOLV) {
        const double zc = p_ld(z_out + c);
        s2[0] += zc;
        s2[1] += p_ld(r + c) * zc;
      }
    });
    p_allreduce<2>(pb, t.partials, s2, PT_FINE_SMOOTH, fin_z);
    return;
  }
  T* cur[kPMaxLevels];
  int bottom = Lv - 1;   // level where the down sweep ends
  // ---- down: fine level
  if (sw == 1) {
    auto xv = [&](int k, int ii, int jj) -> double { return (double)(T)(p_wdinv(wtab, fl[k], ii, jj, g, w) * bf(k)); };
    p_cells(g, [&](int c, int i, int j) {
      const uint8_t f = fl[c];
      const double xc = xv(c, i, j);
      B0.xa[c] = (T)xc;
      B0.res[c] = (T)(bf(c) - p_apply(dtab, f, i, j, c, g, xv));
    });
    p_sync(pb, PT_FINE_PRE);
    cur[0] = B0.xa;
  } else {
    p_cells(g, [&](int c, int i, int j) { B0.xa[c] = (T)(p_wdinv(wtab, fl[c], i, j, g, w) * bf(c)); });
    p_sync(pb, PT_FINE_PRE);
    T* a = B0.xa;
    T* o = B0.xb;
    for (int k = 1; k < sw; ++k) {
      p_cells(g, [&](int c, int i, int j) {
        const uint8_t f = fl[c];
        const double xn = (double)(T)(p_ld(a + c) + p_wdinv(wtab, f, i, j, g, w) *
                                      (bf(c) - p_apply(dtab, f, i, j, c, g, [&](int kk, int, int) { return p_ld(a + kk); })));
        o[c] = (T)xn;
      });
      p_sync(pb, PT_SMOOTH);
      T* tmp = a; a = o; o = tmp;
    }
    p_cells(g, [&](int c, int i, int j) {
      B0.res[c] = (T)(bf(c) - p_apply(dtab, fl[c], i, j, c, g, [&](int kk, int, int) { return p_ld(a + kk); }));
    });
    p_sync(pb, PT_FINE_PRE);
    cur[0] = a;
  }
  // ---- down: coarse levels
  for (int l = 1; l < Lv; ++l) {
    const PLevel<T>& L = t.lv[l];
    const T* res_f = t.lv[l - 1].res;
    if (l == Lv - 1) {   // coarsest: b = R res, x = C b
      if (t.nc <= kPDenseMax) {
        if (blockIdx.x == 0) {   // one CTA, as the separate restrict+dense kernel
          __shared__ double sb[kPDenseMax];
          p_ell(L.R, L.lr, (int)threadIdx.x, (int)blockDim.x, [&](int c) { return p_ld(res_f + c); },
                [&](int row, double s) {
                  sb[row] = (double)(T)s;
                  L.b[row] = (T)s;
                });
          __syncthreads();
          const int wl = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
          for (int row = warp; row < t.nc; row += nw) {
            double acc = 0.0;
            for (int k = wl; k < t.nc; k += 32) acc += (double)t.C[(long)row * t.nc + k] * sb[k];
            acc = warp_sum(acc);
            if (wl == 0) L.xa[row] = (T)acc;
          }
        }
        p_sync(pb, PT_COARSEST | (l << 8));
      } else {
        p_ell(L.R, L.lr, gtid, nthr, [&](int c) { return p_ld(res_f + c); },
              [&](int row, double s) { L.b[row] = (T)s; });
        p_sync(pb, PT_RESTRICT | (l << 8));
        const int lane = gtid & 31;
        for (int row = gtid >> 5; row < t.nc; row += nthr >> 5) {
          double acc = 0.0;
          for (int k = lane; k < t.nc; k += 32) acc += (double)t.C[(long)row * t.nc + k] * p_ld(L.b + k);
          acc = warp_sum(acc);
          if (lane == 0) L.xa[row] = (T)acc;
        }
        p_sync(pb, PT_COARSEST | (l << 8));
      }
      cur[l] = L.xa;
      break;
    }
    p_ell(L.R, L.lr, gtid, nthr, [&](int c) { return p_ld(res_f + c); },
          [&](int row, double s) { L.b[row] = (T)s; });
    p_sync(pb, PT_RESTRICT | (l << 8));
    if (l == t.tail_level) {   // the cycle at and below l as one dense operator
      p_tail(t.tail, L.A.n, (const T*)L.b, L.xa);
      p_sync(pb, PT_TAIL | (l << 8));
      cur[l] = L.xa;
      bottom = l;
      break;
    }
    p_ell(L.A, L.la, gtid, nthr, [&](int c) { return (double)L.wd[c] * p_ld(L.b + c); },
          [&](int row, double s) {
            const double bx = p_ld(L.b + row);
            L.xa[row] = (T)((double)L.wd[row] * bx);
            L.res[row] = (T)(bx - s);
          });
    p_sync(pb, PT_PRE | (l << 8));
    T* a = L.xa;
    T* o = L.xb;
    if (sw > 1) {
      for (int k = 1; k < sw; ++k) {
        p_ell(L.A, L.la, gtid, nthr, [&](int c) { return p_ld(a + c); },
              [&](int row, double s) {
                o[row] = (T)(p_ld(a + row) + (double)L.wd[row] * (p_ld(L.b + row) - s));
              });
        p_sync(pb, PT_SMOOTH | (l << 8));
        T* tmp = a; a = o; o = tmp;
      }
      p_ell(L.A, L.la, gtid, nthr, [&](int c) { return p_ld(a + c); },
            [&](int row, double s) { L.res[row] = (T)(p_ld(L.b + row) - s); });
      p_sync(pb, PT_PRE | (l << 8));
    }
    cur[l] = a;
  }
  // ---- up
  for (int l = bottom - 1; l >= 0; --l) {
    const PLevel<T>& L = t.lv[l];
    const PLevel<T>& Lc = t.lv[l + 1];
    T* xf = cur[l];
    const T* xc = cur[l + 1];
    p_ell(Lc.P, Lc.lp, gtid, nthr, [&](int c) { return p_ld(xc + c); },
          [&](int row, double s) { xf[row] = (T)(p_ld(xf + row) + s); });
    p_sync(pb, PT_PROLONG | (l << 8));
    T* o = (xf == L.xa) ? L.xb : L.xa;
    for (int k = 1; k <= sw; ++k) {
      if (l == 0) {
        T* dst = (k == sw) ? z_out : o;
        const T* xs = xf;
        double s2[2] = {0.0, 0.0};
        p_cells(g, [&](int c, int i, int j) {
          const uint8_t f = fl[c];
          const double xn = (double)(T)(p_ld(xs + c) + p_wdinv(wtab, f, i, j, g, w) *
                                        (bf(c) - p_apply(dtab, f, i, j, c, g, [&](int kk, int, int) { return p_ld(xs + kk); })));
          dst[c] = (T)xn;
          if (k == sw && (f & F_SOLV)) {
            s2[0] += xn;
            s2[1] += p_ld(r + c) * xn;
          }
        });
        if (k == sw) p_allreduce<2>(pb, t.partials, s2, PT_FINE_SMOOTH, fin_z);
        else p_sync(pb, PT_SMOOTH);
        o = xf;
        xf = dst;
      } else {
        p_ell(L.A, L.la, gtid, nthr, [&](int c) { return p_ld(xf + c); },
              [&](int row, double s) {
                o[row] = (T)(p_ld(xf + row) + (double)L.wd[row] * (p_ld(L.b + row) - s));
              });
        p_sync(pb, PT_SMOOTH | (l << 8));
        T* tmp = xf; xf = o; o = tmp;
      }
    }
    cur[l] = xf;
  }
}

// ---- the solve ---------------------------------------------------------------
// rhs conditioning and r = b - A x0 (k_rhs_init), the CG passes (k_cg_pq,
// k_cg_xr, with the V-cycle for PC_MG), ||b - A x|| and the mean of x
// (k_finish_stats), the mean removal (k_finish_apply); CTA 0 then leaves the
// scalars those kernels would have left in S and I.  T = double.
template <class T, int PC>
__global__ void __launch_bounds__(kPThreads, 2) k_solve_persistent(PSolve<T> t) {
  __shared__ PScal sc;
  __shared__ double dtab[32], wtab[32];
  const Geo& g = t.g;
  const uint8_t* fl = t.flags;
  const SolveCfg cfg = t.cfg;
  const int nf = g.n_fluid;
  PBar pb{t.bar, 0u, 0u, (blockIdx.x == 0) ? t.trace : nullptr, 0, t.wait_ns};
  if (threadIdx.x < 32) {
    Geo g0 = g;   // fine_diag's sums without the Dirichlet terms
    g0.dir_w = g0.dir_e = g0.dir_s = g0.dir_n = 0;
    const double d = fine_diag((uint8_t)threadIdx.x, 1, 1, g0);
    dtab[threadIdx.x] = d;
    wtab[threadIdx.x] = t.w0 * (1.0 / d);
  }
  if (threadIdx.x == 0) {
    sc.total0 = t.I[I_TOTAL_IT];
    sc.status = 0;
  }
  // ---- b <- b - mean (solvable rows), r = b - A x0, norms
  {
    const double mean = cfg.singular ? t.S[S_MEAN_B] : 0.0;
    double acc[4] = {0, 0, 0, 0};
    double* b = t.b;
    T* x = t.x;
    T* r = t.r;
    const int has_x0 = t.has_x0;
    __syncthreads();
    p_cells(g, [&](int c, int i, int j) {
      const uint8_t f = fl[c];
      double bc = b[c];
      if (f & F_SOLV) bc = bc - mean;
      else bc = 0.0;
      b[c] = bc;
      double ax = 0.0;
      if (has_x0) ax = p_apply(dtab, f, i, j, c, g, [&](int k, int, int) { return (double)x[k]; });
      else x[c] = (T)0;
      const double rc = bc - ax;
      r[c] = (T)rc;
      const double d = p_diag(dtab, f, i, j, g);
      acc[0] += bc * bc;
      acc[1] += rc * rc;
      acc[2] += rc * (rc / d);
      if (f & F_SOLV) acc[3] += rc;
    });
    p_allreduce<4>(pb, t.partials, acc, PT_INIT, [&](double* tt) {
      sc.bnorm2 = tt[0];
      sc.atol = cfg.tol * sqrt(tt[0]);
      sc.rnorm2 = tt[1];
      sc.rho = tt[2];
      sc.rho_prev = 1.0;
      sc.sum_r = tt[3];
      sc.mean_r = nf ? tt[3] / nf : 0.0;
      sc.mean_z = 0.0;
      sc.it = 0;
      sc.zero = (tt[0] == 0.0);
      sc.conv = (tt[0] == 0.0) || (sqrt(tt[1]) < sc.atol);
      sc.done = sc.conv || cfg.maxiter <= 0;
    });
  }
  // ---- CG passes
  T* p_old = t.pa;
  T* p_new = t.pb;
  for (;;) {
    // block-uniform: sc is the same in every thread; the error word is read once
    if (__syncthreads_or(threadIdx.x == 0 && (sc.done || p_failed(pb)))) break;
    if (PC == PC_MG) p_vcycle<T>(t, pb, sc, dtab, wtab, t.r, t.z);
    {   // p = z + beta p_old, q = A p, p.q -> alpha
      const bool first = sc.it == 0;
      const double beta = first ? 0.0 : sc.rho / sc.rho_prev;
      const double mz = sc.mean_z;
      const T* r = t.r;
      const T* zr = t.z;
      const T* po = p_old;
      auto pval = [&](int k, int ii, int jj) -> double {
        const uint8_t fk = fl[k];
        double z;
        if (PC == PC_JACOBI) z = p_ld(r + k) / p_diag(dtab, fk, ii, jj, g);
        else z = (fk & F_SOLV) ? p_ld(zr + k) - mz : 0.0;
        if (first) return (double)(T)z;
        return (double)(T)(p_ld(po + k) * beta + z);
      };
      double acc[1] = {0.0};
      T* pn = p_new;
      T* q = t.q;
      p_cells(g, [&](int c, int i, int j) {
        const uint8_t f = fl[c];
        const double pc = pval(c, i, j);
        const double qc = p_apply(dtab, f, i, j, c, g, pval);
        pn[c] = (T)pc;
        q[c] = (T)qc;
        acc[0] += pc * qc;
      });
      p_allreduce<1>(pb, t.partials, acc, PT_PQ, [&](double* tt) {
        sc.pq = tt[0];
        sc.alpha = sc.rho / tt[0];
      });
    }
    {   // x += alpha p, r -= alpha q, norms, convergence of the next pass
      const double alpha = sc.alpha;
      double acc[3] = {0, 0, 0};
      T* x = t.x;
      T* r = t.r;
      const T* pn = p_new;
      const T* q = t.q;
      p_cells(g, [&](int c, int i, int j) {
        const uint8_t f = fl[c];
        const T pc = __ldcg(pn + c);
        const double xc = p_ld(x + c) + alpha * (double)pc;
        const double rc = (double)(T)(p_ld(r + c) - alpha * p_ld(q + c));
        x[c] = (T)xc;
        r[c] = (T)rc;
        acc[0] += rc * rc;
        if (PC == PC_JACOBI) acc[1] += rc * (rc / p_diag(dtab, f, i, j, g));
        if (f & F_SOLV) acc[2] += rc;
      });
      p_allreduce<3>(pb, t.partials, acc, PT_XR, [&](double* tt) {
        const int it = sc.it + 1;
        sc.it = it;
        sc.rnorm2 = tt[0];
        if (PC == PC_JACOBI) {
          sc.rho_prev = sc.rho;
          sc.rho = tt[1];
        }
        sc.sum_r = tt[2];
        sc.mean_r = nf ? tt[2] / nf : 0.0;
        sc.conv = sqrt(tt[0]) < sc.atol;
        sc.done = sc.conv || it >= cfg.maxiter;
      });
    }
    T* tmp = p_old; p_old = p_new; p_new = tmp;
  }
  // ---- ||b - A x||, mean of x, then x <- x - mean
  {
    const bool zero = sc.zero != 0;
    const T* x = t.x;
    const double* b = t.b;
    auto xv = [&](int k, int, int) -> double { return zero ? 0.0 : p_ld(x + k); };
    double acc[2] = {0, 0};
    p_cells(g, [&](int c, int i, int j) {
      const uint8_t f = fl[c];
      const double rc = __ldcg(b + c) - p_apply(dtab, f, i, j, c, g, xv);
      acc[0] += rc * rc;
      if (f & F_SOLV) acc[1] += xv(c, i, j);
    });
    p_allreduce<2>(pb, t.partials, acc, PT_FINISH, [&](double* tt) {
      const double nb = sqrt(sc.bnorm2);
      sc.resid = sqrt(tt[0]) / (nb > 1e-300 ? nb : 1.0);
      if (!sc.conv && sc.resid > fmax(cfg.tol * 10.0, 1e-8)) sc.status = -3;
      sc.mean_x = (cfg.singular && nf) ? tt[1] / nf : 0.0;
    });
  }
  {
    const bool zero = sc.zero != 0;
    const double m = sc.mean_x;
    T* x = t.x;
    p_cells(g, [&](int c, int, int) {
      const double v = (!zero && (fl[c] & F_SOLV)) ? p_ld(x + c) - m : 0.0;
      x[c] = (T)v;
    });
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double* S = t.S;
    int* I = t.I;
    S[S_BNORM2] = sc.bnorm2;
    S[S_ATOL] = sc.atol;
    S[S_RNORM2] = sc.rnorm2;
    S[S_RHO] = sc.rho;
    S[S_RHO_PREV] = sc.rho_prev;
    S[S_ALPHA] = sc.alpha;
    S[S_PQ] = sc.pq;
    S[S_SUM_R] = sc.sum_r;
    S[S_MEAN_R] = sc.mean_r;
    S[S_MEAN_Z] = sc.mean_z;
    S[S_RESID] = sc.resid;
    S[S_MEAN_X] = sc.mean_x;
    I[I_IT] = sc.it;
    I[I_TOTAL_IT] = sc.total0 + sc.it;
    I[I_ZERO_RHS] = sc.zero;
    I[I_CONVERGED] = sc.conv;
    I[I_DONE] = sc.done;
    I[I_STATUS] = sc.status;
    if (p_failed(pb)) {
      I[I_STATUS] = kPStatusTimeout;
      I[I_HEALTH] |= 8;
    }
    if (pb.trace) pb.trace[0] = (unsigned long long)pb.ntr;
  }
}

}  // namespace pcfd
