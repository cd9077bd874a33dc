// Fine-level Poisson kernels: right-hand-side conditioning, the conjugate-
// gradient recurrence (Jacobi- or multigrid-preconditioned), damped Jacobi,
// red/black SOR, residual norms and result normalisation.
//
// The fine operator is applied matrix-free from one flag byte per cell.  CG
// follows SciPy's recurrence (scipy/sparse/linalg/_isolve/iterative.py:311 in
// SciPy 1.18.1, as called by pycfd/core/pressure.py:388-391 and :619-623):
// each pass tests the recurrence residual first, then z = M r, rho = r.z,
// p = z + (rho/rho_prev) p, q = A p, alpha = rho/(p.q), x += alpha p,
// r -= alpha q.  Two kernels per pass: p/q/(p.q) and x/r/(r.r, r.z).
// Vector kernels are templated on the storage type T (double, or float for the
// inner solve of the mixed form); scalars and dot products are always double.
#pragma once
#include "common.cuh"

namespace pcfd {

enum Precond { PC_JACOBI = 0, PC_MG = 1 };

// Solve-level constants the finishers need.
struct SolveCfg {
  double tol;
  int maxiter;
  int singular;
  int check_every;   // stationary solvers: residual cadence
};

// Loop control of a solve recorded in a CUDA graph: the finisher of the kernel
// that decides convergence sets the WHILE node's condition (0 ends the loop).
struct LoopCtl {
  cudaGraphConditionalHandle handle;
  int active;
  __device__ __forceinline__ void set(bool keep_going) const {
    if (active) cudaGraphSetConditional(handle, keep_going ? 1u : 0u);
  }
};

template <class T> struct VecRef { T* p; };

// ---- right-hand side and initial residual --------------------------------
// b <- b_raw - mean (solvable rows, singular systems), r = b - A x0 (x0 = 0
// when has_x0 == 0), with ||b||^2, ||r||^2, r.(r/d) and sum_solvable(r).
// (pycfd/core/pressure.py:300-308; scipy cg: r = b - A x0)
template <class T>
__global__ void k_rhs_init(double* __restrict__ b, T* __restrict__ x, T* __restrict__ r,
                           const uint8_t* __restrict__ flags, Geo g, SolveCfg cfg,
                           int has_x0, double* __restrict__ S, int* __restrict__ I, RedBuf rb,
                           LoopCtl loop) {
  pdl_begin();
  const double mean = cfg.singular ? S[S_MEAN_B] : 0.0;
  double acc[4] = {0, 0, 0, 0};
  FOR_CELLS(g) {
    const int c = i * g.ny + j;
    const uint8_t f = flags[c];
    double bc = b[c];
    if (f & F_SOLV) bc = bc - mean;
    else bc = 0.0;
    b[c] = bc;
    double ax = 0.0;
    if (has_x0) ax = fine_apply<double>(f, i, j, c, g, [&](int k, int, int) { return (double)x[k]; });
    else x[c] = (T)0;
    const double rc = bc - ax;
    r[c] = (T)rc;
    const double d = fine_diag(f, i, j, g);
    acc[0] += bc * bc;
    acc[1] += rc * rc;
    acc[2] += rc * (rc / d);
    if (f & F_SOLV) acc[3] += rc;
  }
  grid_reduce<4>(acc, rb, [&](double* t) {
    S[S_BNORM2] = t[0];
    S[S_ATOL] = cfg.tol * sqrt(t[0]);
    S[S_RNORM2] = t[1];
    S[S_RHO] = t[2];
    S[S_RHO_PREV] = 1.0;
    S[S_SUM_R] = t[3];
    S[S_MEAN_R] = g.n_fluid ? t[3] / g.n_fluid : 0.0;
    I[I_IT] = 0;
    I[I_ZERO_RHS] = (t[0] == 0.0);
    const bool conv = (t[0] == 0.0) || (sqrt(t[1]) < S[S_ATOL]);
    I[I_CONVERGED] = conv;
    I[I_DONE] = conv || cfg.maxiter <= 0;
    I[I_STATUS] = 0;
    loop.set(!I[I_DONE]);
  });
}

// p = z + beta p_old with z = r/d (Jacobi) or z = z_raw - mean_z on solvable
// rows (multigrid; z_raw from the V-cycle), q = A p, and p.q -> alpha.
template <class T, int PC>
__global__ void k_cg_pq(const T* __restrict__ r, const T* __restrict__ zraw,
                        const T* __restrict__ p_old, T* __restrict__ p_new, T* __restrict__ q,
                        const uint8_t* __restrict__ flags, Geo g, double* __restrict__ S,
                        const int* __restrict__ I, RedBuf rb) {
  pdl_begin();
  const bool first = I[I_IT] == 0;
  const double beta = first ? 0.0 : S[S_RHO] / S[S_RHO_PREV];
  const double mz = S[S_MEAN_Z];
  auto pval = [&](int k, int ii, int jj) -> double {
    const uint8_t fk = flags[k];
    double z;
    if (PC == PC_JACOBI) z = (double)r[k] / fine_diag(fk, ii, jj, g);
    else z = (fk & F_SOLV) ? (double)zraw[k] - mz : 0.0;
    if (first) return (double)(T)z;
    return (double)(T)((double)p_old[k] * beta + z);
  };
  double acc[1] = {0.0};
  uint8_t fv[kStripRows];
  strip_cells<true>(g, pval, [&](int u, int c) { fv[u] = flags[c]; },
                    [&](int u, int c, int i, int j, double pc, double pw, double pe, double ps, double pn) {
                      const double qc = fine_apply5(fv[u], i, j, g, pc, pw, pe, ps, pn);
                      p_new[c] = (T)pc;
                      q[c] = (T)qc;
                      acc[0] += pc * qc;
                    });
  grid_reduce<1>(acc, rb, [&](double* t) {
    S[S_PQ] = t[0];
    S[S_ALPHA] = S[S_RHO] / t[0];
  });
}

// x += alpha p, r -= alpha q; ||r||^2, r.(r/d), sum_solvable(r); convergence
// test of the next pass (scipy's top-of-loop ||r|| < atol), iteration count.
// p_keep != nullptr: also store p there, so a recorded loop body always reads
// the previous direction from the same buffer.
template <class T, int PC>
__global__ void k_cg_xr(T* __restrict__ x, T* __restrict__ r, const T* __restrict__ p,
                        const T* __restrict__ q, T* __restrict__ p_keep,
                        const uint8_t* __restrict__ flags, Geo g, SolveCfg cfg,
                        double* __restrict__ S, int* __restrict__ I, RedBuf rb, LoopCtl loop) {
  pdl_begin();
  const double alpha = S[S_ALPHA];
  double acc[3] = {0, 0, 0};
  T pv[kStripRows], xv[kStripRows], rv[kStripRows], qv[kStripRows];
  uint8_t fv[kStripRows];
  strip_cells<false>(
      g, [](int, int, int) { return 0.0; },
      [&](int u, int c) {
        pv[u] = p[c];
        xv[u] = x[c];
        rv[u] = r[c];
        qv[u] = q[c];
        fv[u] = flags[c];
      },
      [&](int u, int c, int i, int j, double, double, double, double, double) {
        const T pc = pv[u];
        const double xc = (double)xv[u] + alpha * (double)pc;
        const double rc = (double)(T)((double)rv[u] - alpha * (double)qv[u]);
        if (p_keep) p_keep[c] = pc;
        x[c] = (T)xc;
        r[c] = (T)rc;
        acc[0] += rc * rc;
        if (PC == PC_JACOBI) acc[1] += rc * (rc / fine_diag(fv[u], i, j, g));
        if (fv[u] & F_SOLV) acc[2] += rc;
      });
  grid_reduce<3>(acc, rb, [&](double* t) {
    const int it = I[I_IT] + 1;
    I[I_IT] = it;
    I[I_TOTAL_IT] += 1;
    S[S_RNORM2] = t[0];
    if (PC == PC_JACOBI) { S[S_RHO_PREV] = S[S_RHO]; S[S_RHO] = t[1]; }
    S[S_SUM_R] = t[2];
    S[S_MEAN_R] = g.n_fluid ? t[2] / g.n_fluid : 0.0;
    const bool conv = sqrt(t[0]) < S[S_ATOL];
    I[I_CONVERGED] = conv;
    I[I_DONE] = conv || it >= cfg.maxiter;
    loop.set(!I[I_DONE]);
  });
}

// ---- result normalisation -------------------------------------------------
// ||b - A x||^2 and sum_solvable(x) -> last_residual and the mean
// (pycfd/core/pressure.py:310-322).  keep_resid: the stationary solvers
// report the residual of their last check instead.
template <class T>
__global__ void k_finish_stats(const T* __restrict__ x, const double* __restrict__ b,
                               const uint8_t* __restrict__ flags, Geo g, SolveCfg cfg,
                               int pcg, double* __restrict__ S, int* __restrict__ I, RedBuf rb) {
  pdl_begin();
  const bool zero = I[I_ZERO_RHS] != 0;
  auto xv = [&](int k, int, int) -> double { return zero ? 0.0 : (double)x[k]; };
  double acc[2] = {0, 0};
  FOR_CELLS(g) {
    const int c = i * g.ny + j;
    const uint8_t f = flags[c];
    if (pcg) {
      const double rc = b[c] - fine_apply<double>(f, i, j, c, g, xv);
      acc[0] += rc * rc;
    }
    if (f & F_SOLV) acc[1] += xv(c, i, j);
  }
  grid_reduce<2>(acc, rb, [&](double* t) {
    const double nb = sqrt(S[S_BNORM2]);
    if (pcg) {
      S[S_RESID] = sqrt(t[0]) / (nb > 1e-300 ? nb : 1.0);
      if (!I[I_CONVERGED] && S[S_RESID] > fmax(cfg.tol * 10.0, 1e-8)) I[I_STATUS] = -3;
    }
    S[S_MEAN_X] = (cfg.singular && g.n_fluid) ? t[1] / g.n_fluid : 0.0;
  });
}

// x <- x - mean on solvable rows, 0 elsewhere; also the double copy for the
// projection (xo may alias x when T is double).
template <class T>
__global__ void k_finish_apply(T* x, double* xo,
                               const uint8_t* __restrict__ flags, Geo g,
                               const double* __restrict__ S, const int* __restrict__ I) {
  pdl_begin();
  const bool zero = I[I_ZERO_RHS] != 0;
  const double m = S[S_MEAN_X];
  FOR_CELLS(g) {
    const int c = i * g.ny + j;
    const double v = (!zero && (flags[c] & F_SOLV)) ? (double)x[c] - m : 0.0;
    x[c] = (T)v;
    xo[c] = v;
  }
}

// ---- stationary solvers -----------------------------------------------------
// Initial iterate and right-hand side of Jacobi/SOR/standalone multigrid:
// b final (mean removed), x = x0 with non-solvable rows zeroed (or 0),
// ||b||^2 and sum_solvable(x) (pycfd/core/pressure.py:420-430, :506-513).
__global__ void k_stationary_init(double* __restrict__ b, double* __restrict__ x,
                                  const uint8_t* __restrict__ flags, Geo g, SolveCfg cfg,
                                  int has_x0, int project_x0, double* __restrict__ S,
                                  int* __restrict__ I, RedBuf rb) {
  pdl_begin();
  const double mean = cfg.singular ? S[S_MEAN_B] : 0.0;
  double acc[3] = {0, 0, 0};
  FOR_CELLS(g) {
    const int c = i * g.ny + j;
    const uint8_t f = flags[c];
    const double bc = (f & F_SOLV) ? b[c] - mean : 0.0;
    b[c] = bc;
    const double xc = (has_x0 && (f & F_SOLV)) ? x[c] : 0.0;
    x[c] = xc;
    acc[0] += bc * bc;
    if (f & F_SOLV) { acc[1] += bc; acc[2] += xc; }
  }
  grid_reduce<3>(acc, rb, [&](double* t) {
    S[S_BNORM2] = t[0];
    // standalone multigrid projects b and x0 once more (multigrid.py:490-493)
    S[S_MEAN_B] = (project_x0 && cfg.singular && g.n_fluid) ? t[1] / g.n_fluid : 0.0;
    S[S_MEAN_X] = (project_x0 && cfg.singular && g.n_fluid) ? t[2] / g.n_fluid : 0.0;
    S[S_RES_PREV] = 0.0;
    I[I_IT] = 0;
    I[I_DONE] = 0;
    I[I_CONVERGED] = 0;
    I[I_STATUS] = 0;
    I[I_STALLED] = 0;
    I[I_ZERO_RHS] = 0;
  });
}

// One damped-Jacobi sweep p <- p + omega*dinv*(b - A p) on the iterate with its
// pending mean removed, plus the new fluid sum (pycfd/core/pressure.py:432-436).
__global__ void k_jacobi_sweep(const double* __restrict__ xin, double* __restrict__ xout,
                               const double* __restrict__ b, const uint8_t* __restrict__ flags,
                               Geo g, double omega, int singular, double* __restrict__ S,
                               int* __restrict__ I, RedBuf rb) {
  pdl_begin();
  const double m = S[S_MEAN_X];
  auto xe = [&](int k, int, int) -> double { return (flags[k] & F_SOLV) ? xin[k] - m : xin[k]; };
  double acc[1] = {0.0};
  FOR_CELLS(g) {
    const int c = i * g.ny + j;
    const uint8_t f = flags[c];
    const double d = fine_diag(f, i, j, g);
    const double dinv = 1.0 / d;
    const double xn = xe(c, i, j) + omega * dinv * (b[c] - fine_apply<double>(f, i, j, c, g, xe));
    xout[c] = xn;
    if (f & F_SOLV) acc[0] += xn;
  }
  grid_reduce<1>(acc, rb, [&](double* t) {
    S[S_MEAN_X] = (singular && g.n_fluid) ? t[0] / g.n_fluid : 0.0;
    I[I_IT] += 1;
    I[I_TOTAL_IT] += 1;
  });
}

// One red (colour 0) or black (colour 1) SOR half-sweep in place
// (pycfd/core/pressure.py:514-517).  Values of the colour being updated and, on
// the red pass, its neighbours still carry the previous sweep's mean; the
// black pass finishes the new fluid mean.
__global__ void k_sor_half(double* __restrict__ x, const double* __restrict__ b,
                           const uint8_t* __restrict__ flags, Geo g, double omega, int colour,
                           int singular, double* __restrict__ S, int* __restrict__ I, RedBuf rb) {
  pdl_begin();
  const double m = S[S_MEAN_X];
  // red pass: every value is in the old frame; black pass: red neighbours are new.
  auto xe = [&](int k, int ii, int jj) -> double {
    const bool adj = (flags[k] & F_SOLV) && (colour == 0 || ((ii + jj) & 1) == 1);
    return adj ? x[k] - m : x[k];
  };
  double acc[1] = {0.0};
  FOR_CELLS(g) {
    const int c = i * g.ny + j;
    if (((i + j) & 1) != colour) continue;
    const uint8_t f = flags[c];
    const double d = fine_diag(f, i, j, g);
    double off = 0.0;
    double cw = g.cx, ce = g.cx, cs = g.cy, cn = g.cy;
    if (g.met) {   // stretched: the face coefficients of this cell
      const Metrics M(g);
      cw = M.cw(i, j);
      ce = M.ce(i, j);
      cs = M.cs(i, j);
      cn = M.cn(i, j);
    }
    if (f & F_W) { const int a = wrap_w(i, g); off += cw * xe(a * g.ny + j, a, j); }
    if (f & F_E) { const int a = wrap_e(i, g); off += ce * xe(a * g.ny + j, a, j); }
    if (f & F_S) { const int bb = wrap_s(j, g); off += cs * xe(i * g.ny + bb, i, bb); }
    if (f & F_N) { const int bb = wrap_n(j, g); off += cn * xe(i * g.ny + bb, i, bb); }
    const double xn = (1.0 - omega) * xe(c, i, j) + omega * (b[c] - off) / d;
    x[c] = xn;
    if (f & F_SOLV) acc[0] += xn;
  }
  grid_reduce<1>(acc, rb, [&](double* t) {
    if (colour == 0) {
      S[S_SUM_R] = t[0];
    } else {
      S[S_MEAN_X] = (singular && g.n_fluid) ? (S[S_SUM_R] + t[0]) / g.n_fluid : 0.0;
      I[I_IT] += 1;
      I[I_TOTAL_IT] += 1;
    }
  });
}

// ||b - A(x - m)|| / ||b|| on the iterate with its pending mean m, then the
// stopping rule of the calling solver:
//   mode 0 (Jacobi/SOR): done when res < tol or the sweep budget is spent;
//   mode 1 (standalone multigrid, pycfd/core/multigrid.py:498-511): also stop
//   after three cycles that fail to shrink the residual by 0.995.
// write_back: store the projected iterate x - m (multigrid projects every cycle).
__global__ void k_resnorm(double* __restrict__ x, const double* __restrict__ b,
                          const uint8_t* __restrict__ flags, Geo g, SolveCfg cfg, int mode,
                          int count_cycle, int pending, double* __restrict__ S, int* __restrict__ I,
                          RedBuf rb, LoopCtl loop) {
  pdl_begin();
  const double m = pending ? S[S_MEAN_X] : 0.0;
  auto xe = [&](int k, int, int) -> double { return (flags[k] & F_SOLV) ? x[k] - m : 0.0; };
  double acc[1] = {0.0};
  FOR_CELLS(g) {
    const int c = i * g.ny + j;
    const double rc = b[c] - fine_apply<double>(flags[c], i, j, c, g, xe);
    acc[0] += rc * rc;
  }
  grid_reduce<1>(acc, rb, [&](double* t) {
    const double nb = sqrt(S[S_BNORM2]);
    const double res = sqrt(t[0]) / (nb > 1e-300 ? nb : 1.0);
    const int it = I[I_IT] + (count_cycle ? 1 : 0);
    if (count_cycle) { I[I_IT] = it; I[I_TOTAL_IT] += 1; }
    const double prev = S[S_RES_PREV];
    S[S_RESID] = res;
    const bool conv = res < cfg.tol;
    I[I_CONVERGED] = conv;
    if (mode == 1) {
      if (count_cycle) I[I_STALLED] = (res > 0.995 * prev) ? I[I_STALLED] + 1 : 0;
      S[S_RES_PREV] = res;
      I[I_DONE] = !(it < cfg.maxiter && res >= cfg.tol && I[I_STALLED] < 3);
    } else {
      I[I_DONE] = conv || it >= cfg.maxiter;
    }
    if (I[I_DONE] && res > cfg.tol) I[I_STATUS] = -4;
    loop.set(!I[I_DONE]);
  });
}

// ---- mixed form: FP64 iterative refinement around an FP32 MG-PCG ----------
// One refinement pass: r = b - A x in FP64 (first pass: finalise b from the raw
// right-hand side and take x from the warm start or zero), the outer stopping
// rule ||r|| < tol ||b|| on this true residual, and the set-up of the inner
// FP32 solve A e = r from e = 0 (r32 = r).  The inner solve stops at
// max(inner_tol ||r||, kIrLastFraction tol ||b||): a pass that only has to take
// the residual the rest of the way to the outer target stops there instead of
// reducing it by the full inner_tol (the outer test on the true residual still
// decides convergence).
constexpr double kIrLastFraction = 0.5;
__global__ void k_ir_residual(double* __restrict__ b, double* __restrict__ x,
                              float* __restrict__ r32, float* __restrict__ e32,
                              const uint8_t* __restrict__ flags, Geo g, SolveCfg cfg,
                              double inner_tol, int max_passes, int first, int has_x0,
                              double* __restrict__ S, int* __restrict__ I, RedBuf rb,
                              LoopCtl outer) {
  pdl_begin();
  const double mean = (first && cfg.singular) ? S[S_MEAN_B] : 0.0;
  double acc[3] = {0, 0, 0};
  FOR_CELLS(g) {
    const int c = i * g.ny + j;
    const uint8_t f = flags[c];
    double bc = b[c];
    if (first) {
      bc = (f & F_SOLV) ? bc - mean : 0.0;
      b[c] = bc;
      if (!has_x0) x[c] = 0.0;
    }
    const double ax = (first && !has_x0) ? 0.0
                      : fine_apply<double>(f, i, j, c, g, [&](int k, int, int) { return x[k]; });
    const double rc = bc - ax;
    r32[c] = (float)rc;
    e32[c] = 0.0f;
    acc[0] += rc * rc;
    if (f & F_SOLV) acc[1] += (double)(float)rc;
    if (first) acc[2] += bc * bc;
  }
  grid_reduce<3>(acc, rb, [&](double* t) {
    if (first) {
      S[S_IR_BNORM] = sqrt(t[2]);
      S[S_BNORM2_0] = t[2];
      S[S_BNORM2] = t[2];   // ||b||^2 of the outer system: the reported residual's scale
      I[I_IR_IT] = 0;
      I[I_ZERO_RHS] = (t[2] == 0.0);
      I[I_STATUS] = 0;
    }
    const double nb = S[S_IR_BNORM];
    S[S_IR_RNORM2] = t[0];
    const bool conv = (nb == 0.0) || (sqrt(t[0]) < cfg.tol * nb);
    const bool done = conv || I[I_IR_IT] >= max_passes;
    I[I_CONVERGED] = conv;
    I[I_IR_DONE] = done;
    // inner solve from e = 0: its residual is r itself
    S[S_ATOL] = fmax(inner_tol * sqrt(t[0]), kIrLastFraction * cfg.tol * nb);
    S[S_RNORM2] = t[0];
    S[S_SUM_R] = t[1];
    S[S_MEAN_R] = g.n_fluid ? t[1] / g.n_fluid : 0.0;
    I[I_IT] = 0;
    I[I_DONE] = done;
    outer.set(!done);
  });
}

// Arm the inner solve's loop from the flags of the last refinement pass.
__global__ void k_ir_arm(const int* __restrict__ I, LoopCtl inner) {
  pdl_begin();
  if (threadIdx.x == 0) inner.set(!I[I_DONE]);
}

// x += e (FP32 correction promoted to FP64) on solvable rows; count the pass.
__global__ void k_ir_update(double* __restrict__ x, const float* __restrict__ e32,
                            const uint8_t* __restrict__ flags, Geo g, int* __restrict__ I) {
  pdl_begin();
  FOR_CELLS(g) {
    const int c = i * g.ny + j;
    if (flags[c] & F_SOLV) x[c] = x[c] + (double)e32[c];
  }
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0 && threadIdx.y == 0) I[I_IR_IT] += 1;
}

// Device-side time-step control (pycfd/core/timestepper.py:94-142) from the
// field statistics of the current state left in the scalar block:
// dt = min(cfl/(umax/dx + vmax/dy), viscous limit, dt_cap) (the same double
// operations, so the same dt), health flags on the unclamped dt (sticky bits:
// 1 non-finite, 2 velocity above the divergence limit, 4 collapsed dt), the
// clamp onto t_end, the donor-cell blend, and the clock.
struct DtControl {
  int adaptive;
  double cfl, visc_limit, dt_cap, t_end, dx, dy;
  int blend_mode;     // 0 fixed blend (below), 1 follow the Courant number
  double blend;
  double steady_tol;  // device loop: stop once max|du|/dt falls below it (0: never)
  int history;        // 1: the step is gated and appends a row to the device history
  double ke_scale;    // the history's kinetic energy factor: dx dy (uniform), 1 (stretched: integrated per cell)
};

__device__ __forceinline__ void adaptive_dt_update(double* S, int* I, const DtControl& c) {
  const double umax = S[S_STAT0], vmax = S[S_STAT0 + 1];
  double dt = c.dt_cap;
  if (c.adaptive) {
    const double scale = umax / c.dx + vmax / c.dy;
    const double dt_conv = scale > 1.0e-12 ? c.cfl / scale : INFINITY;
    dt = fmin(fmin(dt_conv, c.visc_limit), c.dt_cap);
  }
  int h = I[I_HEALTH];
  if (S[S_STAT0 + 7] != 0.0) h |= 1;
  if (fmax(umax, vmax) > 1.0e6) h |= 2;
  if (dt < 1.0e-8) h |= 4;
  I[I_HEALTH] = h;
  const double t = S[S_T];
  dt = fmin(dt, c.t_end - t);
  S[S_DT] = dt;
  S[S_BLEND] = c.blend_mode ? fmin(1.0, 1.2 * fmax(umax * dt / c.dx, vmax * dt / c.dy)) : c.blend;
  S[S_T] = t + dt;
  I[I_STEPS] += 1;
  I[I_TOTAL_IT] = 0;
}

__global__ void k_adaptive_dt(double* __restrict__ S, int* __restrict__ I, DtControl c) {
  pdl_begin();
  if (threadIdx.x != 0) return;
  adaptive_dt_update(S, I, c);
}

// Gate of a device-loop step (TimeStepper.run, pycfd/core/timestepper.py:183-231):
// a frozen run takes no more steps; once the clock is within 1e-12 of the end
// time (the reference's loop condition) it freezes (2); the dt and health
// checks run on the unclamped dt as in k_adaptive_dt, and a health flag freezes
// the run (1) with the clock left at the last good step -- the step the
// reference refuses with DivergenceError.  `gate` is the condition of the
// graph's IF node around the step.
__global__ void k_step_gate(double* __restrict__ S, int* __restrict__ I, DtControl c, LoopCtl gate) {
  if (threadIdx.x != 0) return;
  if (I[I_FROZEN]) {
    gate.set(false);
    return;
  }
  if (!(S[S_T] < c.t_end - 1e-12)) {
    I[I_FROZEN] = 2;
    gate.set(false);
    return;
  }
  const double t0 = S[S_T], dt0 = S[S_DT];
  const int n0 = I[I_STEPS];
  adaptive_dt_update(S, I, c);
  if (I[I_HEALTH] != 0) {
    S[S_T] = t0;
    S[S_DT] = dt0;
    I[I_STEPS] = n0;
    I[I_FROZEN] = 1;
    gate.set(false);
    return;
  }
  gate.set(true);
}

// One row of the device history after a step (timestepper.py:251-266): step,
// t, dt, CFL number, max|div u|, kinetic energy, last Poisson residual, body
// force (fx, fy), max|du|/dt.  The field statistics of the new state (and its
// change over the step) are in the stats slots.  A run whose rate of change
// falls below steady_tol freezes (3) after this step, as the reference stops.
constexpr int kHistCols = 10;
constexpr int kHistRows = 4096;   // rows the device history holds between reads

__global__ void k_history_append(double* __restrict__ S, int* __restrict__ I, double* __restrict__ hist,
                                 int cap, DtControl c) {
  if (threadIdx.x != 0) return;
  const double dt = S[S_DT];
  const double umax = S[S_STAT0], vmax = S[S_STAT0 + 1];
  const double rate = fmax(S[S_STAT0 + 2], S[S_STAT0 + 3]) / dt;
  const int row = I[I_HIST];
  if (row < cap) {
    double* h = hist + (long)row * kHistCols;
    h[0] = (double)I[I_STEPS];
    h[1] = S[S_T];
    h[2] = dt;
    h[3] = dt * (umax / c.dx + vmax / c.dy);
    h[4] = S[S_STAT0 + 4];
    h[5] = S[S_STAT0 + 5] * c.ke_scale;
    h[6] = S[S_RESID];
    h[7] = S[S_FX];
    h[8] = S[S_FY];
    h[9] = rate;
  }
  I[I_HIST] = row + 1;
  if (c.steady_tol > 0.0 && rate < c.steady_tol) I[I_FROZEN] = 3;
}

__global__ void k_set_clock(double* __restrict__ S, int* __restrict__ I, double t) {
  pdl_begin();
  if (threadIdx.x == 0) {
    S[S_T] = t;
    I[I_STEPS] = 0;
    I[I_HEALTH] = 0;
    I[I_FROZEN] = 0;
    I[I_HIST] = 0;
  }
}

// Start of a call: step parameters into the device scalar block (kernel
// arguments, so no host synchronisation is needed) and the per-call counters.
__global__ void k_begin(double* __restrict__ S, int* __restrict__ I, double dt, double blend) {
  pdl_begin();
  if (threadIdx.x == 0) {
    S[S_DT] = dt;
    S[S_BLEND] = blend;
    I[I_TOTAL_IT] = 0;
  }
}

// Apply a pending mean: x <- x - S[slot] on solvable rows.
__global__ void k_apply_mean(double* __restrict__ x, const uint8_t* __restrict__ flags, Geo g,
                             const double* __restrict__ S, int slot) {
  pdl_begin();
  const double m = S[slot];
  FOR_CELLS(g) {
    const int c = i * g.ny + j;
    if (flags[c] & F_SOLV) x[c] = x[c] - m;
  }
}

}  // namespace pcfd
