/*
 * pycfd_b200 -- C ABI of the B200-native projection hot path.
 *
 * The reference solver (kiliancmd/pycfd) is pure Python and exposes no foreign
 * function interface; the entry points below are the calls its Python layer
 * would bind if the per-timestep path were moved behind one.  Each one names
 * the reference function or method it replaces (file:line in the reference
 * project).  All device pointers are CUDA global memory on the current device;
 * every launch goes to the `stream` argument (a cudaStream_t, NULL = legacy
 * default stream).  Nothing here takes a framework tensor type.
 *
 * Array layout (pycfd/core/mesh.py:13-38): row-major doubles with y fastest,
 *   u: (nx+3) x (ny+2)   v: (nx+2) x (ny+3)   p: (nx+2) x (ny+2)
 * Poisson vectors are flat (nx*ny), index i*ny + j (pycfd/core/pressure.py:178).
 *
 * Every function returns 0 on success or a negative PCFD_E_* code;
 * pycfd_last_error() gives the message of the last failure on this thread.
 */
#ifndef PYCFD_B200_H
#define PYCFD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define PCFD_OK 0
#define PCFD_E_ARG (-1)        /* bad argument: maps to ValueError          */
#define PCFD_E_CUDA (-2)       /* CUDA runtime error                         */
#define PCFD_E_NOCONV (-3)     /* iterative solve failed: RuntimeError       */
#define PCFD_E_STALL (-4)      /* SOR/Jacobi/MG stalled: RuntimeError        */
#define PCFD_E_UNSUPPORTED (-5) /* configuration the GPU path rejects        */

/* ---- boundary kinds (pycfd/config.py:85-94) ----------------------------- */
#define PCFD_BC_NO_SLIP 0
#define PCFD_BC_MOVING_WALL 1
#define PCFD_BC_INLET 2
#define PCFD_BC_OUTLET 3
#define PCFD_BC_PRESSURE_OUTLET 4
#define PCFD_BC_PERIODIC 5
#define PCFD_BC_SYMMETRY 6

/* ---- pressure solvers (pycfd/config.py:74-82; "direct" is not provided) -- */
#define PCFD_SOLVER_CG 1
#define PCFD_SOLVER_JACOBI 2
#define PCFD_SOLVER_SOR 3
#define PCFD_SOLVER_MULTIGRID 4
#define PCFD_SOLVER_MGCG 5

/* ---- time schemes (pycfd/config.py:46-59) ------------------------------- */
#define PCFD_EULER 0
#define PCFD_RK2 1
#define PCFD_RK3 2

/* ---- precision forms ---------------------------------------------------- */
#define PCFD_FP64 0
#define PCFD_MIXED 1   /* FP32 MG-PCG inner solve inside FP64 iterative refinement */

#define PCFD_MAX_BODIES 8

typedef struct pycfd_solver pycfd_solver;

/* One multigrid level as built on the host (pycfd/core/multigrid.py:293-321).
 * Level 0 is the fine Poisson operator, which the device applies matrix-free
 * from the cell flags; its a_* fields are ignored.  For l >= 1, A_l is given
 * in CSR and P_l (the prolongation from level l to level l-1, n_{l-1} x n_l)
 * in CSR; restriction is its transpose, formed on the device side.         */
typedef struct {
    int n;                       /* unknowns on this level                   */
    int shape_x, shape_y;        /* grid this level's unknowns lie on        */
    double weight;               /* damped-Jacobi weight (4/3)/rho           */
    const double* weighted_dinv; /* n: weight / diag (ignored on level 0)    */
    const uint8_t* active;       /* n: 1 where the row is an active unknown  */
    const int64_t* a_indptr;     /* CSR of A_l (l >= 1)                      */
    const int32_t* a_indices;
    const double* a_data;
    const int64_t* p_indptr;     /* CSR of P_l (l >= 1)                      */
    const int32_t* p_indices;
    const double* p_data;
    const int64_t* m_indptr;     /* optional, 1 <= l <= tail level: CSR of the
                                    fused restriction R_l (I - A_{l-1} W_{l-1})
                                    (n_l x n_{l-1}; one sweep from zero and the
                                    restriction of its residual in one pass) */
    const int32_t* m_indices;
    const double* m_data;
} pycfd_mg_level;

typedef struct {
    int nx, ny;
    double dx, dy, nu;                        /* dx, dy: the uniform spacing; on a stretched
                                                 mesh the smallest cell width / height (what
                                                 the time-step limits answer to,
                                                 timestepper.py:91-119)                */
    double body_fx, body_fy;                  /* config.body_force          */
    int bc_kind[4];                           /* left, right, bottom, top   */
    double bc_velocity[4];
    double bc_p_ref[4];
    const double* bc_profile[4];              /* parabolic inlet normal-face line
                                                 (full ghosted line), or NULL */
    const uint8_t* solid;                     /* nx*ny cell mask, or NULL    */
    const uint8_t* body_id;                   /* nx*ny: body index+1 of a solid
                                                 cell when several bodies report
                                                 separate forces, else NULL  */
    int n_bodies;                             /* 0 or 2..PCFD_MAX_BODIES     */
    int solver_kind;                          /* PCFD_SOLVER_*               */
    double tol;
    int maxiter;
    double sor_omega;
    int mg_sweeps;
    int time_scheme;                          /* PCFD_EULER/RK2/RK3          */
    int precision;                            /* PCFD_FP64 / PCFD_MIXED      */
    double inner_tol;                         /* mixed: inner FP32 relative tol */
    int n_levels;                             /* multigrid solvers only      */
    const pycfd_mg_level* levels;
    const double* coarsest_inverse;           /* n_L x n_L row-major pseudo-inverse
                                                 of the coarsest operator    */
    int coarse_cluster_rows;                  /* levels with at most this many rows run
                                                 as one thread-block cluster per V-cycle;
                                                 0 = one kernel per phase    */
    int sequential_launch;                    /* 1: plain stream order between kernels;
                                                 0: programmatic dependent launch */
    int persistent_solve;                     /* CG / MG-PCG: 1 = the whole solve as one
                                                 cooperative launch (phases separated by
                                                 grid barriers); 0 = one kernel per phase */
    int tail_level;                           /* multigrid: level l >= 1 above the coarsest
                                                 whose cycle (sweeps, coarser levels,
                                                 sweeps back) is applied as one dense
                                                 operator; 0 = level by level      */
    const double* tail_operator;              /* n_l x n_l row-major, x_l = M b_l   */
    int ell_thread_budget;                    /* resident threads one coarse-level pass
                                                 may spread its rows over (lanes per row
                                                 follow from it); 0 = 8 blocks of 256 per
                                                 SM, -1 = the storage lane count   */
    int use_les;                              /* config.use_les: Smagorinsky closure, viscous
                                                 term in stress-divergence form   */
    double les_coeff;                         /* (Cs Delta)^2, Delta = sqrt(dx dy) */
    const double* metrics;                    /* stretched mesh (pycfd/core/mesh.py:122-218):
                                                 5 nx + 5 ny + 11 doubles, hx[nx], hy[ny],
                                                 hxu[nx+1], hyv[ny+1], hx_ext[nx+2],
                                                 hy_ext[ny+2], wx[nx+1], wy[ny+1],
                                                 hxu*vbar[nx+1], hyv*vbar[ny+1], vbar;
                                                 NULL on a uniform mesh (dx, dy used) */
    double outlet_width;                      /* stretched mesh: summed widths of the
                                                 outlet walls' faces (boundary.py:480-483) */
    const double* les_coeff_field;            /* stretched mesh with use_les: (Cs Delta)^2 on
                                                 the ghosted cell grid (nx+2)*(ny+2), Delta =
                                                 sqrt(dx_i dy_j), ghost ring repeating its
                                                 neighbour (physics/turbulence.py:43-58) */
} pycfd_solver_desc;

/* Per-call results the Python layer reads back (one small D2H copy). */
typedef struct {
    int iterations;          /* last solve: CG/MG-PCG iterations, sweeps or cycles */
    int converged;           /* last solve met its tolerance                  */
    int status;              /* 0 ok, PCFD_E_NOCONV / PCFD_E_STALL otherwise   */
    int total_iterations;    /* summed over the solves of the last call        */
    double last_residual;    /* ||b - A p|| / ||b|| of the last solve         */
    double fx, fy;           /* immersed-boundary reaction force (solver.py:553-599) */
    double body_fx[PCFD_MAX_BODIES], body_fy[PCFD_MAX_BODIES];
    int ir_iterations;       /* mixed form: outer refinement passes, last solve */
    int pad_;
} pycfd_stats;

/* Reductions over a state, for dt control, health and diagnostics
 * (pycfd/core/timestepper.py:94-142, :208-212, :251-266;
 *  pycfd/analysis/postprocess.py:73-79; pycfd/core/solver.py:545-550). */
typedef struct {
    double max_u, max_v;     /* max |u|, |v| over the physical faces          */
    double max_du, max_dv;   /* max |u - u_prev|, |v - v_prev| (whole arrays) */
    double max_div;          /* max |div u| over fluid cells                  */
    double kinetic_energy;   /* 0.5 sum(uc^2+vc^2) dA, solid cells zeroed     */
    double max_vorticity;    /* max |omega| averaged to cell centres          */
    int finite;              /* 1 if u, v, p hold no NaN/Inf                  */
    int pad_;
} pycfd_field_stats;

const char* pycfd_last_error(void);
int pycfd_version(void);

/* Build a solver: uploads masks, boundary tables and the multigrid hierarchy,
 * allocates the device workspace.  Replaces ProjectionSolver.__init__
 * (pycfd/core/solver.py:101-195) minus host assembly, and
 * make_pressure_solver (pycfd/core/pressure.py:645-660). */
int pycfd_solver_create(const pycfd_solver_desc* desc, pycfd_solver** out);
int pycfd_solver_destroy(pycfd_solver* s);

/* Fused momentum RHS, stateless: rhs_u (nx+1)*ny, rhs_v nx*(ny+1).
 * Replaces kernels._momentum_rhs_body (pycfd/core/kernels.py:39-110). */
int pycfd_momentum_rhs(const double* u, const double* v, int nx, int ny, double dx, double dy,
                       double nu, double blend, double fx, double fy, double* rhs_u,
                       double* rhs_v, void* stream);

/* Cell divergence, stateless: out nx*ny.  ProjectionSolver.divergence
 * (pycfd/core/solver.py:532-543). */
/* The momentum RHS with the Smagorinsky closure (ProjectionSolver.momentum_rhs
 * with config.use_les, pycfd/core/solver.py:501-529, :467-499, and
 * SmagorinskyModel.eddy_viscosity, pycfd/physics/turbulence.py:68-118), uniform
 * mesh: the effective viscosity nu + les_coeff |S| on the ghosted cell grid
 * into nu_c ((nx+2) x (ny+2)), its corner average into nu_corner
 * ((nx+1) x (ny+1)), and the right-hand side with the viscous term in
 * stress-divergence form, bit-identical to the reference's array path. */
int pycfd_momentum_rhs_les(const double* u, const double* v, int nx, int ny, double dx, double dy, double nu,
                           double les_coeff, double blend, double fx, double fy, double* nu_c, double* nu_corner,
                           double* rhs_u, double* rhs_v, void* stream);

/* The momentum RHS and the divergence on the solver's own mesh, uniform or
 * stretched (replaces ProjectionSolver.momentum_rhs, pycfd/core/solver.py:500-529,
 * and .divergence, :530-543, on the array path; laminar).  Shapes as above. */
int pycfd_solver_momentum_rhs(pycfd_solver* s, const double* u, const double* v, double blend,
                              double* rhs_u, double* rhs_v, void* stream);
int pycfd_solver_divergence(pycfd_solver* s, const double* u, const double* v, double* out, void* stream);
/* The Smagorinsky eddy viscosities (cells, corners) and the LES momentum RHS on the
 * solver's own mesh, uniform or stretched (solver.py:467-529, turbulence.py:60-118). */
int pycfd_solver_momentum_rhs_les(pycfd_solver* s, const double* u, const double* v, double blend,
                                  double* nu_c, double* nu_corner, double* rhs_u, double* rhs_v, void* stream);

int pycfd_divergence(const double* u, const double* v, int nx, int ny, double dx, double dy,
                     double* out, void* stream);

/* Boundary pass on (u, v) in place.  BoundaryManager.apply_velocity
 * (pycfd/core/boundary.py:375-379), plus enforce_global_mass_balance (:423-487)
 * when mass_balance != 0. */
int pycfd_apply_velocity_bc(pycfd_solver* s, double* u, double* v, int predictor,
                            int mass_balance, void* stream);

/* Poisson solve: rhs (nx*ny, the divergence over dt) -> p (nx*ny).  p0 is the
 * warm start or NULL.  PoissonSolverBase.solve (pycfd/core/pressure.py:325-327)
 * with CGSolver :366-398, JacobiSolver :410-454, SORSolver :457-526,
 * MultigridSolver :545-574, MultigridCGSolver :577-632. */
int pycfd_poisson_solve(pycfd_solver* s, const double* rhs, const double* p0, double* p,
                        void* stream);

/* One V-cycle from zero applied to r: the preconditioner.
 * MultigridHierarchy.apply (pycfd/core/multigrid.py:460-474). */
int pycfd_mg_apply(pycfd_solver* s, const double* r, double* z, void* stream);

/* Project (u, v) in place and write the ghosted pressure p.  Uses and updates
 * the solver's warm start.  ProjectionSolver.project (pycfd/core/solver.py:643-683). */
int pycfd_project(pycfd_solver* s, double* u, double* v, double* p, double dt, void* stream);

/* Initial state: BCs, mass balance, mask, projection with dt = 1.
 * ProjectionSolver.initialize (pycfd/core/solver.py:301-329); u, v hold the
 * initial physical faces on entry (ghosts zero) and p receives the pressure. */
int pycfd_initialize(pycfd_solver* s, double* u, double* v, double* p, void* stream);

/* One projected Euler substep: (u, v) -> (us, vs, p); inputs untouched.
 * ProjectionSolver.substep (pycfd/core/solver.py:612-640). */
int pycfd_substep(pycfd_solver* s, const double* u, const double* v, double* us, double* vs,
                  double* p, double dt, double blend, void* stream);

/* One time step with the configured scheme: (u0, v0) -> (u, v, p).
 * ProjectionSolver.step (pycfd/core/solver.py:686-731). */
int pycfd_step(pycfd_solver* s, const double* u0, const double* v0, double* u, double* v,
               double* p, double dt, double blend, void* stream);

/* The same step, recorded once per (u0, v0, u, v, p) address tuple into a
 * CUDA graph whose Poisson iteration loops are device-side conditional WHILE
 * nodes, then replayed: no host round trip inside a step.  Jacobi and SOR
 * solves (host-checked residual cadence) run eagerly instead. */
int pycfd_step_graph(pycfd_solver* s, const double* u0, const double* v0, double* u, double* v,
                     double* p, double dt, double blend, void* stream);

/* Device-side time-step control for stepping without host round trips. */
typedef struct {
    int adaptive;          /* config.adaptive_dt                                  */
    double cfl;            /* config.cfl_max                                      */
    double visc_limit;     /* 0.8 / (2 nu (1/dx^2 + 1/dy^2))                      */
    double dt_cap;         /* config.dt                                           */
    double t_end;          /* dt is clamped so the clock lands on t_end            */
    int blend_mode;        /* 0: fixed blend below; 1: 1.2 x Courant number (upwind) */
    double blend;
    double steady_tol;     /* history runs: stop once max|du|/dt < steady_tol (0: never) */
    int history;           /* 1: gated step with a device history row (see below)     */
} pycfd_dt_control;

/* One step whose dt is computed on the device from the current state, with
 * the reference's formula and order (TimeStepper.compute_dt and _check_health,
 * pycfd/core/timestepper.py:94-142), recorded once per address tuple into a
 * CUDA graph together with that reduction.  Health problems set sticky flags
 * read by pycfd_get_clock (1 non-finite, 2 |u| > 1e6, 4 dt < 1e-8). */
int pycfd_step_adaptive(pycfd_solver* s, const double* u0, const double* v0, double* u, double* v,
                        double* p, const pycfd_dt_control* ctl, void* stream);
int pycfd_set_clock(pycfd_solver* s, double t, void* stream);

/* Device-side run loop (TimeStepper.run, pycfd/core/timestepper.py:145-266).
 * With ctl->history = 1 the recorded step is gated on the device: a run whose
 * clock has reached t_end (frozen 2), that tripped a health check on the
 * unclamped dt (frozen 1: the step is not taken and the clock stays at the last
 * good step, as the reference raises DivergenceError before it), or that went
 * steady (frozen 3: max|du|/dt < steady_tol after a step, which is kept) takes
 * no further steps; every step taken appends a row to a device history: step,
 * t, dt, CFL number, max|div u|, kinetic energy, last Poisson residual, fx, fy,
 * max|du|/dt (timestepper.py:251-266).  pycfd_history_read copies the rows
 * appended since the last read (at most 4096 between reads) into rows (10
 * doubles each), gives their count and the frozen state, and clears the
 * history; pycfd_set_clock clears the clock, health, frozen state and history. */
int pycfd_history_read(pycfd_solver* s, double* rows, int max_rows, int* n_rows, int* frozen, void* stream);
int pycfd_get_clock(pycfd_solver* s, double* t, double* dt, int* steps, int* health, void* stream);

/* The same step on HOST buffers: copies the inputs in, steps (the step is
 * recorded on the first call and replayed after, as pycfd_step_graph), copies
 * u, v, p back, all on `stream`, and returns after the stream has finished.
 * Pinned host buffers make the copies asynchronous DMA. */
int pycfd_step_host(pycfd_solver* s, const double* u0_host, const double* v0_host,
                    double* u_host, double* v_host, double* p_host, double dt, double blend,
                    void* stream);

/* Measurement support (no counterpart in the reference): bracket every eager
 * launch of one kernel with CUDA events on its stream, then read the summed
 * device time.  Ids: 1 CG direction/A-product (k_cg_pq), 2 last fine smoothing
 * sweep of the V-cycle, 3 first fine sweep + residual, 4 coarse-level cluster
 * cycle, 6 momentum predictor, 7 projection correction, 8 whole persistent
 * solve (k_solve_persistent); 0 switches it off.
 * Steps replayed from a recorded graph are not bracketed. */
int pycfd_profile_kernel(pycfd_solver* s, int kernel_id);
/* CTAs of the cooperative launch that runs each CG / MG-PCG solve whole
 * (0: the solver launches one kernel per phase). */
int pycfd_solver_persistent(pycfd_solver* s, int* ctas);
/* No counterpart in the reference (failure detection of the persistent solve).
 * Limit, in nanoseconds, of one grid-barrier wait of the cooperative solve
 * (default 2 s).  A CTA that waits longer sets the launch's error word; every
 * CTA then leaves its waits, the kernel ends, and the solve reports status -6
 * (pycfd_get_stats) -- the context stays usable.  Applies to solves launched
 * after the call (a step graph recorded earlier keeps the limit it was recorded
 * with).  PCFD_E_UNSUPPORTED when the solver runs one kernel per phase. */
int pycfd_solver_set_wait_limit(pycfd_solver* s, unsigned long long ns);
/* Phase trace of the persistent solve (measurement support).  enable 1 turns
 * it on (each later solve overwrites it), 0 off, -1 leaves it as it is.  With
 * out != NULL: waits for `stream`, then copies the last solve's trace -- out[0]
 * = entries n, then n pairs (globaltimer ns when the barrier ending a phase
 * released, phase tag: low byte the phase kind, next byte the level) -- at
 * most cap words. */
int pycfd_solve_trace(pycfd_solver* s, int enable, unsigned long long* out, int cap, void* stream);
/* Kernel launches issued by this library so far (eager launches; a recorded
 * step counts its launches once, when it is recorded). */
long long pycfd_launch_count(void);
int pycfd_profile_read(pycfd_solver* s, double* total_ms, int* launches, void* stream);

/* Results of the last solve/step (synchronises `stream`). */
int pycfd_get_stats(pycfd_solver* s, pycfd_stats* out, void* stream);

/* The masked-face lists the device applies the direct forcing to
 * (ProjectionSolver._build_slices' u_face_solid / v_face_solid and the per-body
 * u_face_body / v_face_body, pycfd/core/solver.py:62-79, :280-296): linear
 * indices into u (nx+3, ny+2) and v (nx+2, ny+3), grouped by body;
 * body_*_start[b] .. body_*_start[b+1] are body b's entries (PCFD_MAX_BODIES + 1
 * slots each), *n_bodies the count (0: the total only).  Copies at most u_cap /
 * v_cap entries; *n_u / *n_v get the full counts.  The face ranges u_lo/u_hi,
 * v_lo/v_hi (solver.py:250-258) go to lohi[4]. */
int pycfd_face_lists(pycfd_solver* s, int* u_faces, int u_cap, int* v_faces, int v_cap, int* n_u,
                     int* n_v, int* body_u_start, int* body_v_start, int* n_bodies, int* lohi);

/* ---- Immersed bodies rasterised on the device (circle_mask, rectangle_mask,
 * polygon_mask, mask_from_image; pycfd/geometry/obstacles.py:87-367).  The solid
 * fraction of a cell is the mean of a subsamples x subsamples midpoint
 * supersample of the shape's inside test, sample coordinates
 * xf[i] + ((a + 0.5) / S) * dx_cells[i] (and the same in y) from the mesh's
 * face coordinates; mask = fraction > 0.5.  Bit-identical to the reference's
 * fraction and mask on the same mesh.  All arrays are device memory:
 * xf, dx_cells (nx), yf, dy_cells (ny), fraction (nx*ny doubles), mask (nx*ny
 * bytes). */
#define PCFD_SHAPE_CIRCLE 0      /* p = cx, cy, r                                     */
#define PCFD_SHAPE_RECTANGLE 1   /* p = x0, y0, x1, y1 (closed box)                    */
#define PCFD_SHAPE_POLYGON 2     /* p = bounding box x0, y0, x1, y1 of the vertices;
                                    verts: n_verts (x, y) pairs, even-odd ray test    */
#define PCFD_SHAPE_IMAGE 3       /* image: rows x cols luminance, row 0 at y = 0,
                                    stretched over [0, lx] x [0, ly]; solid where
                                    luminance < threshold (the opposite if invert)    */
typedef struct {
    int kind;
    double p[4];
    const double* verts;
    int n_verts;
    const double* image;
    int rows, cols;
    double threshold;
    int invert;
} pycfd_shape;
int pycfd_rasterize(const pycfd_shape* shape, const double* xf, const double* dx_cells, const double* yf,
                    const double* dy_cells, int nx, int ny, double lx, double ly, int subsamples,
                    double* fraction, uint8_t* mask, void* stream);

/* ---- Discrete adjoint of the cavity step (no counterpart in the reference,
 * whose step has no adjoint): the primitives of one SSP-RK3 step of the
 * lid-driven cavity with a lid profile U(x) and a smoothed obstacle chi, and
 * their exact transposes, as hand-written kernels.  The forward primitives are
 * the library step's arithmetic for the cavity (pycfd/core/solver.py:612-731,
 * kernels.py:54-110, boundary.py:141-164 with a profile on the moving lid,
 * solver.py:553-599 with u <- (1 - chi) u on the solvable faces); the Poisson
 * solves of the projection and its transpose go through pycfd_poisson_solve.
 * Arrays are device pointers in the ghosted layout (u (n+3) x (n+2), v
 * (n+2) x (n+3)); cell arrays are n x n. */
#define PCFD_ADJ_PREDICTOR 1    /* out_u, out_v = u, v + dt rhs(u, v) on solvable faces      */
#define PCFD_ADJ_WALLS 2        /* out_u, out_v (in place): cavity walls, lid[n+3] on top     */
#define PCFD_ADJ_MASK 3         /* out_u, out_v = (1 - cu, cv) (u, v) on solvable faces       */
#define PCFD_ADJ_DIV 4          /* out[n*n] = div(u, v) / dt                                  */
#define PCFD_ADJ_CORRECT 5      /* out_u, out_v (in place) -= dt grad(a), a = p (n*n)         */
#define PCFD_ADJ_LINCOMB 6      /* out[count] = ca a + cb b                                   */
#define PCFD_ADJ_OBJECTIVE 7    /* out[0] = h^2 sum 0.5 (uc^2 + vc^2) lower[j]                */
#define PCFD_ADJ_PREDICTOR_T 8  /* out_u, out_v = predictor^T at (u, v) applied to (gu, gv)   */
#define PCFD_ADJ_WALLS_T 9      /* out_u, out_v (in place) = walls^T; acc_u[n+3] += d/dlid   */
#define PCFD_ADJ_MASK_T 10      /* out_u, out_v (in place) = mask^T at input (u, v); acc_u,
                                   acc_v += d/dchi                                         */
#define PCFD_ADJ_GRAD_T 11      /* out[n*n] = G^T (gu, gv) (transposed face gradient)         */
#define PCFD_ADJ_DIV_T 12       /* out_u, out_v (in place) -= D^T a (a = psi, n*n)            */
#define PCFD_ADJ_OBJECTIVE_T 13 /* out_u, out_v = d objective / d(u, v) at (u, v)             */
typedef struct {
    int n;                       /* cells per side                                   */
    double h, nu, dt;            /* spacing, viscosity, time step                    */
    double ca, cb;               /* lincomb weights                                  */
    long count;                  /* lincomb length                                   */
    const double *u, *v;         /* state the primitive (or its transpose) is taken at */
    const double *gu, *gv;       /* incoming gradients (predictor_T, grad_T)         */
    const double *a, *b;         /* extra operands (lincomb, correct/div_T field)   */
    const double *lid, *cu, *cv, *lower;
    double *out_u, *out_v, *out, *acc_u, *acc_v;
} pycfd_adj_args;
int pycfd_adjoint_apply(int op, const pycfd_adj_args* args, void* stream);

/* Field reductions (synchronises `stream`).  u_prev/v_prev may be NULL. */
int pycfd_reduce_fields(pycfd_solver* s, const double* u, const double* v, const double* p,
                      const double* u_prev, const double* v_prev, pycfd_field_stats* out,
                      void* stream);

/* ---- Batched stepping (no counterpart in the reference, whose Simulation
 * advances one problem).  Many independent problems -- grids of uneven size,
 * their own viscosity, boundary conditions, time step and end time -- advance
 * together, every stage of the SSP-RK3 step ONE launch over all of them
 * (block maps of (problem, tile)), the Poisson solves as MG-PCG (FP64) or as
 * FP32 MG-PCG inside FP64 iterative refinement (mixed), with device-side loops
 * that run while any problem still iterates.  Each problem keeps the
 * single-problem arithmetic: ProjectionSolver.step (pycfd/core/solver.py:686-731)
 * with TimeStepper.compute_dt (pycfd/core/timestepper.py:94-142). */
typedef struct pycfd_batch pycfd_batch;

typedef struct {
    int precision;      /* PCFD_FP64 or PCFD_MIXED                                */
    double tol;         /* relative Poisson tolerance (outer one, mixed form)     */
    int maxiter;        /* CG iterations per solve (FP64 form)                    */
    double inner_tol;   /* mixed: relative tolerance of each FP32 inner solve     */
    int mg_sweeps;      /* damped-Jacobi sweeps before and after each coarse step */
    int tile_rows;      /* rows of x per fine-level block: 8, 16, 32 or 64        */
    int coarse_level;   /* multigrid levels from this one down run in one thread
                           block per problem (one launch per V-cycle); 0: one
                           launch per phase on every level                      */
    int fused_from;     /* with fused restrictions in the hierarchies: the first
                           level restricted by R (I - A W) (1: from the fine level;
                           2: the fine sweep and restriction stay separate); 0
                           reads as 1                                           */
    int ell_group;      /* problems of one structure per block of a coarse-level
                           launch, sharing each matrix entry's load: 1 or 8 (0
                           reads as 8)                                          */
    int programmatic_launch;  /* 1: programmatic dependent launch between the batched
                                 kernels; 0: plain stream order (measured faster on
                                 the 256-cavity batch: 19.45 against 19.90 ms/step) */
    int stencil_transfer;     /* 1: with the fused down sweep from the fine level,
                                 the transfers between levels 0 and 1 run as stencils
                                 over the fine cells (the fused restriction, and the
                                 prolongation together with the last fine sweep)
                                 instead of products with the stored P_1 and M_1.
                                 They stand for P_1 = (I - W_0 A_0) T and
                                 M_1 = P_1^T (I - A_0 W_0), T the aggregation of 2 x 2
                                 fine cells: every structure's level 1 must have the
                                 shape (ceil(nx/2), ceil(ny/2)) (else PCFD_E_UNSUPPORTED)
                                 and its P_1 must be that smoothed aggregation (the
                                 hierarchy this library's host side builds).  Equal to
                                 the matrix products to rounding.  0: the products. */
    int scalar_strips;        /* 1: the mixed form's FP32 CG and level-0 sweep kernels
                                 walk every problem in 30-column scalar strips; 0:
                                 problems whose ny is a multiple of 4 walk 128-column
                                 vector strips (four cells per lane, 16-byte loads),
                                 the same per-cell arithmetic, the per-problem sums
                                 added in another order.  The FP64 form always
                                 walks scalar strips.                              */
} pycfd_batch_opts;

/* n problems: descs[i] describes problem i (time_scheme PCFD_RK3; solver
 * fields other than the hierarchy are taken from opts).  structure[i] names
 * the problem whose multigrid hierarchy problem i shares (i itself, or an
 * earlier problem with the same grid, boundary kinds and mask); only those
 * leading problems need levels/coarsest_inverse, of at least 2 levels.  The
 * state u[i], v[i], p[i] (device, the ghosted layout of pycfd_step) is advanced
 * in place; dt_ctl[i] is problem i's time-step control; its clock starts at 0;
 * it stops after max_steps[i] steps (max_steps may be NULL: no limit). */
int pycfd_batch_create(const pycfd_solver_desc* descs, const int* structure,
                       const pycfd_dt_control* dt_ctl, const int* max_steps, double* const* u,
                       double* const* v, double* const* p, int n, const pycfd_batch_opts* opts,
                       pycfd_batch** out);
int pycfd_batch_destroy(pycfd_batch* b);
/* Initial projection of every problem (pycfd_initialize, batched). */
int pycfd_batch_initialize(pycfd_batch* b, void* stream);
/* `steps` adaptive steps of every problem; record != 0 replays one recorded
 * CUDA graph per step (recorded on first use).  A problem whose health flags
 * trip (pycfd_get_clock), whose clock reaches t_end or that has taken its
 * max_steps stops; the others go on. */
int pycfd_batch_step(pycfd_batch* b, int steps, int record, void* stream);
/* Problem i's single-problem handle (clock, stats, reductions; not for stepping). */
pycfd_solver* pycfd_batch_problem(pycfd_batch* b, int i);
/* Per-problem arrays of n: frozen (0 running, 1 stopped by a health flag,
 * 2 reached t_end or max_steps), steps taken, solver iterations of the last step, solver
 * status, clock and last dt.  Any pointer may be NULL. */
int pycfd_batch_status(pycfd_batch* b, int* frozen, int* steps, int* iterations, int* status,
                       double* t, double* dt, void* stream);
/* Measurement support: bracket every eager launch (record = 0) of one kernel
 * kind with CUDA events, then read the summed device time.  Ids: 1 CG
 * direction/A-product, 2 last fine V-cycle sweep (with stencil transfers: and
 * the prolongation onto the fine level), 3 first fine sweep + residual (with
 * stencil transfers: the fused restriction into level 1), 4 coarse levels, 5 CG
 * update, 6 predictor; 0 off. */
int pycfd_batch_profile(pycfd_batch* b, int kernel_id);
int pycfd_batch_profile_read(pycfd_batch* b, double* total_ms, int* launches, void* stream);
/* Kernel launches the device executed for `steps` recorded steps since the
 * last call (fixed part per step plus the loop bodies times the passes run). */
int pycfd_batch_launches(pycfd_batch* b, int steps, long long* launches, void* stream);
/* No counterpart in the reference (failure detection of the device loops).
 * Every device-side WHILE loop of a batched solve ends after a pass cap, above
 * the problems' own iteration limits, so the loop always ends.  cap > 0 sets
 * that cap for the CG and refinement loops of later steps (recorded or eager;
 * the device reads it at every pass), 0 restores the built-in caps.  A solve
 * cut short leaves its problems unconverged: status PCFD_E_NOCONV in
 * pycfd_batch_status when the residual is above the solver's bound, and the
 * step goes on.  pycfd_batch_capped reports (and clears) which loops a cap
 * ended since the last call: bit 0 the CG loop, bit 1 the refinement loop. */
int pycfd_batch_set_loop_cap(pycfd_batch* b, int cap, void* stream);
int pycfd_batch_capped(pycfd_batch* b, int* capped, void* stream);

/* No counterpart in the reference.  The reductions of pycfd_reduce_fields for
 * callers that cannot allocate device memory at the moment they need them: a
 * host whose own allocator owns all device memory (cudaMalloc would fail or
 * steal from its pool), or a loop that cannot afford the device-wide
 * synchronisation a cudaMalloc/cudaFree pair may impose.  It needs no solver
 * handle and calls no allocator.  Its scratch is a static device array of
 * PCFD_NOALLOC_MAX_ROWS*8 + 66 doubles (about 258 KiB) that every GPU which
 * loads the library holds until the process exits; one thread block runs per
 * row of u, so nx may be at most PCFD_NOALLOC_MAX_ROWS - 3 (larger grids are
 * refused with PCFD_E_ARG).  Every call on a device shares that scratch and it
 * keeps the last call's contents (the call clears its ticket counter itself):
 * calls whose work overlaps on the GPU (for instance on two streams) race, so
 * serialise them.  The first call on a device looks up the scratch's device
 * address with that device current and keeps it for the life of the process;
 * after a cudaDeviceReset that address is stale, so do not call this entry
 * point again in that process.  The call waits for its stream to finish the
 * reduction before it returns.  u, v, p, u_prev, v_prev and solid (nx*ny
 * bytes, or NULL) are device pointers. */
#define PCFD_NOALLOC_MAX_ROWS 4096
int pycfd_reduce_fields_noalloc(const double* u, const double* v, const double* p,
                                const double* u_prev, const double* v_prev, const uint8_t* solid,
                                int nx, int ny, double dx, double dy, pycfd_field_stats* out,
                                void* stream);

#ifdef __cplusplus
}
#endif
#endif
