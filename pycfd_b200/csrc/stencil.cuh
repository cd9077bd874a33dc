// MAC-grid stencils: momentum predictor, divergence, projection correction,
// Runge-Kutta stage combination, field statistics.
//
// Arithmetic follows the reference expression by expression (every product
// that feeds a sum is formed with rmul, so no multiply-add is fused), so the
// predictor, the divergence and the correction are bit-identical to the
// reference's NumPy/Numba path on the same inputs.
#pragma once
#include "common.cuh"

namespace pcfd {

constexpr int TJ = 32;   // threads along y (contiguous)
constexpr int TI = 8;    // threads along x

// A stage field read either directly or as the Runge-Kutta combination
// ca*a + cb*b formed on the fly (pycfd/core/solver.py:716-717).
struct StageIn {
  const double* a;
  const double* b;   // nullptr: plain read of a
  double ca, cb;
  __device__ __forceinline__ double operator[](long k) const {
    return b ? rmul(ca, a[k]) + rmul(cb, b[k]) : a[k];
  }
};

// u-momentum RHS at a u face from the values it reads (pycfd/core/kernels.py:54-80):
// the face's own value, its east/west/north/south neighbours, and the four v faces
// around it (v_tl = v[m-1, j+1], v_tr = v[m, j+1], v_bl = v[m-1, j], v_br = v[m, j]).
__device__ __forceinline__ double rhs_u_core(double u0, double ue, double uw, double un, double us, double v_tl,
                                             double v_tr, double v_bl, double v_br, double dx, double dy,
                                             double nu, double blend, double fx) {
  const double u_right = 0.5 * (u0 + ue);
  const double u_left = 0.5 * (uw + u0);
  double duudx = (rmul(u_right, u_right) - rmul(u_left, u_left)) / dx;
  const double u_top = 0.5 * (u0 + un);
  const double v_top = 0.5 * (v_tl + v_tr);
  const double u_bot = 0.5 * (us + u0);
  const double v_bot = 0.5 * (v_bl + v_br);
  double duvdy = (rmul(u_top, v_top) - rmul(u_bot, v_bot)) / dy;
  if (blend > 0.0) {
    duudx += rmul(blend / dx, rmul(fabs(u_right), u0 - ue) * 0.5 - rmul(fabs(u_left), uw - u0) * 0.5);
    duvdy += rmul(blend / dy, rmul(fabs(v_top), u0 - un) * 0.5 - rmul(fabs(v_bot), us - u0) * 0.5);
  }
  const double lap = ((uw - 2.0 * u0 + ue) / (dx * dx) + (us - 2.0 * u0 + un) / (dy * dy));
  return -(duudx + duvdy) + rmul(nu, lap) + fx;
}

// v-momentum RHS at a v face from its values (pycfd/core/kernels.py:83-110): the
// face, its north/south/east/west neighbours, and the four u faces around it
// (u_rb = u[i+1, n-1], u_rt = u[i+1, n], u_lb = u[i, n-1], u_lt = u[i, n]).
__device__ __forceinline__ double rhs_v_core(double v0, double vn, double vs, double ve, double vw, double u_rb,
                                             double u_rt, double u_lb, double u_lt, double dx, double dy,
                                             double nu, double blend, double fy) {
  const double v_top = 0.5 * (v0 + vn);
  const double v_bot = 0.5 * (vs + v0);
  double dvvdy = (rmul(v_top, v_top) - rmul(v_bot, v_bot)) / dy;
  const double u_right = 0.5 * (u_rb + u_rt);
  const double v_right = 0.5 * (v0 + ve);
  const double u_left = 0.5 * (u_lb + u_lt);
  const double v_left = 0.5 * (vw + v0);
  double duvdx = (rmul(u_right, v_right) - rmul(u_left, v_left)) / dx;
  if (blend > 0.0) {
    dvvdy += rmul(blend / dy, rmul(fabs(v_top), v0 - vn) * 0.5 - rmul(fabs(v_bot), vs - v0) * 0.5);
    duvdx += rmul(blend / dx, rmul(fabs(u_right), v0 - ve) * 0.5 - rmul(fabs(u_left), vw - v0) * 0.5);
  }
  const double lap = ((vw - 2.0 * v0 + ve) / (dx * dx) + (vs - 2.0 * v0 + vn) / (dy * dy));
  return -(duvdx + dvvdy) + rmul(nu, lap) + fy;
}

// u-momentum RHS at u-face (m, j), 1<=m<=nx+1, 1<=j<=ny.
template <class U, class V>
__device__ __forceinline__ double rhs_u_at(const U& u, const V& v, int m, int j, int ny,
                                           double dx, double dy, double nu, double blend,
                                           double fx) {
  const long W = ny + 2, WV = ny + 3;
  return rhs_u_core(u[m * W + j], u[(m + 1) * W + j], u[(m - 1) * W + j], u[m * W + j + 1], u[m * W + j - 1],
                    v[(m - 1) * WV + j + 1], v[m * WV + j + 1], v[(m - 1) * WV + j], v[m * WV + j], dx, dy, nu,
                    blend, fx);
}

// v-momentum RHS at v-face (i, n), 1<=i<=nx, 1<=n<=ny+1.
template <class U, class V>
__device__ __forceinline__ double rhs_v_at(const U& u, const V& v, int i, int n, int ny,
                                           double dx, double dy, double nu, double blend,
                                           double fy) {
  const long W = ny + 2, WV = ny + 3;
  return rhs_v_core(v[i * WV + n], v[i * WV + n + 1], v[i * WV + n - 1], v[(i + 1) * WV + n], v[(i - 1) * WV + n],
                    u[(i + 1) * W + n - 1], u[(i + 1) * W + n], u[i * W + n - 1], u[i * W + n], dx, dy, nu,
                    blend, fy);
}

// ---- stretched mesh (pycfd/core/solver.py:336-466, the array path) ------------
// Advection in conservative form with corner interpolants weighted by the
// geometry (u along y with wy, v along x with wx), the donor-cell correction over
// the same control volumes, and diffusion as a difference of two first
// derivatives (inner gradients across the flanking cells, outer difference
// across the face's own control volume).  Same operations, same order as the
// reference's arrays, so the right-hand side is bit-identical to it.
// Advective term A_u at u face (m, j) of a stretched mesh (duudx + duvdy, the donor-cell
// correction included).
template <class U, class V>
__device__ __forceinline__ double adv_u_str(const U& u, const V& v, int m, int j, int ny, const Metrics& M,
                                            double blend) {
  const long W = ny + 2, WV = ny + 3;
  const double u0 = u[m * W + j], ue = u[(m + 1) * W + j], uw = u[(m - 1) * W + j];
  const double un = u[m * W + j + 1], us = u[m * W + j - 1];
  const double wxa = M.wx(m - 1);
  // corner interpolants of u (along y) and v (along x) above and below the face
  const double uc_t = u0 + rmul(M.wy(j), un - u0);
  const double uc_b = us + rmul(M.wy(j - 1), u0 - us);
  const double vt0 = v[(m - 1) * WV + j + 1], vb0 = v[(m - 1) * WV + j];
  const double vc_t = vt0 + rmul(wxa, v[m * WV + j + 1] - vt0);
  const double vc_b = vb0 + rmul(wxa, v[m * WV + j] - vb0);
  const double uu_r = 0.5 * (u0 + ue), uu_l = 0.5 * (uw + u0);
  const double hxu = M.hxu(m - 1), hy = M.hy(j - 1);
  double duudx = (rmul(uu_r, uu_r) - rmul(uu_l, uu_l)) / hxu;
  double duvdy = (rmul(uc_t, vc_t) - rmul(uc_b, vc_b)) / hy;
  if (blend > 0.0) {
    duudx += rmul(blend / hxu, rmul(fabs(uu_r), u0 - ue) / 2.0 - rmul(fabs(uu_l), uw - u0) / 2.0);
    duvdy += rmul(blend / hy, rmul(fabs(vc_t), u0 - un) / 2.0 - rmul(fabs(vc_b), us - u0) / 2.0);
  }
  return duudx + duvdy;
}

template <class U, class V>
__device__ __forceinline__ double rhs_u_str(const U& u, const V& v, int m, int j, int ny, const Metrics& M,
                                            double nu, double blend, double fx) {
  const long W = ny + 2;
  const double u0 = u[m * W + j], ue = u[(m + 1) * W + j], uw = u[(m - 1) * W + j];
  const double un = u[m * W + j + 1], us = u[m * W + j - 1];
  const double adv = adv_u_str(u, v, m, j, ny, M, blend);
  const double gx_hi = (ue - u0) / M.hx_ext(m), gx_lo = (u0 - uw) / M.hx_ext(m - 1);
  const double gy_hi = (un - u0) / M.hyv(j), gy_lo = (u0 - us) / M.hyv(j - 1);
  const double d2u = (gx_hi - gx_lo) / M.hxu(m - 1) + (gy_hi - gy_lo) / M.hy(j - 1);
  return -adv + rmul(nu, d2u) + fx;
}

// Advective term A_v at v face (i, n) of a stretched mesh (duvdx + dvvdy).
template <class U, class V>
__device__ __forceinline__ double adv_v_str(const U& u, const V& v, int i, int n, int ny, const Metrics& M,
                                            double blend) {
  const long W = ny + 2, WV = ny + 3;
  const double v0 = v[i * WV + n], vn = v[i * WV + n + 1], vs = v[i * WV + n - 1];
  const double ve = v[(i + 1) * WV + n], vw = v[(i - 1) * WV + n];
  const double wyb = M.wy(n - 1);
  // corner interpolants at the right (i, n-1) and left (i-1, n-1) corners of the face
  const double ur0 = u[(i + 1) * W + n - 1], ul0 = u[i * W + n - 1];
  const double uc_r = ur0 + rmul(wyb, u[(i + 1) * W + n] - ur0);
  const double uc_l = ul0 + rmul(wyb, u[i * W + n] - ul0);
  const double vc_r = v0 + rmul(M.wx(i), ve - v0);
  const double vc_l = vw + rmul(M.wx(i - 1), v0 - vw);
  const double vv_t = 0.5 * (v0 + vn), vv_b = 0.5 * (vs + v0);
  const double hyv = M.hyv(n - 1), hx = M.hx(i - 1);
  double dvvdy = (rmul(vv_t, vv_t) - rmul(vv_b, vv_b)) / hyv;
  double duvdx = (rmul(uc_r, vc_r) - rmul(uc_l, vc_l)) / hx;
  if (blend > 0.0) {
    dvvdy += rmul(blend / hyv, rmul(fabs(vv_t), v0 - vn) / 2.0 - rmul(fabs(vv_b), vs - v0) / 2.0);
    duvdx += rmul(blend / hx, rmul(fabs(uc_r), v0 - ve) / 2.0 - rmul(fabs(uc_l), vw - v0) / 2.0);
  }
  return duvdx + dvvdy;
}

template <class U, class V>
__device__ __forceinline__ double rhs_v_str(const U& u, const V& v, int i, int n, int ny, const Metrics& M,
                                            double nu, double blend, double fy) {
  const long WV = ny + 3;
  const double v0 = v[i * WV + n], vn = v[i * WV + n + 1], vs = v[i * WV + n - 1];
  const double ve = v[(i + 1) * WV + n], vw = v[(i - 1) * WV + n];
  const double adv = adv_v_str(u, v, i, n, ny, M, blend);
  const double hx_hi = (ve - v0) / M.hxu(i), hx_lo = (v0 - vw) / M.hxu(i - 1);
  const double hy_hi = (vn - v0) / M.hy_ext(n), hy_lo = (v0 - vs) / M.hy_ext(n - 1);
  const double d2v = (hx_hi - hx_lo) / M.hx(i - 1) + (hy_hi - hy_lo) / M.hyv(n - 1);
  return -adv + rmul(nu, d2v) + fy;
}

// ---- Smagorinsky large-eddy closure (pycfd/physics/turbulence.py:25-118) -------
// Effective viscosity nu + (Cs Delta)^2 |S| on the ghosted cell grid (nx+2, ny+2)
// and its corner average on (nx+1, ny+1), then the viscous term in
// stress-divergence form (pycfd/core/solver.py:467-499), uniform mesh.  The
// expressions follow the reference's array code term by term, so the
// viscosities and the right-hand side are bit-identical to it.
// Spacings of a uniform mesh behind the same accessors as Metrics, so one
// template serves both: every accessor returns dx or dy.
struct UniSp {
  double dx, dy;
  __device__ __forceinline__ double hx(int) const { return dx; }
  __device__ __forceinline__ double hy(int) const { return dy; }
  __device__ __forceinline__ double hxu(int) const { return dx; }
  __device__ __forceinline__ double hyv(int) const { return dy; }
  __device__ __forceinline__ double hx_ext(int) const { return dx; }
  __device__ __forceinline__ double hy_ext(int) const { return dy; }
};

// S_12 at corner (i, j): both derivatives cross a face, so both divide by a
// centre-to-centre distance (pycfd/physics/turbulence.py:62-65).
template <class U, class V, class Sp>
__device__ __forceinline__ double les_s12_corner(const U& u, const V& v, int i, int j, int ny, const Sp& sp) {
  const long W = ny + 2, WV = ny + 3;
  const double dudy = (u[(long)(i + 1) * W + j + 1] - u[(long)(i + 1) * W + j]) / sp.hyv(j);
  const double dvdx = (v[(long)(i + 1) * WV + j + 1] - v[(long)i * WV + j + 1]) / sp.hxu(i);
  return 0.5 * (dudy + dvdx);
}

// nu_c at every ghosted cell: |S| = sqrt(2 s11^2 + 2 s22^2 + 4 s12^2), s11 and s22
// across the cell (the ghost-extended widths), s12 the mean of the cell's four
// corner shear rates (ghost cells take the nearest interior cell's mean, as the
// reference extends it).  The coefficient (Cs Delta)^2 is one number on a uniform
// mesh, a ghosted per-cell array on a stretched one (coeff_c, formed on the host
// with the reference's operations, pycfd/physics/turbulence.py:43-58).
template <class Sp>
__global__ void k_les_nu(StageIn u, StageIn v, Geo g, Sp sp, double coeff, const double* __restrict__ coeff_c,
                         double* __restrict__ nu_c) {
  pdl_begin();
  const int nx = g.nx, ny = g.ny;
  const long W = ny + 2, WV = ny + 3;
  const long total = (long)(nx + 2) * (ny + 2);
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const int i = (int)(e / (ny + 2)), j = (int)(e % (ny + 2));
    const double s11 = (u[(long)(i + 1) * W + j] - u[(long)i * W + j]) / sp.hx_ext(i);
    const double s22 = (v[(long)i * WV + j + 1] - v[(long)i * WV + j]) / sp.hy_ext(j);
    const int ic = i < 1 ? 1 : (i > nx ? nx : i), jc = j < 1 ? 1 : (j > ny ? ny : j);
    const double s12 = 0.25 * (les_s12_corner(u, v, ic - 1, jc - 1, ny, sp) +
                               les_s12_corner(u, v, ic, jc - 1, ny, sp) +
                               les_s12_corner(u, v, ic - 1, jc, ny, sp) +
                               les_s12_corner(u, v, ic, jc, ny, sp));
    const double smag = sqrt(2.0 * rmul(s11, s11) + 2.0 * rmul(s22, s22) + 4.0 * rmul(s12, s12));
    nu_c[e] = g.nu + rmul(coeff_c ? coeff_c[e] : coeff, smag);
  }
}

__global__ void k_les_corner(const double* __restrict__ nu_c, Geo g, double* __restrict__ nu_k) {
  pdl_begin();
  const int nx = g.nx, ny = g.ny;
  const long W = ny + 2;
  const long total = (long)(nx + 1) * (ny + 1);
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const int i = (int)(e / (ny + 1)), j = (int)(e % (ny + 1));
    nu_k[e] = 0.25 * (nu_c[(long)i * W + j] + nu_c[(long)(i + 1) * W + j] + nu_c[(long)i * W + j + 1] +
                      nu_c[(long)(i + 1) * W + j + 1]);
  }
}

// Advection as rhs_u_at, diffusion in stress-divergence form with the cell
// viscosities nu_c (nx+2, ny+2) and corner viscosities nu_k (nx+1, ny+1).
template <class U, class V>
__device__ __forceinline__ double rhs_u_les_at(const U& u, const V& v, int m, int j, int ny, double dx, double dy,
                                               double blend, double fx, const double* nu_c,
                                               const double* nu_k) {
  const long W = ny + 2, WV = ny + 3, WK = ny + 1;
  const double u0 = u[m * W + j];
  const double ue = u[(m + 1) * W + j], uw = u[(m - 1) * W + j];
  const double un = u[m * W + j + 1], us = u[m * W + j - 1];
  const double u_right = 0.5 * (u0 + ue);
  const double u_left = 0.5 * (uw + u0);
  double duudx = (rmul(u_right, u_right) - rmul(u_left, u_left)) / dx;
  const double u_top = 0.5 * (u0 + un);
  const double v_top = 0.5 * (v[(m - 1) * WV + j + 1] + v[m * WV + j + 1]);
  const double u_bot = 0.5 * (us + u0);
  const double v_bot = 0.5 * (v[(m - 1) * WV + j] + v[m * WV + j]);
  double duvdy = (rmul(u_top, v_top) - rmul(u_bot, v_bot)) / dy;
  if (blend > 0.0) {
    duudx += rmul(blend / dx, rmul(fabs(u_right), u0 - ue) * 0.5 - rmul(fabs(u_left), uw - u0) * 0.5);
    duvdy += rmul(blend / dy, rmul(fabs(v_top), u0 - un) * 0.5 - rmul(fabs(v_bot), us - u0) * 0.5);
  }
  const double dudx_r = (ue - u0) / dx, dudx_l = (u0 - uw) / dx;
  const double tau_t = rmul(nu_k[(long)(m - 1) * WK + j],
                            (un - u0) / dy + (v[(long)m * WV + j + 1] - v[(long)(m - 1) * WV + j + 1]) / dx);
  const double tau_b = rmul(nu_k[(long)(m - 1) * WK + j - 1],
                            (u0 - us) / dy + (v[(long)m * WV + j] - v[(long)(m - 1) * WV + j]) / dx);
  const double d = 2.0 * (rmul(nu_c[(long)m * W + j], dudx_r) - rmul(nu_c[(long)(m - 1) * W + j], dudx_l)) / dx +
                   (tau_t - tau_b) / dy;
  return -(duudx + duvdy) + d + fx;
}

template <class U, class V>
__device__ __forceinline__ double rhs_v_les_at(const U& u, const V& v, int i, int n, int ny, double dx, double dy,
                                               double blend, double fy, const double* nu_c,
                                               const double* nu_k) {
  const long W = ny + 2, WV = ny + 3, WK = ny + 1;
  const double v0 = v[i * WV + n];
  const double vn = v[i * WV + n + 1], vs = v[i * WV + n - 1];
  const double ve = v[(i + 1) * WV + n], vw = v[(i - 1) * WV + n];
  const double v_top = 0.5 * (v0 + vn);
  const double v_bot = 0.5 * (vs + v0);
  double dvvdy = (rmul(v_top, v_top) - rmul(v_bot, v_bot)) / dy;
  const double u_right = 0.5 * (u[(i + 1) * W + n - 1] + u[(i + 1) * W + n]);
  const double v_right = 0.5 * (v0 + ve);
  const double u_left = 0.5 * (u[i * W + n - 1] + u[i * W + n]);
  const double v_left = 0.5 * (vw + v0);
  double duvdx = (rmul(u_right, v_right) - rmul(u_left, v_left)) / dx;
  if (blend > 0.0) {
    dvvdy += rmul(blend / dy, rmul(fabs(v_top), v0 - vn) * 0.5 - rmul(fabs(v_bot), vs - v0) * 0.5);
    duvdx += rmul(blend / dx, rmul(fabs(u_right), v0 - ve) * 0.5 - rmul(fabs(u_left), vw - v0) * 0.5);
  }
  // corners (i, n-1) and (i-1, n-1) of the v face
  const double tau_r = rmul(nu_k[(long)i * WK + n - 1],
                            (u[(long)(i + 1) * W + n] - u[(long)(i + 1) * W + n - 1]) / dy + (ve - v0) / dx);
  const double tau_l = rmul(nu_k[(long)(i - 1) * WK + n - 1],
                            (u[(long)i * W + n] - u[(long)i * W + n - 1]) / dy + (v0 - vw) / dx);
  const double dvdy_t = (vn - v0) / dy, dvdy_b = (v0 - vs) / dy;
  const double d = (tau_r - tau_l) / dx +
                   2.0 * (rmul(nu_c[(long)i * W + n], dvdy_t) - rmul(nu_c[(long)i * W + n - 1], dvdy_b)) / dy;
  return -(duvdx + dvvdy) + d + fy;
}

// The LES viscous term on a stretched mesh (pycfd/core/solver.py:467-499 with the
// metric arrays) after the stretched advection.
template <class U, class V>
__device__ __forceinline__ double rhs_u_les_str(const U& u, const V& v, int m, int j, int ny, const Metrics& M,
                                                double blend, double fx, const double* nu_c, const double* nu_k) {
  const long W = ny + 2, WV = ny + 3, WK = ny + 1;
  const double u0 = u[m * W + j], ue = u[(m + 1) * W + j], uw = u[(m - 1) * W + j];
  const double un = u[m * W + j + 1], us = u[m * W + j - 1];
  const double adv = adv_u_str(u, v, m, j, ny, M, blend);
  const double hxu = M.hxu(m - 1);
  const double dudx_r = (ue - u0) / M.hx_ext(m), dudx_l = (u0 - uw) / M.hx_ext(m - 1);
  const double tau_t = rmul(nu_k[(long)(m - 1) * WK + j],
                            (un - u0) / M.hyv(j) + (v[(long)m * WV + j + 1] - v[(long)(m - 1) * WV + j + 1]) / hxu);
  const double tau_b = rmul(nu_k[(long)(m - 1) * WK + j - 1],
                            (u0 - us) / M.hyv(j - 1) + (v[(long)m * WV + j] - v[(long)(m - 1) * WV + j]) / hxu);
  const double d = 2.0 * (rmul(nu_c[(long)m * W + j], dudx_r) - rmul(nu_c[(long)(m - 1) * W + j], dudx_l)) / hxu +
                   (tau_t - tau_b) / M.hy(j - 1);
  return -adv + d + fx;
}

template <class U, class V>
__device__ __forceinline__ double rhs_v_les_str(const U& u, const V& v, int i, int n, int ny, const Metrics& M,
                                                double blend, double fy, const double* nu_c, const double* nu_k) {
  const long W = ny + 2, WV = ny + 3, WK = ny + 1;
  const double v0 = v[i * WV + n], vn = v[i * WV + n + 1], vs = v[i * WV + n - 1];
  const double ve = v[(i + 1) * WV + n], vw = v[(i - 1) * WV + n];
  const double adv = adv_v_str(u, v, i, n, ny, M, blend);
  const double hyv = M.hyv(n - 1);
  const double tau_r = rmul(nu_k[(long)i * WK + n - 1],
                            (u[(long)(i + 1) * W + n] - u[(long)(i + 1) * W + n - 1]) / hyv + (ve - v0) / M.hxu(i));
  const double tau_l = rmul(nu_k[(long)(i - 1) * WK + n - 1],
                            (u[(long)i * W + n] - u[(long)i * W + n - 1]) / hyv + (v0 - vw) / M.hxu(i - 1));
  const double dvdy_t = (vn - v0) / M.hy_ext(n), dvdy_b = (v0 - vs) / M.hy_ext(n - 1);
  const double d = (tau_r - tau_l) / M.hx(i - 1) +
                   2.0 * (rmul(nu_c[(long)i * W + n], dvdy_t) - rmul(nu_c[(long)i * W + n - 1], dvdy_b)) / hyv;
  return -adv + d + fy;
}

// LES RHS of the solver's own mesh (uniform or stretched).
__global__ void k_rhs_les_g(const double* __restrict__ u, const double* __restrict__ v, Geo g, double blend,
                            const double* __restrict__ nu_c, const double* __restrict__ nu_k,
                            double* __restrict__ rhs_u, double* __restrict__ rhs_v) {
  pdl_begin();
  const int nx = g.nx, ny = g.ny;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y * blockDim.y + threadIdx.y;
  if (i <= nx && j < ny)
    rhs_u[(long)i * ny + j] = g.met ? rhs_u_les_str(u, v, i + 1, j + 1, ny, Metrics(g), blend, g.fx, nu_c, nu_k)
                                    : rhs_u_les_at(u, v, i + 1, j + 1, ny, g.dx, g.dy, blend, g.fx, nu_c, nu_k);
  if (i < nx && j <= ny)
    rhs_v[(long)i * (ny + 1) + j] =
        g.met ? rhs_v_les_str(u, v, i + 1, j + 1, ny, Metrics(g), blend, g.fy, nu_c, nu_k)
              : rhs_v_les_at(u, v, i + 1, j + 1, ny, g.dx, g.dy, blend, g.fy, nu_c, nu_k);
}

// Stateless LES RHS into (nx+1, ny) and (nx, ny+1) blocks.
__global__ void k_rhs_les(const double* __restrict__ u, const double* __restrict__ v, int nx, int ny, double dx,
                          double dy, double blend, double fx, double fy, const double* __restrict__ nu_c,
                          const double* __restrict__ nu_k, double* __restrict__ rhs_u,
                          double* __restrict__ rhs_v) {
  pdl_begin();
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y * blockDim.y + threadIdx.y;
  if (i <= nx && j < ny)
    rhs_u[(long)i * ny + j] = rhs_u_les_at(u, v, i + 1, j + 1, ny, dx, dy, blend, fx, nu_c, nu_k);
  if (i < nx && j <= ny)
    rhs_v[(long)i * (ny + 1) + j] = rhs_v_les_at(u, v, i + 1, j + 1, ny, dx, dy, blend, fy, nu_c, nu_k);
}

// Predictor with the LES right-hand side (the stage input's viscosities precomputed).
__global__ void k_predictor_les(StageIn u, StageIn v, double* __restrict__ us, double* __restrict__ vs, Geo g,
                                const double* __restrict__ S, const double* __restrict__ nu_c,
                                const double* __restrict__ nu_k) {
  pdl_begin();
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y * blockDim.y + threadIdx.y;
  const int nx = g.nx, ny = g.ny;
  const double dt = S[S_DT], blend = S[S_BLEND];
  if (i < nx + 3 && j < ny + 2) {
    const long k = (long)i * (ny + 2) + j;
    double val = u[k];
    if (i >= g.u_lo && i < g.u_hi && j >= 1 && j <= ny)
      val = val + rmul(dt, g.met ? rhs_u_les_str(u, v, i, j, ny, Metrics(g), blend, g.fx, nu_c, nu_k)
                                 : rhs_u_les_at(u, v, i, j, ny, g.dx, g.dy, blend, g.fx, nu_c, nu_k));
    us[k] = val;
  }
  if (i < nx + 2 && j < ny + 3) {
    const long k = (long)i * (ny + 3) + j;
    double val = v[k];
    if (i >= 1 && i <= nx && j >= g.v_lo && j < g.v_hi)
      val = val + rmul(dt, g.met ? rhs_v_les_str(u, v, i, j, ny, Metrics(g), blend, g.fy, nu_c, nu_k)
                                 : rhs_v_les_at(u, v, i, j, ny, g.dx, g.dy, blend, g.fy, nu_c, nu_k));
    vs[k] = val;
  }
}

// Stateless RHS into (nx+1, ny) and (nx, ny+1) blocks.
__global__ void k_rhs(const double* __restrict__ u, const double* __restrict__ v, int nx, int ny,
                      double dx, double dy, double nu, double blend, double fx, double fy,
                      double* __restrict__ rhs_u, double* __restrict__ rhs_v) {
  pdl_begin();
  const int j = blockIdx.x * blockDim.x + threadIdx.x;   // 0..ny
  const int i = blockIdx.y * blockDim.y + threadIdx.y;   // 0..nx
  if (i <= nx && j < ny) rhs_u[(long)i * ny + j] = rhs_u_at(u, v, i + 1, j + 1, ny, dx, dy, nu, blend, fx);
  if (i < nx && j <= ny) rhs_v[(long)i * (ny + 1) + j] = rhs_v_at(u, v, i + 1, j + 1, ny, dx, dy, nu, blend, fy);
}

// Stateless RHS of a stretched mesh.
__global__ void k_rhs_str(const double* __restrict__ u, const double* __restrict__ v, Geo g, double blend,
                          double* __restrict__ rhs_u, double* __restrict__ rhs_v) {
  pdl_begin();
  const int nx = g.nx, ny = g.ny;
  const Metrics M(g);
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y * blockDim.y + threadIdx.y;
  if (i <= nx && j < ny) rhs_u[(long)i * ny + j] = rhs_u_str(u, v, i + 1, j + 1, ny, M, g.nu, blend, g.fx);
  if (i < nx && j <= ny) rhs_v[(long)i * (ny + 1) + j] = rhs_v_str(u, v, i + 1, j + 1, ny, M, g.nu, blend, g.fy);
}

// Predictor: us = U + dt*rhs_u on the solvable u-faces, U elsewhere (same for
// v), where U is the stage input (pycfd/core/solver.py:619-622).  dt and the
// upwind blend are read from device scalars so a captured step can be replayed.
__global__ void k_predictor(StageIn u, StageIn v, double* __restrict__ us, double* __restrict__ vs,
                            Geo g, const double* __restrict__ S) {
  pdl_begin();
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y * blockDim.y + threadIdx.y;
  const int nx = g.nx, ny = g.ny;
  const double dt = S[S_DT], blend = S[S_BLEND];
  if (i < nx + 3 && j < ny + 2) {
    const long k = (long)i * (ny + 2) + j;
    double val = u[k];
    if (i >= g.u_lo && i < g.u_hi && j >= 1 && j <= ny)
      val = val + rmul(dt, g.met ? rhs_u_str(u, v, i, j, ny, Metrics(g), g.nu, blend, g.fx)
                                 : rhs_u_at(u, v, i, j, ny, g.dx, g.dy, g.nu, blend, g.fx));
    us[k] = val;
  }
  if (i < nx + 2 && j < ny + 3) {
    const long k = (long)i * (ny + 3) + j;
    double val = v[k];
    if (i >= 1 && i <= nx && j >= g.v_lo && j < g.v_hi)
      val = val + rmul(dt, g.met ? rhs_v_str(u, v, i, j, ny, Metrics(g), g.nu, blend, g.fy)
                                 : rhs_v_at(u, v, i, j, ny, g.dx, g.dy, g.nu, blend, g.fy));
    vs[k] = val;
  }
}

__device__ __forceinline__ double cell_div(const double* u, const double* v, int ci, int cj,
                                           int ny, double dx, double dy) {
  const long W = ny + 2, WV = ny + 3;
  return (u[(long)(ci + 2) * W + cj + 1] - u[(long)(ci + 1) * W + cj + 1]) / dx +
         (v[(long)(ci + 1) * WV + cj + 2] - v[(long)(ci + 1) * WV + cj + 1]) / dy;
}

// The divergence of cell (ci, cj) divided by the cell's own width and height
// (pycfd/core/solver.py:530-543): hx[ci], hy[cj] on a stretched mesh.
__device__ __forceinline__ double cell_div_g(const double* u, const double* v, int ci, int cj, const Geo& g) {
  if (g.met) {
    const Metrics M(g);
    return cell_div(u, v, ci, cj, g.ny, M.hx(ci), M.hy(cj));
  }
  return cell_div(u, v, ci, cj, g.ny, g.dx, g.dy);
}

__global__ void k_divergence(const double* __restrict__ u, const double* __restrict__ v, int nx,
                             int ny, double dx, double dy, double* __restrict__ out) {
  pdl_begin();
  for (int i = blockIdx.y * blockDim.y + threadIdx.y; i < nx; i += gridDim.y * blockDim.y)
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < ny; j += gridDim.x * blockDim.x)
      out[(long)i * ny + j] = cell_div(u, v, i, j, ny, dx, dy);
}

// Divergence on the solver's mesh (uniform or stretched), flat (nx, ny).
__global__ void k_divergence_g(const double* __restrict__ u, const double* __restrict__ v, Geo g,
                               double* __restrict__ out) {
  pdl_begin();
  const long n = (long)g.nx * g.ny;
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
    const int i = (int)(c / g.ny), j = (int)(c - (long)i * g.ny);
    out[c] = cell_div_g(u, v, i, j, g);
  }
}

// Poisson right-hand side b = div/dt (+ Dirichlet term), zero on non-solvable
// rows, with the fluid sum for the compatibility mean
// (pycfd/core/solver.py:659-661, pycfd/core/pressure.py:300-308).
// rhs_in != nullptr: take a given right-hand side instead of the divergence.
__global__ void k_div_rhs(const double* __restrict__ u, const double* __restrict__ v,
                          const double* __restrict__ rhs_in, const uint8_t* __restrict__ flags,
                          Geo g, const double* __restrict__ S, double* __restrict__ b,
                          RedBuf rb, double* __restrict__ Sout) {
  pdl_begin();
  const double dt = S[S_DT];
  double acc[1] = {0.0};
  FOR_CELLS(g) {
    const int c = i * g.ny + j;
    const uint8_t f = flags[c];
    double val = 0.0;
    if (f & F_SOLV) {
      const double r = rhs_in ? rhs_in[c] : cell_div_g(u, v, i, j, g) / dt;
      // b = rhs * row_scale + bc (pycfd/core/pressure.py:300-308); row_scale is 1 on a uniform mesh
      val = (g.met ? rmul(r, Metrics(g).row_scale(i, j)) : r * 1.0) + fine_bc(f, i, j, g);
      acc[0] += val;
    }
    b[c] = val;
  }
  grid_reduce<1>(acc, rb, [&](double* t) { Sout[S_MEAN_B] = g.n_fluid ? t[0] / g.n_fluid : 0.0; });
}

// Ghosted pressure at a face-adjacent ghost or interior position from the
// normalised interior solution x (pycfd/core/boundary.py:166-169, :293-303,
// :412-420).  Only non-corner ghosts are formed here.
__device__ __forceinline__ double p_at(const double* x, int i, int j, const Geo& g) {
  const int nx = g.nx, ny = g.ny;
  if (i == 0) {
    if (g.periodic_x) return x[(long)(nx - 1) * ny + (j - 1)];
    const double in = x[(long)(j - 1)];
    return g.dir_w ? 2.0 * g.pref_w - in : in;
  }
  if (i == nx + 1) {
    if (g.periodic_x) return x[(long)(j - 1)];
    const double in = x[(long)(nx - 1) * ny + (j - 1)];
    return g.dir_e ? 2.0 * g.pref_e - in : in;
  }
  if (j == 0) {
    if (g.periodic_y) return x[(long)(i - 1) * ny + ny - 1];
    const double in = x[(long)(i - 1) * ny];
    return g.dir_s ? 2.0 * g.pref_s - in : in;
  }
  if (j == ny + 1) {
    if (g.periodic_y) return x[(long)(i - 1) * ny];
    const double in = x[(long)(i - 1) * ny + ny - 1];
    return g.dir_n ? 2.0 * g.pref_n - in : in;
  }
  return x[(long)(i - 1) * ny + (j - 1)];
}

// Pressure ghost ring of the ghosted p from the interior solution x, run by
// one thread block: rebuilt from zero (the reference fills a fresh zero
// array) wall by wall in the reference's order, so the corners agree too
// (pycfd/core/boundary.py:166-169, :293-303, :412-420).
__device__ void p_ghost_ring(double* __restrict__ p, const double* __restrict__ x, const Geo& g,
                             const int* __restrict__ bc_kind) {
  const int nx = g.nx, ny = g.ny;
  const long WP = ny + 2;
  for (int k = threadIdx.x; k < 2 * (nx + 2) + 2 * ny; k += blockDim.x) {
    long idx;
    if (k < ny + 2) idx = k;                                         // row 0
    else if (k < 2 * (ny + 2)) idx = (long)(nx + 1) * WP + (k - (ny + 2));  // row nx+1
    else if (k < 2 * (ny + 2) + nx) idx = (long)(k - 2 * (ny + 2) + 1) * WP;  // col 0
    else idx = (long)(k - 2 * (ny + 2) - nx + 1) * WP + ny + 1;            // col ny+1
    p[idx] = 0.0;
  }
  __syncthreads();
  for (int w = 0; w < 4; ++w) {
    const int kind = bc_kind[w];
    if (kind == BC_PERIODIC) continue;
    const int axis = w < 2 ? 0 : 1;
    const int ghost = (w == W_LEFT || w == W_BOTTOM) ? 0 : (axis == 0 ? nx + 1 : ny + 1);
    const int inner = (w == W_LEFT || w == W_BOTTOM) ? 1 : (axis == 0 ? nx : ny);
    const double pref = w == W_LEFT ? g.pref_w : w == W_RIGHT ? g.pref_e : w == W_BOTTOM ? g.pref_s : g.pref_n;
    const int len = axis == 0 ? ny + 2 : nx + 2;
    for (int k = threadIdx.x; k < len; k += blockDim.x) {
      // interior value of the line (may itself be a ghost set earlier: read p)
      const int ii = axis == 0 ? inner : k, jj = axis == 0 ? k : inner;
      double in;
      if (ii >= 1 && ii <= nx && jj >= 1 && jj <= ny) in = x[(long)(ii - 1) * ny + (jj - 1)];
      else in = p[(long)ii * WP + jj];
      const double val = (kind == BC_PRESSURE_OUTLET) ? 2.0 * pref - in : in;
      const int gi = axis == 0 ? ghost : k, gj = axis == 0 ? k : ghost;
      p[(long)gi * WP + gj] = val;
    }
    __syncthreads();
  }
  if (g.periodic_x) {
    for (int k = threadIdx.x; k < ny + 2; k += blockDim.x) {
      const double a = (k >= 1 && k <= ny) ? x[(long)(nx - 1) * ny + k - 1] : p[(long)nx * WP + k];
      p[k] = a;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < ny + 2; k += blockDim.x) {
      const double a = (k >= 1 && k <= ny) ? x[(long)(k - 1)] : p[WP + k];
      p[(long)(nx + 1) * WP + k] = a;
    }
    __syncthreads();
  }
  if (g.periodic_y) {
    for (int k = threadIdx.x; k < nx + 2; k += blockDim.x) {
      const double a = (k >= 1 && k <= nx) ? x[(long)(k - 1) * ny + ny - 1] : p[(long)k * WP + ny];
      p[(long)k * WP] = a;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nx + 2; k += blockDim.x) {
      const double a = (k >= 1 && k <= nx) ? x[(long)(k - 1) * ny] : p[(long)k * WP + 1];
      p[(long)k * WP + ny + 1] = a;
    }
  }
}

// Velocity correction u -= dt*(p[m]-p[m-1])/dx on exactly the solvable faces
// (pycfd/core/solver.py:665-682), plus the ghosted pressure output.  The last
// block fills the pressure ghost layer wall by wall in the reference's order
// (so the corner values agree too); all other blocks update faces and copy
// the interior.  dt_override < 0 reads dt from the device scalars.
__global__ void k_correct(double* __restrict__ u, double* __restrict__ v,
                          double* __restrict__ p, const double* __restrict__ x, Geo g,
                          const double* __restrict__ S, double dt_override,
                          const int* __restrict__ bc_kind) {
  pdl_begin();
  const int nx = g.nx, ny = g.ny;
  const double dt = dt_override > 0.0 ? dt_override : S[S_DT];
  if (blockIdx.x == gridDim.x - 1) {
    // The other blocks copy the interior and update the faces.
    p_ghost_ring(p, x, g, bc_kind);
    return;
  }
  // 2D sweep over rows i = 0..nx+1 (blocks in y), columns j = 0..ny+1 (threads)
  const int rows = nx + 2;
  for (int r = blockIdx.x; r < rows; r += gridDim.x - 1) {
    for (int j = threadIdx.x; j < ny + 3; j += blockDim.x) {
      // interior copy of p: ghosted row r = i+1 for i in [0, nx)
      if (r >= 1 && r <= nx && j >= 1 && j <= ny) p[(long)r * (ny + 2) + j] = x[(long)(r - 1) * ny + (j - 1)];
      // u faces [u_lo, u_hi) x [1, ny]: row m = r
      if (r >= g.u_lo && r < g.u_hi && j >= 1 && j <= ny) {
        const long k = (long)r * (ny + 2) + j;
        u[k] = u[k] - dt * (p_at(x, r, j, g) - p_at(x, r - 1, j, g)) / (g.met ? Metrics(g).hxu(r - 1) : g.dx);
      }
      // v faces [1, nx] x [v_lo, v_hi): row i = r
      if (r >= 1 && r <= nx && j >= g.v_lo && j < g.v_hi) {
        const long k = (long)r * (ny + 3) + j;
        v[k] = v[k] - dt * (p_at(x, r, j, g) - p_at(x, r, j - 1, g)) / (g.met ? Metrics(g).hyv(j - 1) : g.dy);
      }
    }
  }
}

// out = ca*a + cb*b over whole arrays (pycfd/core/solver.py:705-721).
__global__ void k_combine(const double* __restrict__ a, const double* __restrict__ b, double ca,
                          double cb, double* __restrict__ out, long n) {
  pdl_begin();
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
    out[k] = rmul(ca, a[k]) + rmul(cb, b[k]);
}

// Field statistics: max|u|, max|v| (physical faces), max|du|, max|dv|,
// max|div| (fluid), kinetic energy sum, max|vorticity|, non-finite count.
// Blocks stride over array rows, threads over the contiguous y index.
__global__ void k_field_stats(const double* __restrict__ u, const double* __restrict__ v,
                              const double* __restrict__ p, const double* __restrict__ up,
                              const double* __restrict__ vp, const uint8_t* __restrict__ solid,
                              Geo g, RedBuf rb, double* __restrict__ Sout) {
  pdl_begin();
  const int nx = g.nx, ny = g.ny;
  const long W = ny + 2, WV = ny + 3;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // max,max,max,max,max,sum,max,sum
  for (int r = blockIdx.x; r < nx + 3; r += gridDim.x) {
    for (int j = threadIdx.x; j < ny + 3; j += blockDim.x) {
      if (j < ny + 2) {
        const long k = (long)r * W + j;
        const double a = u[k];
        if (!isfinite(a)) acc[7] += 1.0;
        if (r >= 1 && r <= nx + 1 && j >= 1 && j <= ny) acc[0] = fmax(acc[0], fabs(a));
        if (up) acc[2] = fmax(acc[2], fabs(a - up[k]));
      }
      if (r < nx + 2) {
        const long k = (long)r * WV + j;
        const double a = v[k];
        if (!isfinite(a)) acc[7] += 1.0;
        if (r >= 1 && r <= nx && j >= 1 && j <= ny + 1) acc[1] = fmax(acc[1], fabs(a));
        if (vp) acc[3] = fmax(acc[3], fabs(a - vp[k]));
        if (p && j < ny + 2 && !isfinite(p[(long)r * W + j])) acc[7] += 1.0;
      }
      if (r < nx && j < ny) {
        const int i = r;
        const bool sol = solid && solid[(long)i * ny + j];
        if (!sol) acc[4] = fmax(acc[4], fabs(cell_div_g(u, v, i, j, g)));
        const double uc = 0.5 * (u[(long)(i + 1) * W + j + 1] + u[(long)(i + 2) * W + j + 1]);
        const double vc = 0.5 * (v[(long)(i + 1) * WV + j + 1] + v[(long)(i + 1) * WV + j + 2]);
        // kinetic energy density; on a stretched mesh weighted by the cell area here
        // (the integral), on a uniform one multiplied by dx dy by the reader
        if (!sol) acc[5] += g.met ? rmul(0.5 * (uc * uc + vc * vc), rmul(Metrics(g).hx(i), Metrics(g).hy(j)))
                                  : 0.5 * (uc * uc + vc * vc);
        // vorticity at the four corners of the cell (pycfd/analysis/postprocess.py:21-40)
        double w4 = 0.0;
        for (int di = 0; di < 2; ++di)
          for (int dj = 0; dj < 2; ++dj) {
            const int a = i + di, bb = j + dj;
            const double dvdx = (v[(long)(a + 1) * WV + bb + 1] - v[(long)a * WV + bb + 1]) /
                                (g.met ? Metrics(g).hxu(a) : g.dx);
            const double dudy = (u[(long)(a + 1) * W + bb + 1] - u[(long)(a + 1) * W + bb]) /
                                (g.met ? Metrics(g).hyv(bb) : g.dy);
            w4 += dvdx - dudy;
          }
        acc[6] = fmax(acc[6], fabs(0.25 * w4));
      }
    }
  }
  grid_reduce<8, 0x5Fu>(acc, rb, [&](double* t) {
    for (int k = 0; k < 8; ++k) Sout[S_STAT0 + k] = t[k];
  });
}

}  // namespace pcfd
