// Discrete adjoint of the lid-driven cavity step (the controls: a lid-velocity
// profile and a smoothed obstacle), as hand-written kernels.  The forward
// primitives are the library step's own arithmetic for the cavity (predictor
// from rhs_u_at / rhs_v_at, the ordered wall lines, the projection's
// divergence and correction, the Runge-Kutta combinations), extended by the
// profile U(x) on the moving lid and by direct forcing u <- (1 - chi) u on the
// solvable faces (a 0/1 chi is the reference's mask, pycfd/core/solver.py:553-599).
// Each adjoint kernel is the exact transpose of its forward primitive written
// in GATHER form: every output element sums, in a fixed order, the
// contributions of the forward entries that read it, so results are
// deterministic and need no atomics.
//
// Layout: u (n+3) x (n+2), v (n+2) x (n+3), row-major, y fastest; the Poisson
// vectors n x n.  Solvable faces: u m = 2..n, j = 1..n; v i = 1..n, k = 2..n.
#pragma once
#include "common.cuh"
#include "stencil.cuh"

namespace pcfd {

struct AdjGeo {
  int n;
  double h, nu;
  __device__ __forceinline__ long U(int m, int j) const { return (long)m * (n + 2) + j; }
  __device__ __forceinline__ long V(int i, int k) const { return (long)i * (n + 3) + k; }
  __device__ __forceinline__ bool u_solv(int m, int j) const { return m >= 2 && m <= n && j >= 1 && j <= n; }
  __device__ __forceinline__ bool v_solv(int i, int k) const { return i >= 1 && i <= n && k >= 2 && k <= n; }
};

#define ADJ_FOR(count) \
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < (count); e += (long)gridDim.x * blockDim.x)

// ---- forward ------------------------------------------------------------------------
// us = U + dt rhs(U) on the solvable faces, U elsewhere (the predictor of the library step).
__global__ void k_adj_predictor(AdjGeo G, const double* __restrict__ U, const double* __restrict__ V,
                                double* __restrict__ us, double* __restrict__ vs, double dt) {
  const int n = G.n;
  const long nu = (long)(n + 3) * (n + 2), nv = (long)(n + 2) * (n + 3);
  ADJ_FOR(nu + nv) {
    if (e < nu) {
      const int m = (int)(e / (n + 2)), j = (int)(e % (n + 2));
      double val = U[e];
      if (G.u_solv(m, j)) val = val + rmul(dt, rhs_u_at(U, V, m, j, n, G.h, G.h, G.nu, 0.0, 0.0));
      us[e] = val;
    } else {
      const long f = e - nu;
      const int i = (int)(f / (n + 3)), k = (int)(f % (n + 3));
      double val = V[f];
      if (G.v_solv(i, k)) val = val + rmul(dt, rhs_v_at(U, V, i, k, n, G.h, G.h, G.nu, 0.0, 0.0));
      vs[f] = val;
    }
  }
}

// The cavity's wall pass in the reference's order (left, right, bottom, top),
// each line assignment completed before the next (corners), the top wall
// moving with the profile lid[m] (m = 0..n+2).  One block.
__global__ void k_adj_walls(AdjGeo G, double* __restrict__ u, double* __restrict__ v,
                           const double* __restrict__ lid) {
  const int n = G.n, t = threadIdx.x, T = blockDim.x;
  // left
  for (int j = t; j < n + 2; j += T) u[G.U(1, j)] = 0.0;
  __syncthreads();
  for (int j = t; j < n + 2; j += T) u[G.U(0, j)] = 2.0 * u[G.U(1, j)] - u[G.U(2, j)];
  for (int k = t; k < n + 3; k += T) v[G.V(0, k)] = -v[G.V(1, k)];
  __syncthreads();
  // right
  for (int j = t; j < n + 2; j += T) u[G.U(n + 1, j)] = 0.0;
  __syncthreads();
  for (int j = t; j < n + 2; j += T) u[G.U(n + 2, j)] = 2.0 * u[G.U(n + 1, j)] - u[G.U(n, j)];
  for (int k = t; k < n + 3; k += T) v[G.V(n + 1, k)] = -v[G.V(n, k)];
  __syncthreads();
  // bottom
  for (int i = t; i < n + 2; i += T) v[G.V(i, 1)] = 0.0;
  __syncthreads();
  for (int i = t; i < n + 2; i += T) v[G.V(i, 0)] = 2.0 * v[G.V(i, 1)] - v[G.V(i, 2)];
  for (int m = t; m < n + 3; m += T) u[G.U(m, 0)] = -u[G.U(m, 1)];
  __syncthreads();
  // top
  for (int i = t; i < n + 2; i += T) v[G.V(i, n + 1)] = 0.0;
  __syncthreads();
  for (int i = t; i < n + 2; i += T) v[G.V(i, n + 2)] = 2.0 * v[G.V(i, n + 1)] - v[G.V(i, n)];
  for (int m = t; m < n + 3; m += T) u[G.U(m, n + 1)] = 2.0 * lid[m] - u[G.U(m, n)];
}

// Direct forcing with a smoothed mask: out = (1 - chi) in on the solvable faces, in elsewhere.
__global__ void k_adj_mask(AdjGeo G, const double* __restrict__ ui, const double* __restrict__ vi,
                           double* __restrict__ uo, double* __restrict__ vo, const double* __restrict__ cu,
                           const double* __restrict__ cv) {
  const int n = G.n;
  const long nu = (long)(n + 3) * (n + 2), nv = (long)(n + 2) * (n + 3);
  ADJ_FOR(nu + nv) {
    if (e < nu) {
      const int m = (int)(e / (n + 2)), j = (int)(e % (n + 2));
      uo[e] = G.u_solv(m, j) ? (1.0 - cu[e]) * ui[e] : ui[e];
    } else {
      const long f = e - nu;
      const int i = (int)(f / (n + 3)), k = (int)(f % (n + 3));
      vo[f] = G.v_solv(i, k) ? (1.0 - cv[f]) * vi[f] : vi[f];
    }
  }
}

// Poisson right-hand side of the projection: div(u) / dt on the cells.
__global__ void k_adj_div(AdjGeo G, const double* __restrict__ u, const double* __restrict__ v,
                          double* __restrict__ b, double dt) {
  const int n = G.n;
  ADJ_FOR((long)n * n) {
    const int i = (int)(e / n), j = (int)(e % n);
    b[e] = cell_div(u, v, i, j, n, G.h, G.h) / dt;
  }
}

// Correction of the solvable faces by the pressure gradient (p: n x n cells).
__global__ void k_adj_correct(AdjGeo G, double* __restrict__ u, double* __restrict__ v,
                              const double* __restrict__ p, double dt) {
  const int n = G.n;
  const long nu = (long)(n + 3) * (n + 2), nv = (long)(n + 2) * (n + 3);
  ADJ_FOR(nu + nv) {
    if (e < nu) {
      const int m = (int)(e / (n + 2)), j = (int)(e % (n + 2));
      if (G.u_solv(m, j)) u[e] = u[e] - dt * (p[(long)(m - 1) * n + (j - 1)] - p[(long)(m - 2) * n + (j - 1)]) / G.h;
    } else {
      const long f = e - nu;
      const int i = (int)(f / (n + 3)), k = (int)(f % (n + 3));
      if (G.v_solv(i, k)) v[f] = v[f] - dt * (p[(long)(i - 1) * n + (k - 1)] - p[(long)(i - 1) * n + (k - 2)]) / G.h;
    }
  }
}

// out = ca a + cb b, elementwise (the Runge-Kutta combinations and their transposes).
__global__ void k_adj_lincomb(double* __restrict__ out, const double* __restrict__ a, double ca,
                              const double* __restrict__ b, double cb, long count) {
  ADJ_FOR(count) out[e] = rmul(ca, a[e]) + rmul(cb, b[e]);
}

// Kinetic energy of the cells below the split, one block: 0.5 (uc^2 + vc^2)
// weighted by lower[j], summed in a fixed order, times h^2.
__global__ void k_adj_objective(AdjGeo G, const double* __restrict__ u, const double* __restrict__ v,
                                const double* __restrict__ lower, double* __restrict__ out) {
  const int n = G.n;
  double acc = 0.0;
  for (long e = threadIdx.x; e < (long)n * n; e += blockDim.x) {
    const int i = (int)(e / n), j = (int)(e % n);
    const double uc = 0.5 * (u[G.U(i + 1, j + 1)] + u[G.U(i + 2, j + 1)]);
    const double vc = 0.5 * (v[G.V(i + 1, j + 1)] + v[G.V(i + 1, j + 2)]);
    acc += rmul(0.5 * (rmul(uc, uc) + rmul(vc, vc)), lower[j]);
  }
  double a[1] = {acc};
  block_reduce<1>(a);
  if (threadIdx.x == 0) *out = a[0] * G.h * G.h;
}

// ---- adjoints ------------------------------------------------------------------------
// Transpose of the predictor at (U, V): with gr = dt gus on the solvable faces
// (0 elsewhere), gU = (d rhs / dU)^T gr + gus and the same for V.  The
// transposed advection-diffusion Jacobian is gathered per face in the order of
// its scatter statements: u-momentum centre, east, west, north, south, then the
// v-momentum's u terms (and symmetrically for v).
struct AdjRhs {
  AdjGeo G;
  const double* U;
  const double* V;
  const double* gus;
  const double* gvs;
  double dt;
  // the u-momentum entry (k, l), k = 0..n, l = 0..n-1, lives at u face (k+1, l+1)
  __device__ __forceinline__ double gru(int k, int l) const {
    return G.u_solv(k + 1, l + 1) ? dt * gus[G.U(k + 1, l + 1)] : 0.0;
  }
  __device__ __forceinline__ double grv(int i, int q) const {
    return G.v_solv(i + 1, q + 1) ? dt * gvs[G.V(i + 1, q + 1)] : 0.0;
  }
};

// The pieces of one u-momentum entry's transpose (gur, gul, gut, gVT, gub, gVB, gl).
__device__ __forceinline__ void adj_u_terms(const AdjRhs& R, int k, int l, double* o) {
  const AdjGeo& G = R.G;
  const double* u = R.U;
  const double* v = R.V;
  const double h = G.h;
  const double U0 = u[G.U(k + 1, l + 1)], UE = u[G.U(k + 2, l + 1)], UW = u[G.U(k, l + 1)];
  const double UN = u[G.U(k + 1, l + 2)], US = u[G.U(k + 1, l)];
  const double VT = 0.5 * (v[G.V(k, l + 2)] + v[G.V(k + 1, l + 2)]);
  const double VB = 0.5 * (v[G.V(k, l + 1)] + v[G.V(k + 1, l + 1)]);
  const double ur = 0.5 * (U0 + UE), ul = 0.5 * (UW + U0);
  const double ut = 0.5 * (U0 + UN), ub = 0.5 * (US + U0);
  const double g = R.gru(k, l);
  o[0] = -2.0 * ur * g / h;   // gur
  o[1] = 2.0 * ul * g / h;    // gul
  o[2] = -VT * g / h;         // gut
  o[3] = -ut * g / h;         // gVT
  o[4] = VB * g / h;          // gub
  o[5] = ub * g / h;          // gVB
  o[6] = G.nu * g / (h * h);  // gl
}

// The pieces of one v-momentum entry's transpose (gUR, gvr, gUL, gvl, gvt, gvb, gl).
__device__ __forceinline__ void adj_v_terms(const AdjRhs& R, int i, int q, double* o) {
  const AdjGeo& G = R.G;
  const double* u = R.U;
  const double* v = R.V;
  const double h = G.h;
  const double V0 = v[G.V(i + 1, q + 1)], VN = v[G.V(i + 1, q + 2)], VS = v[G.V(i + 1, q)];
  const double VE = v[G.V(i + 2, q + 1)], VW = v[G.V(i, q + 1)];
  const double UR = 0.5 * (u[G.U(i + 2, q)] + u[G.U(i + 2, q + 1)]);
  const double UL = 0.5 * (u[G.U(i + 1, q)] + u[G.U(i + 1, q + 1)]);
  const double vt = 0.5 * (V0 + VN), vb = 0.5 * (VS + V0);
  const double vr = 0.5 * (V0 + VE), vl = 0.5 * (VW + V0);
  const double g = R.grv(i, q);
  o[0] = -vr * g / h;         // gUR
  o[1] = -UR * g / h;         // gvr
  o[2] = vl * g / h;          // gUL
  o[3] = UL * g / h;          // gvl
  o[4] = -2.0 * vt * g / h;   // gvt
  o[5] = 2.0 * vb * g / h;    // gvb
  o[6] = G.nu * g / (h * h);  // gl
}

__global__ void k_adj_predictor_T(AdjRhs R, double* __restrict__ gU, double* __restrict__ gV) {
  const AdjGeo& G = R.G;
  const int n = G.n;
  const long nu = (long)(n + 3) * (n + 2), nv = (long)(n + 2) * (n + 3);
  double t[7];
  ADJ_FOR(nu + nv) {
    if (e < nu) {
      // u face (m, j): entries (k, l) of the u-momentum with k + a = m, l + b = j
      const int m = (int)(e / (n + 2)), j = (int)(e % (n + 2));
      double acc = 0.0;
      const bool lin = j >= 1 && j <= n;   // rows the u-momentum entries occupy
      if (lin && m >= 1 && m <= n + 1) {   // centre (k, l) = (m-1, j-1)
        adj_u_terms(R, m - 1, j - 1, t);
        acc += 0.5 * t[0] + 0.5 * t[1] + 0.5 * t[2] + 0.5 * t[4] - 4.0 * t[6];
      }
      if (lin && m >= 2 && m <= n + 2) {   // east neighbour of entry (m-2, j-1)
        adj_u_terms(R, m - 2, j - 1, t);
        acc += 0.5 * t[0] + t[6];
      }
      if (lin && m >= 0 && m <= n) {       // west neighbour of entry (m, j-1)
        adj_u_terms(R, m, j - 1, t);
        acc += 0.5 * t[1] + t[6];
      }
      if (m >= 1 && m <= n + 1 && j >= 2 && j <= n + 1) {   // north neighbour of (m-1, j-2)
        adj_u_terms(R, m - 1, j - 2, t);
        acc += 0.5 * t[2] + t[6];
      }
      if (m >= 1 && m <= n + 1 && j >= 0 && j <= n - 1) {   // south neighbour of (m-1, j)
        adj_u_terms(R, m - 1, j, t);
        acc += 0.5 * t[4] + t[6];
      }
      // v-momentum entries (i, q) reading u through UR (u[i+2, q], u[i+2, q+1]) and UL
      if (m >= 2 && m <= n + 1 && j >= 0 && j <= n) {      // UR, first face: (i, q) = (m-2, j)
        adj_v_terms(R, m - 2, j, t);
        acc += 0.5 * t[0];
      }
      if (m >= 2 && m <= n + 1 && j >= 1 && j <= n + 1) {  // UR, second face: (m-2, j-1)
        adj_v_terms(R, m - 2, j - 1, t);
        acc += 0.5 * t[0];
      }
      if (m >= 1 && m <= n && j >= 0 && j <= n) {          // UL, first face: (m-1, j)
        adj_v_terms(R, m - 1, j, t);
        acc += 0.5 * t[2];
      }
      if (m >= 1 && m <= n && j >= 1 && j <= n + 1) {      // UL, second face: (m-1, j-1)
        adj_v_terms(R, m - 1, j - 1, t);
        acc += 0.5 * t[2];
      }
      gU[e] = acc + R.gus[e];
    } else {
      const long f = e - nu;
      const int i = (int)(f / (n + 3)), k = (int)(f % (n + 3));
      double acc = 0.0;
      // u-momentum entries (a, l) reading v through VT (v[a, l+2], v[a+1, l+2]) and VB
      if (i >= 0 && i <= n && k >= 2 && k <= n + 1) {      // VT, first: (a, l) = (i, k-2)
        adj_u_terms(R, i, k - 2, t);
        acc += 0.5 * t[3];
      }
      if (i >= 1 && i <= n + 1 && k >= 2 && k <= n + 1) {  // VT, second: (i-1, k-2)
        adj_u_terms(R, i - 1, k - 2, t);
        acc += 0.5 * t[3];
      }
      if (i >= 0 && i <= n && k >= 1 && k <= n) {          // VB, first: (i, k-1)
        adj_u_terms(R, i, k - 1, t);
        acc += 0.5 * t[5];
      }
      if (i >= 1 && i <= n + 1 && k >= 1 && k <= n) {      // VB, second: (i-1, k-1)
        adj_u_terms(R, i - 1, k - 1, t);
        acc += 0.5 * t[5];
      }
      const bool col = i >= 1 && i <= n;   // columns the v-momentum entries occupy
      if (col && k >= 1 && k <= n + 1) {   // centre (i-1, k-1)
        adj_v_terms(R, i - 1, k - 1, t);
        acc += 0.5 * t[1] + 0.5 * t[3] + 0.5 * t[4] + 0.5 * t[5] - 4.0 * t[6];
      }
      if (i >= 2 && i <= n + 1 && k >= 1 && k <= n + 1) {  // east neighbour of (i-2, k-1)
        adj_v_terms(R, i - 2, k - 1, t);
        acc += 0.5 * t[1] + t[6];
      }
      if (i >= 0 && i <= n - 1 && k >= 1 && k <= n + 1) {  // west neighbour of (i, k-1)
        adj_v_terms(R, i, k - 1, t);
        acc += 0.5 * t[3] + t[6];
      }
      if (col && k >= 2 && k <= n + 2) {   // north neighbour of (i-1, k-2)
        adj_v_terms(R, i - 1, k - 2, t);
        acc += 0.5 * t[4] + t[6];
      }
      if (col && k >= 0 && k <= n) {       // south neighbour of (i-1, k)
        adj_v_terms(R, i - 1, k, t);
        acc += 0.5 * t[5] + t[6];
      }
      gV[f] = acc + R.gvs[f];
    }
  }
}

// Transpose of the wall pass: the line assignments in reverse order (each
// assignment x <- a y + b z becomes y += a gx, z += b gx, gx <- 0), the lid's
// gradient 2 gu[:, n+1] accumulated into glid.  One block.
__global__ void k_adj_walls_T(AdjGeo G, double* __restrict__ gu, double* __restrict__ gv,
                             double* __restrict__ glid) {
  const int n = G.n, t = threadIdx.x, T = blockDim.x;
  // top: u[:, n+1] = 2 lid - u[:, n]; v[:, n+2] = 2 v[:, n+1] - v[:, n]; v[:, n+1] = 0
  for (int m = t; m < n + 3; m += T) {
    const double g = gu[G.U(m, n + 1)];
    glid[m] = glid[m] + 2.0 * g;
    gu[G.U(m, n)] -= g;
    gu[G.U(m, n + 1)] = 0.0;
  }
  for (int i = t; i < n + 2; i += T) {
    const double g = gv[G.V(i, n + 2)];
    gv[G.V(i, n + 2)] = 0.0;
    gv[G.V(i, n + 1)] += 2.0 * g;
    gv[G.V(i, n)] -= g;
    gv[G.V(i, n + 1)] = 0.0;
  }
  __syncthreads();
  // bottom: u[:, 0] = -u[:, 1]; v[:, 0] = 2 v[:, 1] - v[:, 2]; v[:, 1] = 0
  for (int m = t; m < n + 3; m += T) {
    gu[G.U(m, 1)] -= gu[G.U(m, 0)];
    gu[G.U(m, 0)] = 0.0;
  }
  for (int i = t; i < n + 2; i += T) {
    const double g = gv[G.V(i, 0)];
    gv[G.V(i, 0)] = 0.0;
    gv[G.V(i, 1)] += 2.0 * g;
    gv[G.V(i, 2)] -= g;
    gv[G.V(i, 1)] = 0.0;
  }
  __syncthreads();
  // right: v[n+1, :] = -v[n, :]; u[n+2, :] = 2 u[n+1, :] - u[n, :]; u[n+1, :] = 0
  for (int k = t; k < n + 3; k += T) {
    gv[G.V(n, k)] -= gv[G.V(n + 1, k)];
    gv[G.V(n + 1, k)] = 0.0;
  }
  for (int j = t; j < n + 2; j += T) {
    const double g = gu[G.U(n + 2, j)];
    gu[G.U(n + 2, j)] = 0.0;
    gu[G.U(n + 1, j)] += 2.0 * g;
    gu[G.U(n, j)] -= g;
    gu[G.U(n + 1, j)] = 0.0;
  }
  __syncthreads();
  // left: v[0, :] = -v[1, :]; u[0, :] = 2 u[1, :] - u[2, :]; u[1, :] = 0
  for (int k = t; k < n + 3; k += T) {
    gv[G.V(1, k)] -= gv[G.V(0, k)];
    gv[G.V(0, k)] = 0.0;
  }
  for (int j = t; j < n + 2; j += T) {
    const double g = gu[G.U(0, j)];
    gu[G.U(0, j)] = 0.0;
    gu[G.U(1, j)] += 2.0 * g;
    gu[G.U(2, j)] -= g;
    gu[G.U(1, j)] = 0.0;
  }
}

// Transpose of the smoothed mask at its input (ui, vi): the chi gradients
// -in * g on the solvable faces accumulated into acc_cu / acc_cv, and
// g <- (1 - chi) g there (in place).
__global__ void k_adj_mask_T(AdjGeo G, const double* __restrict__ ui, const double* __restrict__ vi,
                             double* __restrict__ gu, double* __restrict__ gv, const double* __restrict__ cu,
                             const double* __restrict__ cv, double* __restrict__ acc_cu,
                             double* __restrict__ acc_cv) {
  const int n = G.n;
  const long nu = (long)(n + 3) * (n + 2), nv = (long)(n + 2) * (n + 3);
  ADJ_FOR(nu + nv) {
    if (e < nu) {
      const int m = (int)(e / (n + 2)), j = (int)(e % (n + 2));
      if (G.u_solv(m, j)) {
        const double g = gu[e];
        acc_cu[e] = acc_cu[e] + (-ui[e] * g);
        gu[e] = (1.0 - cu[e]) * g;
      }
    } else {
      const long f = e - nu;
      const int i = (int)(f / (n + 3)), k = (int)(f % (n + 3));
      if (G.v_solv(i, k)) {
        const double g = gv[f];
        acc_cv[f] = acc_cv[f] + (-vi[f] * g);
        gv[f] = (1.0 - cv[f]) * g;
      }
    }
  }
}

// Transpose of the projection, first half: q = G^T g on the cells (the
// transposed gradient of the solvable faces), q[i, j] gathered in the order
// +u(low face), -u(high face), +v(low face), -v(high face).
__global__ void k_adj_grad_T(AdjGeo G, const double* __restrict__ gu, const double* __restrict__ gv,
                             double* __restrict__ q) {
  const int n = G.n;
  const double h = G.h;
  ADJ_FOR((long)n * n) {
    const int i = (int)(e / n), j = (int)(e % n);
    double acc = 0.0;
    if (i >= 1) acc += gu[G.U(i + 1, j + 1)] / h;
    if (i <= n - 2) acc -= gu[G.U(i + 2, j + 1)] / h;
    if (j >= 1) acc += gv[G.V(i + 1, j + 1)] / h;
    if (j <= n - 2) acc -= gv[G.V(i + 1, j + 2)] / h;
    q[e] = acc;
  }
}

// Second half: g <- g - D^T psi (psi the solve of q; D the cell divergence).
__global__ void k_adj_div_T(AdjGeo G, double* __restrict__ gu, double* __restrict__ gv,
                            const double* __restrict__ psi) {
  const int n = G.n;
  const double h = G.h;
  const long nu = (long)(n + 3) * (n + 2), nv = (long)(n + 2) * (n + 3);
  ADJ_FOR(nu + nv) {
    if (e < nu) {
      const int m = (int)(e / (n + 2)), j = (int)(e % (n + 2));
      if (j >= 1 && j <= n) {
        double g = gu[e];
        if (m >= 2 && m <= n + 1) g -= psi[(long)(m - 2) * n + (j - 1)] / h;
        if (m >= 1 && m <= n) g += psi[(long)(m - 1) * n + (j - 1)] / h;
        gu[e] = g;
      }
    } else {
      const long f = e - nu;
      const int i = (int)(f / (n + 3)), k = (int)(f % (n + 3));
      if (i >= 1 && i <= n) {
        double g = gv[f];
        if (k >= 2 && k <= n + 1) g -= psi[(long)(i - 1) * n + (k - 2)] / h;
        if (k >= 1 && k <= n) g += psi[(long)(i - 1) * n + (k - 1)] / h;
        gv[f] = g;
      }
    }
  }
}

// Gradient of the objective at (u, v).
__global__ void k_adj_objective_T(AdjGeo G, const double* __restrict__ u, const double* __restrict__ v,
                                  const double* __restrict__ lower, double* __restrict__ gu,
                                  double* __restrict__ gv) {
  const int n = G.n;
  const double h = G.h;
  const long nu = (long)(n + 3) * (n + 2), nv = (long)(n + 2) * (n + 3);
  ADJ_FOR(nu + nv) {
    if (e < nu) {
      const int m = (int)(e / (n + 2)), j = (int)(e % (n + 2));
      double acc = 0.0;
      if (j >= 1 && j <= n) {
        const double w = lower[j - 1] * h * h;
        if (m >= 1 && m <= n) {   // first face of cell m-1
          const double uc = 0.5 * (u[G.U(m, j)] + u[G.U(m + 1, j)]);
          acc += 0.5 * uc * w;
        }
        if (m >= 2 && m <= n + 1) {   // second face of cell m-2
          const double uc = 0.5 * (u[G.U(m - 1, j)] + u[G.U(m, j)]);
          acc += 0.5 * uc * w;
        }
      }
      gu[e] = acc;
    } else {
      const long f = e - nu;
      const int i = (int)(f / (n + 3)), k = (int)(f % (n + 3));
      double acc = 0.0;
      if (i >= 1 && i <= n) {
        if (k >= 1 && k <= n) {
          const double vc = 0.5 * (v[G.V(i, k)] + v[G.V(i, k + 1)]);
          acc += 0.5 * vc * (lower[k - 1] * h * h);
        }
        if (k >= 2 && k <= n + 1) {
          const double vc = 0.5 * (v[G.V(i, k - 1)] + v[G.V(i, k)]);
          acc += 0.5 * vc * (lower[k - 2] * h * h);
        }
      }
      gv[f] = acc;
    }
  }
}

}  // namespace pcfd
