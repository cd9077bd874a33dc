// Boundary passes, outlet mass balance, immersed-boundary mask and periodic
// face wrap, executed by one thread block as an ordered program of line
// assignments.  The reference applies its walls one after another on whole
// rows/columns (corners included), so later walls overwrite the corner ghosts
// of earlier ones; running the same sequence with a barrier between dependent
// lines reproduces every value, corners included
// (pycfd/core/boundary.py:141-164, :375-420, :423-487;
//  pycfd/core/solver.py:553-607).
#pragma once
#include "common.cuh"

namespace pcfd {

enum BcOp : int { OP_END = 0, OP_VEL_PRED, OP_VEL_CORR, OP_MASS, OP_MASK_NONE, OP_MASK_RESET,
                  OP_MASK_ACC, OP_WRAP_FACES };

struct BcProgram { int op[8]; };

struct BcTable {
  int kind[4];
  double vel[4];
  double pref[4];
  const double* profile[4];          // parabolic inlet line or nullptr
  // mask face lists (linear indices into u / v), grouped by body
  const int* mask_u; int n_mask_u;
  const int* mask_v; int n_mask_v;
  int body_u_start[PCFD_MAX_BODIES_DEV + 1];
  int body_v_start[PCFD_MAX_BODIES_DEV + 1];
  int n_bodies;                      // 0: one total only
  int has_outlet;
  double area;                       // cell area dx*dy
  // stretched mesh: the packed metrics (nullptr when uniform), the grid, and the
  // summed widths of the outlet walls' faces (pycfd/core/boundary.py:480-483)
  const double* met;
  int nx, ny;
  double outlet_width;
};

struct LineRef {
  double* a;
  long W;        // row width of the array
  int axis;      // 0: row a[idx, :] of length W; 1: column a[:, idx] of length H
  int H;
  __device__ __forceinline__ int len() const { return axis == 0 ? (int)W : H; }
  __device__ __forceinline__ double& at(int idx, int k) const {
    return axis == 0 ? a[(long)idx * W + k] : a[(long)k * W + idx];
  }
};

// Sum over the block (thread 0 holds the result; all threads get it back).
__device__ __forceinline__ double block_sum_bcast(double v) {
  double t[1] = {v};
  block_reduce<1>(t);
  __shared__ double out;
  if (threadIdx.x == 0) out = t[0];
  __syncthreads();
  const double r = out;
  __syncthreads();
  return r;
}

__device__ void bc_velocity(double* u, double* v, const Geo& g, const BcTable& T, bool predictor) {
  const int nx = g.nx, ny = g.ny;
  const long WU = ny + 2, WV = ny + 3;
  for (int w = 0; w < 4; ++w) {
    const int kind = T.kind[w];
    if (kind == BC_PERIODIC) continue;
    const int axis = w < 2 ? 0 : 1;
    const bool low = (w == W_LEFT || w == W_BOTTOM);
    const int nlast = axis == 0 ? nx : ny;
    const int n_face = low ? 1 : nlast + 1, n_in = low ? 2 : nlast, n_ghost = low ? 0 : nlast + 2;
    const int t_ghost = low ? 0 : nlast + 1, t_in = low ? 1 : nlast;
    const double outward = low ? -1.0 : 1.0;
    // normal = u for left/right, v for bottom/top
    const LineRef nrm = axis == 0 ? LineRef{u, WU, 0, nx + 3} : LineRef{v, WV, 1, nx + 2};
    const LineRef tan = axis == 0 ? LineRef{v, WV, 0, nx + 2} : LineRef{u, WU, 1, nx + 3};
    const bool prescribes = kind != BC_PRESSURE_OUTLET;
    const bool derives = kind == BC_OUTLET;
    if (prescribes && (predictor || !derives)) {
      const int L = nrm.len();
      for (int k = threadIdx.x; k < L; k += blockDim.x) {
        double val = 0.0;
        if (kind == BC_INLET) val = T.profile[w] ? T.profile[w][k] : -outward * T.vel[w];
        else if (kind == BC_OUTLET) val = nrm.at(n_in, k);
        nrm.at(n_face, k) = val;
      }
      __syncthreads();
    }
    {
      const int L = nrm.len();
      for (int k = threadIdx.x; k < L; k += blockDim.x) {
        const double f = nrm.at(n_face, k);
        nrm.at(n_ghost, k) = (kind == BC_PRESSURE_OUTLET) ? f : 2.0 * f - nrm.at(n_in, k);
      }
      const int LT = tan.len();
      for (int k = threadIdx.x; k < LT; k += blockDim.x) {
        const double ti = tan.at(t_in, k);
        double val;
        if (kind == BC_MOVING_WALL) val = 2.0 * T.vel[w] - ti;
        else if (kind == BC_OUTLET || kind == BC_PRESSURE_OUTLET || kind == BC_SYMMETRY) val = ti;
        else val = -ti;
        tan.at(t_ghost, k) = val;
      }
      __syncthreads();
    }
  }
  // periodic wrap (pycfd/core/boundary.py:388-410)
  if (g.periodic_x) {
    for (int k = threadIdx.x; k < ny + 2; k += blockDim.x) {
      u[(long)(nx + 1) * WU + k] = u[WU + k];
      u[k] = u[(long)nx * WU + k];
      u[(long)(nx + 2) * WU + k] = u[2 * WU + k];
    }
    for (int k = threadIdx.x; k < ny + 3; k += blockDim.x) {
      v[k] = v[(long)nx * WV + k];
      v[(long)(nx + 1) * WV + k] = v[WV + k];
    }
    __syncthreads();
  }
  if (g.periodic_y) {
    for (int k = threadIdx.x; k < nx + 2; k += blockDim.x) {
      v[(long)k * WV + ny + 1] = v[(long)k * WV + 1];
      v[(long)k * WV] = v[(long)k * WV + ny];
      v[(long)k * WV + ny + 2] = v[(long)k * WV + 2];
    }
    for (int k = threadIdx.x; k < nx + 3; k += blockDim.x) {
      u[(long)k * WU] = u[(long)k * WU + ny];
      u[(long)k * WU + ny + 1] = u[(long)k * WU + 1];
    }
    __syncthreads();
  }
}

// enforce_global_mass_balance (pycfd/core/boundary.py:423-487), uniform mesh.
__device__ void bc_mass_balance(double* u, double* v, const Geo& g, const BcTable& T) {
  const int nx = g.nx, ny = g.ny;
  const long WU = ny + 2, WV = ny + 3;
  double influx = 0.0, outflux = 0.0;
  for (int w = 0; w < 4; ++w) {
    if (T.kind[w] == BC_PERIODIC) continue;
    const int axis = w < 2 ? 0 : 1;
    const bool low = (w == W_LEFT || w == W_BOTTOM);
    const int n_face = low ? 1 : (axis == 0 ? nx : ny) + 1;
    const int n = axis == 0 ? ny : nx;
    double s = 0.0;
    if (g.met) {   // a stretched wall's faces differ in width: sum face * width
      const Metrics M(g);
      for (int k = 1 + threadIdx.x; k <= n; k += blockDim.x)
        s += axis == 0 ? rmul(u[(long)n_face * WU + k], M.hy(k - 1)) : rmul(v[(long)k * WV + n_face], M.hx(k - 1));
    } else {
      for (int k = 1 + threadIdx.x; k <= n; k += blockDim.x)
        s += axis == 0 ? u[(long)n_face * WU + k] : v[(long)k * WV + n_face];
    }
    s = block_sum_bcast(s);
    const double width = axis == 0 ? g.dy : g.dx;
    const double flux_out = (low ? -1.0 : 1.0) * (g.met ? s : rmul(s, width));
    if (T.kind[w] == BC_OUTLET) outflux += flux_out;
    else influx -= flux_out;
  }
  double total = 0.0;
  if (g.met) total = T.outlet_width;
  else
    for (int w = 0; w < 4; ++w)
      if (T.kind[w] == BC_OUTLET) total += rmul((double)(w < 2 ? ny : nx), w < 2 ? g.dy : g.dx);
  const bool scale_mode = outflux > 1.0e-12;
  const double scale = influx / outflux;
  const double deficit = influx - outflux;
  for (int w = 0; w < 4; ++w) {
    if (T.kind[w] != BC_OUTLET) continue;
    const int axis = w < 2 ? 0 : 1;
    const bool low = (w == W_LEFT || w == W_BOTTOM);
    const int n_face = low ? 1 : (axis == 0 ? nx : ny) + 1;
    const int n = axis == 0 ? ny : nx;
    const double add = (low ? -1.0 : 1.0) * deficit / total;
    for (int k = 1 + threadIdx.x; k <= n; k += blockDim.x) {
      double& f = axis == 0 ? u[(long)n_face * WU + k] : v[(long)k * WV + n_face];
      f = scale_mode ? f * scale : f + add;
    }
  }
  __syncthreads();
}

// The momentum a masked face carries per unit of the uniform cell area (uniform
// mesh: the face value; the sum is scaled by the area after the reduction), or
// weighted by its control volume on a stretched mesh: hxu[m-1] hy[j-1] behind
// u face (m, j), hx[i-1] hyv[n-1] behind v face (i, n)
// (pycfd/core/solver.py:265-274, :198-207).
__device__ __forceinline__ double bc_momentum_u(const double* u, const BcTable& T, int idx) {
  if (!T.met) return u[idx];
  const int W = T.ny + 2, m = idx / W, j = idx - m * W;
  const double* p = T.met;
  const int nx = T.nx, ny = T.ny;
  const double area = rmul(p[nx + ny + (m - 1)], p[nx + (j - 1)]);   // hxu[m-1] * hy[j-1]
  return rmul(u[idx], area);
}
__device__ __forceinline__ double bc_momentum_v(const double* v, const BcTable& T, int idx) {
  if (!T.met) return v[idx];
  const int W = T.ny + 3, i = idx / W, n = idx - i * W;
  const double* p = T.met;
  const int nx = T.nx, ny = T.ny;
  const double area = rmul(p[i - 1], p[2 * nx + ny + 1 + (n - 1)]);   // hx[i-1] * hyv[n-1]
  return rmul(v[idx], area);
}

// Direct forcing (pycfd/core/solver.py:553-599): sum the masked faces for the
// reaction force (when dt is given), then zero them.  Body b owns the list
// entries [body_*_start[b], body_*_start[b+1]).
__device__ void bc_mask(double* u, double* v, const BcTable& T, double* S, int mode) {
  if (mode != OP_MASK_NONE) {
    const double dt = S[S_DT];
    double su = 0.0, sv = 0.0;
    for (int k = threadIdx.x; k < T.n_mask_u; k += blockDim.x) su += bc_momentum_u(u, T, T.mask_u[k]);
    for (int k = threadIdx.x; k < T.n_mask_v; k += blockDim.x) sv += bc_momentum_v(v, T, T.mask_v[k]);
    su = block_sum_bcast(su);
    sv = block_sum_bcast(sv);
    if (threadIdx.x == 0) {
      const double fx = T.met ? su / dt : su * T.area / dt, fy = T.met ? sv / dt : sv * T.area / dt;
      if (mode == OP_MASK_RESET) { S[S_FX] = fx; S[S_FY] = fy; }
      else { S[S_FX] += fx; S[S_FY] += fy; }
    }
    for (int b = 0; b < T.n_bodies; ++b) {
      double bu = 0.0, bv = 0.0;
      for (int k = T.body_u_start[b] + threadIdx.x; k < T.body_u_start[b + 1]; k += blockDim.x)
        bu += bc_momentum_u(u, T, T.mask_u[k]);
      for (int k = T.body_v_start[b] + threadIdx.x; k < T.body_v_start[b + 1]; k += blockDim.x)
        bv += bc_momentum_v(v, T, T.mask_v[k]);
      bu = block_sum_bcast(bu);
      bv = block_sum_bcast(bv);
      if (threadIdx.x == 0) {
        const double fx = T.met ? bu / dt : bu * T.area / dt, fy = T.met ? bv / dt : bv * T.area / dt;
        if (mode == OP_MASK_RESET) { S[S_BODY_FX + b] = fx; S[S_BODY_FY + b] = fy; }
        else { S[S_BODY_FX + b] += fx; S[S_BODY_FY + b] += fy; }
      }
    }
    __syncthreads();
  }
  for (int k = threadIdx.x; k < T.n_mask_u; k += blockDim.x) u[T.mask_u[k]] = 0.0;
  for (int k = threadIdx.x; k < T.n_mask_v; k += blockDim.x) v[T.mask_v[k]] = 0.0;
  __syncthreads();
}

// pycfd/core/solver.py:601-607
__device__ void bc_wrap_faces(double* u, double* v, const Geo& g) {
  const int nx = g.nx, ny = g.ny;
  const long WU = ny + 2, WV = ny + 3;
  if (g.periodic_x)
    for (int k = threadIdx.x; k < ny + 2; k += blockDim.x) u[(long)(nx + 1) * WU + k] = u[WU + k];
  if (g.periodic_y)
    for (int k = threadIdx.x; k < nx + 2; k += blockDim.x) v[(long)k * WV + ny + 1] = v[(long)k * WV + 1];
  __syncthreads();
}

__global__ void __launch_bounds__(1024) k_boundary(double* u, double* v, Geo g, BcTable T,
                                                   BcProgram prog, double* S) {
  pdl_begin();
  for (int s = 0; s < 8 && prog.op[s] != OP_END; ++s) {
    switch (prog.op[s]) {
      case OP_VEL_PRED: bc_velocity(u, v, g, T, true); break;
      case OP_VEL_CORR: bc_velocity(u, v, g, T, false); break;
      case OP_MASS: if (T.has_outlet) bc_mass_balance(u, v, g, T); break;
      case OP_MASK_NONE:
      case OP_MASK_RESET:
      case OP_MASK_ACC: if (T.n_mask_u + T.n_mask_v > 0) bc_mask(u, v, T, S, prog.op[s]); break;
      case OP_WRAP_FACES: bc_wrap_faces(u, v, g); break;
      default: break;
    }
  }
}

}  // namespace pcfd
