// V-cycle kernels of the smoothed-aggregation multigrid
// (pycfd/core/multigrid.py:424-474, :524-543).
//
// Level 0 is applied matrix-free from the cell flags.  Coarse operators, the
// prolongators P_l and the restrictions R_l = P_l^T are ELLPACK blocks; a row
// is handled by L lanes (L = 1 for the narrow fine-side stencils, up to 32 for
// the wide Galerkin stencils of the coarse levels, whose rows reach 500
// entries).  With L = 1 the entries are column-major so neighbouring rows
// coalesce; with L > 1 a row's entries are contiguous so its lanes coalesce.
// Damped-Jacobi smoothing is x += wdinv*(b - A x); from a zero start the first
// sweep is the pointwise x = wdinv*b, fused with the residual that follows.
#pragma once
#include <cooperative_groups.h>

#include "common.cuh"

namespace pcfd {

template <class T>
struct Ell {
  const int* col;
  const T* val;
  int n;          // rows
  int K;          // stored entries per row
  int rowmajor;   // 1: [row*K + k], 0: [k*n + row]
};

// Per-phase ELL passes (blockDim 256).  A row's entries are split over L
// lanes -- L <= 32: a group within a warp, combined by shuffles; L > 32: L/32
// warps, their sums combined in shared memory in warp order.  A lane gathers
// its entries kEllGather at a time (indices and values, then the vector
// values, then the products added in entry order), so several gathers are in
// flight.  Rows past the end contribute nothing; every thread of a block runs
// the same rounds (the shuffles and the block barrier need them all).
constexpr int kEllGather = 4;

template <int L, class T, class X>
__device__ __forceinline__ double ell_lane_sum(const Ell<T>& E, int row, int lane, X x) {
  double acc = 0.0;
  if (row >= E.n) return acc;
  for (int k0 = lane; k0 < E.K; k0 += kEllGather * L) {
    int cc[kEllGather];
    T vv[kEllGather];
#pragma unroll
    for (int u = 0; u < kEllGather; ++u) {
      const int k = k0 + u * L;
      cc[u] = 0;
      vv[u] = (T)0;
      if (k < E.K) {
        const long e = E.rowmajor ? (long)row * E.K + k : (long)k * E.n + row;
        cc[u] = __ldg(E.col + e);
        vv[u] = __ldg(E.val + e);
      }
    }
    double xx[kEllGather];
#pragma unroll
    for (int u = 0; u < kEllGather; ++u) xx[u] = (k0 + u * L < E.K) ? x(cc[u]) : 0.0;
#pragma unroll
    for (int u = 0; u < kEllGather; ++u)
      if (k0 + u * L < E.K) acc += (double)vv[u] * xx[u];
  }
  return acc;
}

template <int L, class T, class X, class W>
__device__ __forceinline__ void ell_pass(const Ell<T>& E, X x, W write) {
  static_assert(L >= 1 && L <= 256 && (L & (L - 1)) == 0, "lanes per row: a power of two up to 256");
  if constexpr (L <= 32) {
    const int lane = (int)(threadIdx.x % L);
    const int per = (int)(gridDim.x * blockDim.x / L);
    for (int base = (int)(blockIdx.x * blockDim.x / L); base < E.n; base += per) {
      const int row = base + (int)(threadIdx.x / L);
      double acc = ell_lane_sum<L>(E, row, lane, x);
#pragma unroll
      for (int o = L / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o, L);
      if (lane == 0 && row < E.n) write(row, acc);
    }
  } else {
    constexpr int kW = L / 32;              // warps per row
    constexpr int kRows = 256 / L;          // rows per block and round
    __shared__ double part[8];
    const int warp = (int)(threadIdx.x >> 5), wl = (int)(threadIdx.x & 31);
    const int lane = (int)(threadIdx.x % L), rloc = (int)(threadIdx.x / L);
    for (int base = (int)blockIdx.x * kRows; base < E.n; base += (int)gridDim.x * kRows) {
      const int row = base + rloc;
      const double acc = warp_sum(ell_lane_sum<L>(E, row, lane, x));
      if (wl == 0) part[warp] = acc;
      __syncthreads();
      if (lane == 0 && row < E.n) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < kW; ++w) t += part[warp + w];
        write(row, t);
      }
      __syncthreads();
    }
  }
}

// x = wd*b; res = b - A(wd*b)          (first sweep from zero + residual)
template <int L, class T>
__global__ void k_ell_pre(Ell<T> A, const T* __restrict__ wd, const T* __restrict__ b,
                          T* __restrict__ x, T* __restrict__ res) {
  pdl_begin();
  ell_pass<L>(A, [&](int c) { return (double)wd[c] * (double)b[c]; }, [&](int row, double s) {
    const double bx = (double)b[row];
    x[row] = (T)((double)wd[row] * bx);
    res[row] = (T)(bx - s);
  });
}

// xo = x + wd*(b - A x)
template <int L, class T>
__global__ void k_ell_smooth(Ell<T> A, const T* __restrict__ wd, const T* __restrict__ b,
                             const T* __restrict__ x, T* __restrict__ xo) {
  pdl_begin();
  ell_pass<L>(A, [&](int c) { return (double)x[c]; }, [&](int row, double s) {
    xo[row] = (T)((double)x[row] + (double)wd[row] * ((double)b[row] - s));
  });
}

// res = b - A x
template <int L, class T>
__global__ void k_ell_resid(Ell<T> A, const T* __restrict__ b, const T* __restrict__ x,
                            T* __restrict__ res) {
  pdl_begin();
  ell_pass<L>(A, [&](int c) { return (double)x[c]; },
              [&](int row, double s) { res[row] = (T)((double)b[row] - s); });
}

// y = M x (restriction with M = R), or y += M x (prolongation with M = P).
template <int L, bool ADD, class T>
__global__ void k_ell_spmv(Ell<T> M, const T* __restrict__ x, T* __restrict__ y) {
  pdl_begin();
  ell_pass<L>(M, [&](int c) { return (double)x[c]; },
              [&](int row, double s) { y[row] = ADD ? (T)((double)y[row] + s) : (T)s; });
}

// Coarsest level: x = C b with C the precomputed pseudo-inverse (pinned LU
// followed by mean removal, pycfd/core/multigrid.py:524-543), column-major.
// One warp per row of C (row-major), lanes over its columns.
template <class T>
__global__ void k_dense(const T* __restrict__ C, int n, const T* __restrict__ b, T* __restrict__ x) {
  pdl_begin();
  const int lane = threadIdx.x & 31;
  for (int row = threadIdx.x >> 5; row < n; row += blockDim.x >> 5) {
    double acc = 0.0;
    for (int k = lane; k < n; k += 32) acc += (double)C[(long)row * n + k] * (double)b[k];
    acc = warp_sum(acc);
    if (lane == 0) x[row] = (T)acc;
  }
}

// Restriction into the coarsest level and its dense solve in one block:
// b = R res (rows n <= a few hundred, one warp per row), then x = C b.
template <class T>
__global__ void k_restrict_dense(Ell<T> R, int L, const T* __restrict__ res, const T* __restrict__ C,
                                 T* __restrict__ b, T* __restrict__ x) {
  pdl_begin();
  extern __shared__ double sb[];
  // restriction: L lanes per row, the same partial-sum order as the ELL kernels
  const int lane = threadIdx.x % L, per = blockDim.x / L;
  for (int base = 0; base < R.n; base += per) {
    const int row = base + threadIdx.x / L;
    double acc = 0.0;
    if (row < R.n) {
      if (R.rowmajor) {
        const long o = (long)row * R.K;
        for (int k = lane; k < R.K; k += L) acc += (double)R.val[o + k] * (double)res[R.col[o + k]];
      } else {
        for (int k = lane; k < R.K; k += L) {
          const long e = (long)k * R.n + row;
          acc += (double)R.val[e] * (double)res[R.col[e]];
        }
      }
    }
    for (int s = L >> 1; s > 0; s >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, s, L);
    if (lane == 0 && row < R.n) {
      sb[row] = (double)(T)acc;
      b[row] = (T)acc;
    }
  }
  __syncthreads();
  // dense solve: one warp per row
  const int wl = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int n = R.n;
  for (int row = warp; row < n; row += nw) {
    double acc = 0.0;
    for (int k = wl; k < n; k += 32) acc += (double)C[(long)row * n + k] * sb[k];
    acc = warp_sum(acc);
    if (wl == 0) x[row] = (T)acc;
  }
}

// Dense close of the V-cycle: x = M b, M (row-major n x n) the cycle's map at
// and below one level (the host builds it from the hierarchy).  kTailWarps
// warps per row, their lanes striding the columns eight loads at a time; the
// warps' sums are added in warp order.  256-thread blocks, two rows each.
constexpr int kTailWarps = 4;
constexpr int kTailRowsPerBlock = 256 / 32 / kTailWarps;
template <class T>
__global__ void __launch_bounds__(256) k_tail(const T* __restrict__ M, int n, const T* __restrict__ b,
                                              T* __restrict__ x) {
  pdl_begin();
  __shared__ double part[8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.x * kTailRowsPerBlock + warp / kTailWarps;
  const int w = warp % kTailWarps;
  double acc = 0.0;
  if (row < n) {
    const T* m = M + (long)row * n;
    constexpr int stride = 32 * kTailWarps;
    for (int k0 = w * 32 + lane; k0 < n; k0 += 8 * stride) {
      T mm[8], bb[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int k = k0 + u * stride;
        mm[u] = k < n ? __ldg(m + k) : (T)0;
        bb[u] = k < n ? b[k] : (T)0;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) acc += (double)mm[u] * (double)bb[u];
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
}

// ---- level 0 (matrix-free) --------------------------------------------------
// Right-hand side of the fine level: the CG residual projected onto the
// active set (multigrid.py:453-458), or a stored vector.
template <class T>
struct BFromR {
  const T* r;
  const uint8_t* f;
  double mean;
  __device__ __forceinline__ void load() {}
  __device__ __forceinline__ double operator()(int k) const {
    return (f[k] & F_SOLV) ? (double)r[k] - mean : 0.0;
  }
};
// Same projection with the mean read from the device scalars at kernel start.
template <class T>
struct BFromRS {
  const T* r;
  const uint8_t* f;
  const double* S;
  int singular;
  double mean;
  __device__ __forceinline__ void load() { mean = singular ? S[S_MEAN_R] : 0.0; }
  __device__ __forceinline__ double operator()(int k) const {
    return (f[k] & F_SOLV) ? (double)r[k] - mean : 0.0;
  }
};

template <class T>
struct BStored {
  __device__ __forceinline__ void load() {}
  const T* b;
  __device__ __forceinline__ double operator()(int k) const { return (double)b[k]; }
};

__device__ __forceinline__ double fine_wdinv(uint8_t f, int i, int j, const Geo& g, double w) {
  return w * (1.0 / fine_diag(f, i, j, g));
}

// ---- fused down sweep (one sweep per level, from zero) ------------------------
// b_l = M_l b_{l-1} with M_l = R_l (I - A_{l-1} W_{l-1}): the first sweep on
// level l-1 and the restriction of its residual in one pass.  From level 0 the
// right-hand side is the projected CG residual (bf).
template <int L, class T, class B>
__global__ void k_ell_fused_restrict0(Ell<T> M, B bf, T* __restrict__ y) {
  pdl_begin();
  bf.load();
  ell_pass<L>(M, [&](int c) { return bf(c); }, [&](int row, double s) { y[row] = (T)s; });
}

// Up sweep after a fused down sweep: the level's first-sweep iterate W b was
// not stored, so the prolongation forms it on the fly -- x = (T)(W b), then
// x + P x_c, the same two roundings as the stored form.
template <int L, class T>
__global__ void k_ell_prolong_wb(Ell<T> P, const T* __restrict__ wd, const T* __restrict__ b,
                                 const T* __restrict__ xc, T* __restrict__ xf) {
  pdl_begin();
  ell_pass<L>(P, [&](int c) { return (double)xc[c]; }, [&](int row, double s) {
    xf[row] = (T)((double)(T)((double)wd[row] * (double)b[row]) + s);
  });
}

// The same onto level 0, whose W b is fine_wdinv * (projected residual).
template <int L, class T, class B>
__global__ void k_ell_prolong0_wb(Ell<T> P, B bf, const uint8_t* __restrict__ flags, Geo g, double w,
                                  const T* __restrict__ xc, T* __restrict__ xf) {
  pdl_begin();
  bf.load();
  ell_pass<L>(P, [&](int c) { return (double)xc[c]; }, [&](int row, double s) {
    const int i = row / g.ny, j = row - i * g.ny;
    xf[row] = (T)((double)(T)(fine_wdinv(flags[row], i, j, g, w) * bf(row)) + s);
  });
}

// x = wd*b and res = b - A(wd*b) on level 0.
template <class T, class B>
__global__ void k_fine_pre(B bf, const uint8_t* __restrict__ flags, Geo g, double w,
                           T* __restrict__ x, T* __restrict__ res) {
  pdl_begin();
  bf.load();
  auto xv = [&](int k, int ii, int jj) -> double {
    return (double)(T)(fine_wdinv(flags[k], ii, jj, g, w) * bf(k));
  };
  uint8_t fv[kStripRows];
  double bv[kStripRows];
  strip_cells<true>(g, xv, [&](int u, int c) { fv[u] = flags[c]; bv[u] = bf(c); },
                    [&](int u, int c, int i, int j, double xc, double xw, double xe, double xs, double xn) {
                      x[c] = (T)xc;
                      res[c] = (T)(bv[u] - fine_apply5(fv[u], i, j, g, xc, xw, xe, xs, xn));
                    });
}

// xo = x + wd*(b - A x) on level 0.  MODE 0: plain; MODE 1: last sweep of the
// preconditioner, with sum_solvable(xo) and r.xo for the projected z and
// rho = r.z (r = CG residual, rsum = its solvable sum); MODE 2: last sweep of
// a standalone cycle, with sum_solvable(xo) for the projection.
template <class T, class B, int MODE>
__global__ void k_fine_smooth(B bf, const uint8_t* __restrict__ flags, Geo g, double w,
                              const T* __restrict__ x, T* __restrict__ xo,
                              const T* __restrict__ rcg, int singular, double* __restrict__ S,
                              RedBuf rb) {
  pdl_begin();
  bf.load();
  auto xv = [&](int k, int, int) -> double { return (double)x[k]; };
  double acc[2] = {0, 0};
  uint8_t fv[kStripRows];
  double bv[kStripRows], rv[kStripRows];
  strip_cells<true>(g, xv,
                    [&](int u, int c) {
                      fv[u] = flags[c];
                      bv[u] = bf(c);
                      if (MODE == 1) rv[u] = (double)rcg[c];
                    },
                    [&](int u, int c, int i, int j, double xc, double xw, double xe, double xs, double xn_) {
                      const uint8_t f = fv[u];
                      const double xn = (double)(T)(xc + fine_wdinv(f, i, j, g, w) *
                                                    (bv[u] - fine_apply5(f, i, j, g, xc, xw, xe, xs, xn_)));
                      xo[c] = (T)xn;
                      if (MODE != 0 && (f & F_SOLV)) {
                        acc[0] += xn;
                        if (MODE == 1) acc[1] += rv[u] * xn;
                      }
                    });
  if (MODE == 0) return;
  grid_reduce<2>(acc, rb, [&](double* t) {
    const double m = (singular && g.n_fluid) ? t[0] / g.n_fluid : 0.0;
    if (MODE == 1) {
      S[S_MEAN_Z] = m;
      S[S_RHO_PREV] = S[S_RHO];
      S[S_RHO] = t[1] - m * S[S_SUM_R];
    } else {
      S[S_MEAN_X] = m;
    }
  });
}

// res = b - A x on level 0.
template <class T, class B>
__global__ void k_fine_resid(B bf, const uint8_t* __restrict__ flags, Geo g,
                             const T* __restrict__ x, T* __restrict__ res) {
  pdl_begin();
  bf.load();
  auto xv = [&](int k, int, int) -> double { return (double)x[k]; };
  uint8_t fv[kStripRows];
  double bv[kStripRows];
  strip_cells<true>(g, xv, [&](int u, int c) { fv[u] = flags[c]; bv[u] = bf(c); },
                    [&](int u, int c, int i, int j, double xc, double xw, double xe, double xs, double xn) {
                      res[c] = (T)(bv[u] - fine_apply5(fv[u], i, j, g, xc, xw, xe, xs, xn));
                    });
}

// x = wd*b on level 0 (first sweep from zero when more sweeps follow).
template <class T, class B>
__global__ void k_fine_wdb(B bf, const uint8_t* __restrict__ flags, Geo g, double w,
                           T* __restrict__ x) {
  pdl_begin();
  bf.load();
  FOR_CELLS(g) {
    const int c = i * g.ny + j;
    x[c] = (T)(fine_wdinv(flags[c], i, j, g, w) * bf(c));
  }
}

// Materialise a fine right-hand side (single-level hierarchies only).
template <class T, class B>
__global__ void k_fine_store(B bf, Geo g, T* __restrict__ out) {
  pdl_begin();
  FOR_CELLS(g) {
    const int c = i * g.ny + j;
    out[c] = (T)bf(c);
  }
}

// Fine-level sums after a single-level "cycle" (dense solve): same finisher as
// k_fine_smooth MODE 1/2 without the smoothing.
template <class T, int MODE>
__global__ void k_fine_sums(const T* __restrict__ x, const uint8_t* __restrict__ flags, Geo g,
                            const T* __restrict__ rcg, int singular, double* __restrict__ S,
                            RedBuf rb) {
  pdl_begin();
  double acc[2] = {0, 0};
  FOR_CELLS(g) {
    const int c = i * g.ny + j;
    if (flags[c] & F_SOLV) {
      acc[0] += (double)x[c];
      if (MODE == 1) acc[1] += (double)rcg[c] * (double)x[c];
    }
  }
  grid_reduce<2>(acc, rb, [&](double* t) {
    const double m = (singular && g.n_fluid) ? t[0] / g.n_fluid : 0.0;
    if (MODE == 1) {
      S[S_MEAN_Z] = m;
      S[S_RHO_PREV] = S[S_RHO];
      S[S_RHO] = t[1] - m * S[S_SUM_R];
    } else {
      S[S_MEAN_X] = m;
    }
  });
}

// Materialise the projected fine right-hand side of the preconditioner from
// the CG residual r (pycfd/core/multigrid.py:453-458, 468-469).
template <class T>
__global__ void k_fine_store_from_r(const T* __restrict__ r, const uint8_t* __restrict__ flags, Geo g,
                                    const double* __restrict__ S, int singular, T* __restrict__ out) {
  pdl_begin();
  const double m = singular ? S[S_MEAN_R] : 0.0;
  FOR_CELLS(g) {
    const int c = i * g.ny + j;
    out[c] = (flags[c] & F_SOLV) ? (T)((double)r[c] - m) : (T)0;
  }
}

// ---- coarse levels in one thread-block cluster ------------------------------
// The coarse levels of a V-cycle hold few rows (<= ~16K) but wide Galerkin
// stencils; as separate kernels each phase is launch- and latency-bound.  Here
// one cluster of up to 16 CTAs runs every coarse phase -- restriction, first
// smoothing sweep + residual, coarsest dense solve, prolongation, smoothing --
// separated by hardware cluster barriers (no spin loops: every thread reaches
// the same barriers, and the CTAs of a cluster are co-scheduled).  Vectors
// written inside the kernel are read through L2 (ld.global.cg), never a stale L1.
constexpr int kMaxCLevels = 12;

template <class T>
struct CLevel {
  Ell<T> A, R, P;      // A, R: rows of this level; P: prolongation into the finer level
  int la, lr, lp;      // lanes per row of each block
  const T* wd;
  T *b, *xa, *xb, *res;
};

template <class T>
struct CTable {
  CLevel<T> lv[kMaxCLevels];
  int nlev;            // lv[0] is the first cluster level, lv[nlev-1] the coarsest
  const T* res_in;     // residual of the level above lv[0]
  const T* C;          // coarsest pseudo-inverse, row-major nc x nc
  int nc;
  int sweeps;
};

template <class T>
__device__ __forceinline__ double ldcg(const T* p) { return (double)__ldcg(p); }

// One ELL pass over all rows, distributed over the cluster's threads, L lanes
// per row (runtime).  Every thread runs the same number of rounds.
template <class T, class X, class W>
__device__ __forceinline__ void cl_ell(const Ell<T>& E, int L, int gtid, int nthr, X x, W write) {
  const int per = nthr / L;
  const int lane = gtid % L, r0 = gtid / L;
  for (int base = 0; base < E.n; base += per) {
    const int row = base + r0;
    double acc = 0.0;
    if (row < E.n) {
      if (E.rowmajor) {
        const long o = (long)row * E.K;
        for (int k = lane; k < E.K; k += L) acc += (double)E.val[o + k] * x(E.col[o + k]);
      } else {
        for (int k = lane; k < E.K; k += L) {
          const long e = (long)k * E.n + row;
          acc += (double)E.val[e] * x(E.col[e]);
        }
      }
    }
    for (int s = L >> 1; s > 0; s >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, s, L);
    if (lane == 0 && row < E.n) write(row, acc);
  }
}

template <class T>
__global__ void __launch_bounds__(1024) k_coarse_cycle(CTable<T> t) {
  pdl_begin();
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int nthr = (int)(blockDim.x * cl.num_blocks());
  const int gtid = (int)(cl.block_rank() * blockDim.x + threadIdx.x);
  T* cur[kMaxCLevels];
  // ---- down: restrict, first sweep from zero + residual (more sweeps if asked)
  for (int l = 0; l < t.nlev; ++l) {
    const CLevel<T>& L = t.lv[l];
    const T* src = (l == 0) ? t.res_in : t.lv[l - 1].res;
    cl_ell(L.R, L.lr, gtid, nthr, [&](int c) { return ldcg(src + c); },
           [&](int row, double s) { L.b[row] = (T)s; });
    cl.sync();
    if (l == t.nlev - 1) {   // coarsest: x = C b, one warp per row
      const int lane = gtid & 31;
      for (int row = gtid >> 5; row < t.nc; row += nthr >> 5) {   // uniform within a warp
        double acc = 0.0;
        for (int k = lane; k < t.nc; k += 32) acc += (double)t.C[(long)row * t.nc + k] * ldcg(L.b + k);
        acc = warp_sum(acc);
        if (lane == 0) L.xa[row] = (T)acc;
      }
      cur[l] = L.xa;
      cl.sync();
      break;
    }
    cl_ell(L.A, L.la, gtid, nthr, [&](int c) { return (double)L.wd[c] * ldcg(L.b + c); },
           [&](int row, double s) {
             const double bx = ldcg(L.b + row);
             L.xa[row] = (T)((double)L.wd[row] * bx);
             L.res[row] = (T)(bx - s);
           });
    cl.sync();
    T* a = L.xa;
    T* o = L.xb;
    if (t.sweeps > 1) {
      for (int k = 1; k < t.sweeps; ++k) {
        cl_ell(L.A, L.la, gtid, nthr, [&](int c) { return ldcg(a + c); },
               [&](int row, double s) {
                 o[row] = (T)(ldcg(a + row) + (double)L.wd[row] * (ldcg(L.b + row) - s));
               });
        cl.sync();
        T* tmp = a; a = o; o = tmp;
      }
      cl_ell(L.A, L.la, gtid, nthr, [&](int c) { return ldcg(a + c); },
             [&](int row, double s) { L.res[row] = (T)(ldcg(L.b + row) - s); });
      cl.sync();
    }
    cur[l] = a;
  }
  // ---- up: prolong, smooth
  for (int l = t.nlev - 2; l >= 0; --l) {
    const CLevel<T>& L = t.lv[l];
    const CLevel<T>& Lc = t.lv[l + 1];
    T* xf = cur[l];
    const T* xc = cur[l + 1];
    cl_ell(Lc.P, Lc.lp, gtid, nthr, [&](int c) { return ldcg(xc + c); },
           [&](int row, double s) { xf[row] = (T)(ldcg(xf + row) + s); });
    cl.sync();
    T* o = (xf == L.xa) ? L.xb : L.xa;
    for (int k = 0; k < t.sweeps; ++k) {
      cl_ell(L.A, L.la, gtid, nthr, [&](int c) { return ldcg(xf + c); },
             [&](int row, double s) {
               o[row] = (T)(ldcg(xf + row) + (double)L.wd[row] * (ldcg(L.b + row) - s));
             });
      cl.sync();
      T* tmp = xf; xf = o; o = tmp;
    }
    cur[l] = xf;
  }
}

}  // namespace pcfd
