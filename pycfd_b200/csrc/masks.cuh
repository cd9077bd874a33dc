// Immersed bodies rasterised on the device (pycfd/geometry/obstacles.py:87-367).
// The solid fraction of a cell is the mean of an S x S midpoint supersample of
// the body's inside test; a cell with fraction > 0.5 is solid.  One thread per
// cell counts its S*S hits, so the fraction (hits / S^2) is exact, and the
// sample coordinates X = xf[i] + ((a + 0.5) / S) * dx[i] are formed from the
// mesh's own face coordinates with the reference's operations in its order
// (this translation unit has FMA contraction off), so masks and fractions are
// bit-identical to the reference's.
#pragma once
#include "common.cuh"

namespace pcfd {

enum : int { SH_CIRCLE = 0, SH_RECTANGLE = 1, SH_POLYGON = 2, SH_IMAGE = 3 };

struct ShapeDev {
  int kind;
  double p0, p1, p2, p3;      // circle: cx, cy, r; rectangle: x0, y0, x1, y1; polygon: bounding box
  const double* verts;        // polygon: n_verts (x, y) pairs, closed implicitly
  int n_verts;
  const double* image;        // image: rows x cols luminance, row 0 at y = 0
  int rows, cols;
  double lx, ly, threshold;
  int invert;
};

// Inside test of one sample point, each shape as the reference writes it.
__device__ __forceinline__ bool shape_inside(const ShapeDev& s, double X, double Y) {
  switch (s.kind) {
    case SH_CIRCLE: {
      const double ax = X - s.p0, ay = Y - s.p1;
      return rmul(ax, ax) + rmul(ay, ay) <= rmul(s.p2, s.p2);
    }
    case SH_RECTANGLE:
      return (X >= s.p0) && (X <= s.p2) && (Y >= s.p1) && (Y <= s.p3);
    case SH_POLYGON: {
      // bounding-box pre-filter, then the even-odd count of crossings of a ray towards +x
      if (!(X >= s.p0 && X <= s.p2 && Y >= s.p1 && Y <= s.p3)) return false;
      bool hit = false;
      for (int e = 0; e < s.n_verts; ++e) {
        const int f = e + 1 < s.n_verts ? e + 1 : 0;
        const double x0 = s.verts[2 * e], y0 = s.verts[2 * e + 1];
        const double x1 = s.verts[2 * f], y1 = s.verts[2 * f + 1];
        if ((y0 > Y) != (y1 > Y)) {
          const double xc = x0 + (Y - y0) * (x1 - x0) / (y1 - y0);
          if (X < xc) hit = !hit;
        }
      }
      return hit;
    }
    default: {   // SH_IMAGE: the pixel under the sample, dark (below threshold) = solid
      int col = (int)(X / s.lx * (double)s.cols);
      int row = (int)(Y / s.ly * (double)s.rows);
      col = col < 0 ? 0 : (col > s.cols - 1 ? s.cols - 1 : col);
      row = row < 0 ? 0 : (row > s.rows - 1 ? s.rows - 1 : row);
      const bool solid = s.image[(long)row * s.cols + col] < s.threshold;
      return s.invert ? !solid : solid;
    }
  }
}

__global__ void k_solid_fraction(ShapeDev s, const double* __restrict__ xf, const double* __restrict__ dxc,
                                 const double* __restrict__ yf, const double* __restrict__ dyc, int nx, int ny,
                                 int S, double* __restrict__ frac, uint8_t* __restrict__ mask) {
  const long n = (long)nx * ny;
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
    const int i = (int)(c / ny), j = (int)(c - (long)i * ny);
    const double x0 = xf[i], hx = dxc[i], y0 = yf[j], hy = dyc[j];
    int hits = 0;
    for (int a = 0; a < S; ++a) {
      const double X = x0 + rmul(((double)a + 0.5) / (double)S, hx);
      for (int b = 0; b < S; ++b) {
        const double Y = y0 + rmul(((double)b + 0.5) / (double)S, hy);
        hits += shape_inside(s, X, Y) ? 1 : 0;
      }
    }
    const double f = (double)hits / (double)(S * S);
    frac[c] = f;
    mask[c] = f > 0.5 ? 1 : 0;
  }
}

}  // namespace pcfd
