/*
 * or_bathy.h -- still-water-depth functions H(x, y) used by the test configurations.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle). Nothing in the product links this file.
 *
 * The reference solver takes the still depth as a callback
 * (`std::function<double(double,double)> stillDepth`, src/solver/sgn2d.h:57-59) and
 * samples it at the nodes and at the face points (src/solver/sgn2d.cpp:49-83). The
 * test configurations need a handful of concrete depth profiles; this header defines
 * them once, in plain C, so that the oracle restatement (sgn_oracle.c) and the shim
 * around the compiled reference sources (ref_shim.cpp) evaluate bit-identical depths.
 * The product library defines the same profiles in its own host code
 * (csrc/sgnb_setup.cpp); a CPU test checks that the two agree bit for bit.
 *
 * Kinds (parameter vector p[]):
 *   OR_BATHY_NONE      H = 0 everywhere (the reference's empty callback, sgn2d.h:55)
 *   OR_BATHY_CONST     H = p0
 *   OR_BATHY_GAUSS     H = p0 - p1 exp(-((x-p2)^2 + (y-p3)^2) / p4)
 *                      (the bump of test/test_sgn2d.cpp:50-53 is p = {1, 0.4, Lx/2, Ly/2, 6})
 *   OR_BATHY_SHOAL     elliptic shoal on a plane of depth p0: crest depth p1 at
 *                      (p2, p3), semi-axes p4 (x) and p5 (y), profile
 *                      H = p0 - (p0 - p1) (1 - r^2)^3 for r^2 < 1, else p0,
 *                      r^2 = ((x-p2)/p4)^2 + ((y-p3)/p5)^2  (C^2 at the rim)
 *   OR_BATHY_GAUSS_SUM H = p0 - sum_j A_j exp(-((x-x_j)^2 + (y-y_j)^2) / (2 s_j^2)),
 *                      p1 = number of bumps n, then (A_j, x_j, y_j, s_j) for j < n
 *   OR_BATHY_CELLS     piecewise-bilinear interpolant of a grid of cell means:
 *                      p0 = Mx, p1 = My, p2 = Lx, p3 = Ly, then Mx*My means (row-major,
 *                      cell (i, j) at p[4 + i + Mx j]); values are interpolated between
 *                      cell centres with periodic wrap-around. Used to parameterise
 *                      the depth by element means (adjoint configuration).
 */
#ifndef OR_BATHY_H
#define OR_BATHY_H

#include <math.h>

enum {
  OR_BATHY_NONE = 0,
  OR_BATHY_CONST = 1,
  OR_BATHY_GAUSS = 2,
  OR_BATHY_SHOAL = 3,
  OR_BATHY_GAUSS_SUM = 4,
  OR_BATHY_CELLS = 5
};

static inline double or_bathy_eval(int kind, const double* p, double x, double y) {
  switch (kind) {
    case OR_BATHY_CONST:
      return p[0];
    case OR_BATHY_GAUSS: {
      const double dx = x - p[2], dy = y - p[3];
      return p[0] - p[1] * exp(-(dx * dx + dy * dy) / p[4]);
    }
    case OR_BATHY_SHOAL: {
      const double dx = (x - p[2]) / p[4], dy = (y - p[3]) / p[5];
      const double r2 = dx * dx + dy * dy;
      if (r2 >= 1.0) return p[0];
      const double q = 1.0 - r2;
      return p[0] - (p[0] - p[1]) * (q * q * q);
    }
    case OR_BATHY_GAUSS_SUM: {
      const int n = (int)p[1];
      double s = 0.0;
      for (int j = 0; j < n; ++j) {
        const double* b = p + 2 + 4 * j;
        const double dx = x - b[1], dy = y - b[2];
        s += b[0] * exp(-(dx * dx + dy * dy) / (2.0 * b[3] * b[3]));
      }
      return p[0] - s;
    }
    case OR_BATHY_CELLS: {
      const int Mx = (int)p[0], My = (int)p[1];
      const double cx = p[2] / Mx, cy = p[3] / My;
      /* position in cell-centre coordinates */
      const double sx = x / cx - 0.5, sy = y / cy - 0.5;
      const double fx0 = floor(sx), fy0 = floor(sy);
      const double tx = sx - fx0, ty = sy - fy0;
      int i0 = (int)fx0, j0 = (int)fy0;
      int i1 = i0 + 1, j1 = j0 + 1;
      i0 = ((i0 % Mx) + Mx) % Mx; i1 = ((i1 % Mx) + Mx) % Mx;
      j0 = ((j0 % My) + My) % My; j1 = ((j1 % My) + My) % My;
      const double* m = p + 4;
      const double v00 = m[i0 + Mx * j0], v10 = m[i1 + Mx * j0];
      const double v01 = m[i0 + Mx * j1], v11 = m[i1 + Mx * j1];
      const double a = v00 + tx * (v10 - v00);
      const double b = v01 + tx * (v11 - v01);
      return a + ty * (b - a);
    }
    default:
      return 0.0;
  }
}

#endif /* OR_BATHY_H */
