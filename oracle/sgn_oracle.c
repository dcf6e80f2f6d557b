/*
 * sgn_oracle.c -- plain-C restatement of the reference 2D hyperbolic-SGN FR path.
 *
 * TEST INFRASTRUCTURE ONLY: this is the oracle that the CUDA path is checked
 * against. It is never linked into the product library.
 *
 * Every function restates the reference algorithm operation for operation (same
 * expression trees, same summation order), so that compiled without FMA
 * contraction (-ffp-contract=off) it reproduces the reference's doubles bit for bit.
 * Citations are file:line in the reference project (gsalanglada/sgn-hyperbolic-gpu).
 * Parity is pinned by tests/test_oracle.py against the compiled reference sources
 * (_ref/libsgnref.so) and against tests/golden/.
 *
 * Additions the reference lacks, each marked where it appears:
 *   - reflective walls (mirror ghost states), pinned by mirror doubling of the
 *     periodic reference;
 *   - a NaN guard in the adaptive loop (the reference loops forever on a NaN
 *     error norm, src/solver/rk.cpp:129-160);
 *   - an attempt log of the adaptive loop (t, dt, errNorm, accepted).
 */
#include "sgn_oracle.h"
#include "or_bathy.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

enum { NVAR = 5, IH = 0, IHU = 1, IHV = 2, IHW = 3, IHP = 4 };

struct or_ctx {
  int P, np, npp, Nx, Ny, ne;
  int points;  /* OR_POINTS_GLL or OR_POINTS_GAUSS (PointSet, fr_operators.h) */
  long Nd;
  double Lx, Ly, hx, hy, Jx, Jy;
  double g, c, gamma, nManning;
  int bcx, bcy;
  double *xi, *bw, *D, *lL, *lR, *gLp, *gRp, *qw;
  double *Hnod, *Hx, *Hy, *HfaceX, *HfaceY, *HfaceXEnd, *HfaceYEnd;
};

/* ------------------------------------------------------------------------- */
/* FR operators: src/core/fr_operators.cpp                                    */
/* ------------------------------------------------------------------------- */

/* Legendre L_n by the three-term recurrence (fr_operators.cpp:27-37). */
static double leg(int n, double x) {
  if (n == 0) return 1.0;
  if (n == 1) return x;
  double lm1 = 1.0, l = x;
  for (int k = 1; k < n; ++k) {
    const double lp1 = ((2.0 * k + 1.0) * x * l - k * lm1) / (k + 1.0);
    lm1 = l;
    l = lp1;
  }
  return l;
}

/* L_n'(x), closed form at the end points (fr_operators.cpp:40-51). */
static double legd(int n, double x) {
  if (n == 0) return 0.0;
  const double denom = x * x - 1.0;
  if (fabs(denom) < 1e-14) {
    const double s = (x > 0.0) ? 1.0 : ((n - 1) % 2 == 0 ? 1.0 : -1.0);
    return s * 0.5 * n * (n + 1.0);
  }
  return n * (x * leg(n, x) - leg(n - 1, x)) / denom;
}

/* GLL nodes: end points plus Newton roots of L_P' from Chebyshev-Lobatto guesses
 * (fr_operators.cpp:59-81). */
static void gll_nodes(int P, double* x) {
  const double kPi = 3.14159265358979323846;
  if (P == 0) { x[0] = 0.0; return; }
  x[0] = -1.0;
  x[P] = 1.0;
  for (int i = 1; i < P; ++i) {
    double xi = -cos(kPi * i / (double)P);
    for (int it = 0; it < 100; ++it) {
      const double f = legd(P, xi);
      const double fp = (2.0 * xi * legd(P, xi) - P * (P + 1.0) * leg(P, xi)) / (1.0 - xi * xi);
      const double dx = f / fp;
      xi -= dx;
      if (fabs(dx) < 1e-15) break;
    }
    x[i] = xi;
  }
}

/* Gauss-Legendre nodes: the P+1 roots of L_{P+1} by Newton's method from the
 * asymptotic guesses -cos(pi (i + 3/4) / (n + 1/2)) (fr_operators.cpp:86-100). */
static void gauss_nodes(int P, double* x) {
  const double kPi = 3.14159265358979323846;
  const int n = P + 1;
  for (int i = 0; i < n; ++i) {
    double xi = -cos(kPi * (i + 0.75) / (n + 0.5));
    for (int it = 0; it < 100; ++it) {
      const double f = leg(n, xi);
      const double fp = legd(n, xi);
      const double dx = f / fp;
      xi -= dx;
      if (fabs(dx) < 1e-15) break;
    }
    x[i] = xi;
  }
}

/* Lagrange basis j at xq, barycentric form, exact Kronecker delta on a node
 * (fr_operators.cpp:118-127). */
static double lagrange_at(int n, const double* x, const double* w, int j, double xq) {
  for (int k = 0; k < n; ++k)
    if (fabs(xq - x[k]) < 1e-14) return (k == j) ? 1.0 : 0.0;
  const double num = w[j] / (xq - x[j]);
  double den = 0.0;
  for (int k = 0; k < n; ++k) den += w[k] / (xq - x[k]);
  return num / den;
}

/* FROperators1D constructor (fr_operators.cpp:134-200). */
static void build_tables(or_ctx* s) {
  const int P = s->P, n = P + 1;
  if (s->points == OR_POINTS_GAUSS) gauss_nodes(P, s->xi);
  else gll_nodes(P, s->xi);
  /* barycentric weights (fr_operators.cpp:103-113) */
  for (int j = 0; j < n; ++j) {
    double prod = 1.0;
    for (int k = 0; k < n; ++k)
      if (k != j) prod *= (s->xi[j] - s->xi[k]);
    s->bw[j] = 1.0 / prod;
  }
  /* D: off-diagonal barycentric entries, diagonal = minus the row sum (:144-158) */
  for (int i = 0; i < n; ++i) {
    double diag = 0.0;
    for (int j = 0; j < n; ++j) {
      if (i == j) continue;
      const double dij = (s->bw[j] / s->bw[i]) / (s->xi[i] - s->xi[j]);
      s->D[i * n + j] = dij;
      diag -= dij;
    }
    s->D[i * n + i] = diag;
  }
  /* face interpolation rows (:160-166) */
  for (int j = 0; j < n; ++j) {
    s->lL[j] = lagrange_at(n, s->xi, s->bw, j, -1.0);
    s->lR[j] = lagrange_at(n, s->xi, s->bw, j, +1.0);
  }
  /* Huynh g_DG correction derivatives (:168-181) */
  const double signP = (P % 2 == 0) ? 1.0 : -1.0;
  for (int i = 0; i < n; ++i) {
    const double dLP = legd(P, s->xi[i]);
    const double dLP1 = legd(P + 1, s->xi[i]);
    s->gLp[i] = 0.5 * signP * (dLP - dLP1);
    s->gRp[i] = 0.5 * (dLP + dLP1);
  }
  /* quadrature weights (:183-199) */
  if (P == 0) {
    s->qw[0] = 2.0;
  } else if (s->points == OR_POINTS_GAUSS) {
    for (int i = 0; i < n; ++i) {
      const double dLP1 = legd(P + 1, s->xi[i]);
      s->qw[i] = 2.0 / ((1.0 - s->xi[i] * s->xi[i]) * dLP1 * dLP1);
    }
  } else {
    for (int i = 0; i < n; ++i) {
      const double LP = leg(P, s->xi[i]);
      s->qw[i] = 2.0 / (P * (P + 1.0) * LP * LP);
    }
  }
}

/* ------------------------------------------------------------------------- */
/* Pointwise model: src/physics/sgn_flux2d.h                                  */
/* ------------------------------------------------------------------------- */

/* signalSpeed (sgn_flux2d.h:73-78) */
static double signal_speed(const or_ctx* s, const double* U) {
  const double h = U[IH];
  const double p = U[IHP] / h;
  const double arg = s->g * h + p + s->c * s->c;
  return sqrt(arg > 0.0 ? arg : 0.0);
}

/* maxWaveSpeed (sgn_flux2d.h:82-86) */
static double max_wave_speed_pt(const or_ctx* s, const double* U, int dir) {
  const double vn = (dir == 0 ? U[IHU] : U[IHV]) / U[IH];
  return fabs(vn) + signal_speed(s, U);
}

/* fluxX (sgn_flux2d.h:89-101) */
static void flux_x(const or_ctx* s, const double* U, double Hloc, double* F) {
  const double h = U[IH], hu = U[IHU];
  const double u = hu / h, v = U[IHV] / h, w = U[IHW] / h, p = U[IHP] / h;
  const double c2 = s->c * s->c;
  F[IH] = hu;
  F[IHU] = hu * u + 0.5 * s->g * (h * h - Hloc * Hloc) + h * p;
  F[IHV] = hu * v;
  F[IHW] = hu * w;
  F[IHP] = hu * (p + c2);
}

/* fluxY (sgn_flux2d.h:104-116) */
static void flux_y(const or_ctx* s, const double* U, double Hloc, double* G) {
  const double h = U[IH], hv = U[IHV];
  const double u = U[IHU] / h, v = hv / h, w = U[IHW] / h, p = U[IHP] / h;
  const double c2 = s->c * s->c;
  G[IH] = hv;
  G[IHU] = hv * u;
  G[IHV] = hv * v + 0.5 * s->g * (h * h - Hloc * Hloc) + h * p;
  G[IHW] = hv * w;
  G[IHP] = hv * (p + c2);
}

/* source (sgn_flux2d.h:122-143), Manning branch included */
static void source(const or_ctx* s, const double* U, double Hloc, double Hx, double Hy,
                   double* S) {
  const double h = U[IH];
  const double u = U[IHU] / h, v = U[IHV] / h, w = U[IHW] / h, p = U[IHP] / h;
  const double c2 = s->c * s->c;
  const double bath = s->g * (h - Hloc) + s->gamma * p;
  S[IH] = 0.0;
  S[IHU] = bath * Hx;
  S[IHV] = bath * Hy;
  S[IHW] = s->gamma * p;
  S[IHP] = -2.0 * c2 * (w + u * Hx + v * Hy);
  if (s->nManning != 0.0) {
    const double n2 = s->nManning * s->nManning;
    const double vmag = sqrt(u * u + v * v);
    const double cf = n2 * s->g * vmag / cbrt(h);
    S[IHU] -= cf * u;
    S[IHV] -= cf * v;
  }
}

/* ncpX / ncpY (sgn_flux2d.h:150-161): only the hp component is non-zero */
static void ncp_x(const or_ctx* s, const double* U, double hx, double* B) {
  const double u = U[IHU] / U[IH];
  B[IH] = 0.0; B[IHU] = 0.0; B[IHV] = 0.0; B[IHW] = 0.0;
  B[IHP] = -s->c * s->c * u * hx;
}
static void ncp_y(const or_ctx* s, const double* U, double hy, double* B) {
  const double v = U[IHV] / U[IH];
  B[IH] = 0.0; B[IHU] = 0.0; B[IHV] = 0.0; B[IHW] = 0.0;
  B[IHP] = -s->c * s->c * v * hy;
}

/* rusanov (sgn_flux2d.h:169-179) */
static void rusanov(const or_ctx* s, const double* UL, const double* UR, int dir,
                    double Hface, double* Fn) {
  double FL[NVAR], FR[NVAR];
  if (dir == 0) { flux_x(s, UL, Hface, FL); flux_x(s, UR, Hface, FR); }
  else          { flux_y(s, UL, Hface, FL); flux_y(s, UR, Hface, FR); }
  const double lam = fmax(max_wave_speed_pt(s, UL, dir), max_wave_speed_pt(s, UR, dir));
  for (int k = 0; k < NVAR; ++k) Fn[k] = 0.5 * (FL[k] + FR[k]) - 0.5 * lam * (UR[k] - UL[k]);
}

/* energyDensity (sgn_flux2d.h:184-191) */
static double energy_density(const or_ctx* s, const double* U, double Hloc) {
  const double h = U[IH];
  const double u = U[IHU] / h, v = U[IHV] / h, w = U[IHW] / h;
  return 0.5 * h * (u * u + v * v + (1.0 / s->gamma) * w * w + s->g * (h - 2.0 * Hloc));
}

/* ------------------------------------------------------------------------- */
/* Solver set-up: src/solver/sgn2d.cpp:30-102, src/core/mesh2d.h              */
/* ------------------------------------------------------------------------- */

void or_node_coords(const or_ctx* s, double* x, double* y) {
  const int np = s->np;
  for (int e = 0; e < s->ne; ++e) {
    const int ex = e % s->Nx, ey = e / s->Nx;
    for (int b = 0; b < np; ++b)
      for (int a = 0; a < np; ++a) {
        const long gi = (long)e * s->npp + a + np * b;
        x[gi] = ex * s->hx + 0.5 * s->hx * (s->xi[a] + 1.0);
        y[gi] = ey * s->hy + 0.5 * s->hy * (s->xi[b] + 1.0);
      }
  }
}

or_ctx* or_create(int P, int Nx, int Ny, double Lx, double Ly, double g, double c,
                  double gamma, double nManning, int bc_x, int bc_y, int bathy_kind,
                  const double* bp, int n_par) {
  return or_create_points(P, Nx, Ny, Lx, Ly, g, c, gamma, nManning, bc_x, bc_y, bathy_kind,
                          bp, n_par, OR_POINTS_GLL);
}

or_ctx* or_create_points(int P, int Nx, int Ny, double Lx, double Ly, double g, double c,
                         double gamma, double nManning, int bc_x, int bc_y, int bathy_kind,
                         const double* bp, int n_par, int points) {
  (void)n_par;
  if (P < 1 || Nx < 2 || Ny < 2) return NULL; /* sgn2d.cpp:36 */
  if (points != OR_POINTS_GLL && points != OR_POINTS_GAUSS) return NULL;
  /* bathymetry requires GLL points (sgn2d.cpp:46-47) */
  if (points != OR_POINTS_GLL && bathy_kind != OR_BATHY_NONE) return NULL;
  or_ctx* s = (or_ctx*)calloc(1, sizeof(or_ctx));
  s->points = points;
  s->P = P; s->np = P + 1; s->npp = (P + 1) * (P + 1);
  s->Nx = Nx; s->Ny = Ny; s->ne = Nx * Ny;
  s->Nd = (long)s->ne * s->npp;
  s->Lx = Lx; s->Ly = Ly;
  s->hx = Lx / Nx; s->hy = Ly / Ny;            /* mesh2d.h:27-28 */
  s->Jx = 0.5 * s->hx; s->Jy = 0.5 * s->hy;    /* mesh2d.h:49-50 */
  s->g = g; s->c = c; s->gamma = gamma; s->nManning = nManning;
  s->bcx = bc_x; s->bcy = bc_y;
  const int np = s->np;
  s->xi = (double*)calloc(np, sizeof(double));
  s->bw = (double*)calloc(np, sizeof(double));
  s->D = (double*)calloc(np * np, sizeof(double));
  s->lL = (double*)calloc(np, sizeof(double));
  s->lR = (double*)calloc(np, sizeof(double));
  s->gLp = (double*)calloc(np, sizeof(double));
  s->gRp = (double*)calloc(np, sizeof(double));
  s->qw = (double*)calloc(np, sizeof(double));
  build_tables(s);

  const long Nd = s->Nd;
  s->Hnod = (double*)calloc(Nd, sizeof(double));
  s->Hx = (double*)calloc(Nd, sizeof(double));
  s->Hy = (double*)calloc(Nd, sizeof(double));
  s->HfaceX = (double*)calloc((size_t)s->ne * np, sizeof(double));
  s->HfaceY = (double*)calloc((size_t)s->ne * np, sizeof(double));
  s->HfaceXEnd = (double*)calloc((size_t)Ny * np, sizeof(double));
  s->HfaceYEnd = (double*)calloc((size_t)Nx * np, sizeof(double));
  if (bathy_kind == OR_BATHY_NONE) return s; /* flat bottom H = 0 (sgn2d.cpp:45) */

  /* nodal depth (sgn2d.cpp:49-52) */
  double* x = (double*)malloc(Nd * sizeof(double));
  double* y = (double*)malloc(Nd * sizeof(double));
  or_node_coords(s, x, y);
  for (long i = 0; i < Nd; ++i) s->Hnod[i] = or_bathy_eval(bathy_kind, bp, x[i], y[i]);
  free(x);
  free(y);
  /* nodal gradients by element-local differentiation (sgn2d.cpp:54-71) */
  for (int e = 0; e < s->ne; ++e) {
    const double* He = s->Hnod + (long)e * s->npp;
    for (int b = 0; b < np; ++b)
      for (int a = 0; a < np; ++a) {
        double dHx = 0.0, dHy = 0.0;
        for (int k = 0; k < np; ++k) {
          dHx += s->D[a * np + k] * He[k + np * b];
          dHy += s->D[b * np + k] * He[a + np * k];
        }
        s->Hx[(long)e * s->npp + a + np * b] = dHx / s->Jx;
        s->Hy[(long)e * s->npp + a + np * b] = dHy / s->Jy;
      }
  }
  /* face depths sampled on the edges (sgn2d.cpp:72-83) */
  for (int e = 0; e < s->ne; ++e) {
    const int ex = e % Nx, ey = e / Nx;
    for (int t = 0; t < np; ++t) {
      const double yb = ey * s->hy + 0.5 * s->hy * (s->xi[t] + 1.0);
      const double xa = ex * s->hx + 0.5 * s->hx * (s->xi[t] + 1.0);
      s->HfaceX[e * np + t] = or_bathy_eval(bathy_kind, bp, ex * s->hx, yb);
      s->HfaceY[e * np + t] = or_bathy_eval(bathy_kind, bp, xa, ey * s->hy);
    }
  }
  /* [not in the reference] depth on the right / top domain edges, sampled at
   * x = Nx hx and y = Ny hy: the left / bottom edge of the element that periodic
   * indexing (or the mirror-doubled domain) would place there. Walls only. */
  for (int ey = 0; ey < Ny; ++ey)
    for (int t = 0; t < np; ++t) {
      const double yb = ey * s->hy + 0.5 * s->hy * (s->xi[t] + 1.0);
      s->HfaceXEnd[ey * np + t] = or_bathy_eval(bathy_kind, bp, Nx * s->hx, yb);
    }
  for (int ex = 0; ex < Nx; ++ex)
    for (int t = 0; t < np; ++t) {
      const double xa = ex * s->hx + 0.5 * s->hx * (s->xi[t] + 1.0);
      s->HfaceYEnd[ex * np + t] = or_bathy_eval(bathy_kind, bp, xa, Ny * s->hy);
    }
  return s;
}

void or_destroy(or_ctx* s) {
  if (!s) return;
  free(s->xi); free(s->bw); free(s->D); free(s->lL); free(s->lR);
  free(s->gLp); free(s->gRp); free(s->qw);
  free(s->Hnod); free(s->Hx); free(s->Hy); free(s->HfaceX); free(s->HfaceY);
  free(s->HfaceXEnd); free(s->HfaceYEnd);
  free(s);
}

long or_ndof(const or_ctx* s) { return s->Nd; }

void or_tables(const or_ctx* s, double* nodes, double* D, double* lL, double* lR,
               double* gLp, double* gRp, double* qw) {
  const int n = s->np;
  if (nodes) memcpy(nodes, s->xi, n * sizeof(double));
  if (D) memcpy(D, s->D, n * n * sizeof(double));
  if (lL) memcpy(lL, s->lL, n * sizeof(double));
  if (lR) memcpy(lR, s->lR, n * sizeof(double));
  if (gLp) memcpy(gLp, s->gLp, n * sizeof(double));
  if (gRp) memcpy(gRp, s->gRp, n * sizeof(double));
  if (qw) memcpy(qw, s->qw, n * sizeof(double));
}

void or_bathymetry(const or_ctx* s, double* Hnod, double* Hx, double* Hy, double* HfaceX,
                   double* HfaceY, double* HfaceXEnd, double* HfaceYEnd) {
  const size_t nf = (size_t)s->ne * s->np;
  if (Hnod) memcpy(Hnod, s->Hnod, s->Nd * sizeof(double));
  if (Hx) memcpy(Hx, s->Hx, s->Nd * sizeof(double));
  if (Hy) memcpy(Hy, s->Hy, s->Nd * sizeof(double));
  if (HfaceX) memcpy(HfaceX, s->HfaceX, nf * sizeof(double));
  if (HfaceY) memcpy(HfaceY, s->HfaceY, nf * sizeof(double));
  if (HfaceXEnd) memcpy(HfaceXEnd, s->HfaceXEnd, (size_t)s->Ny * s->np * sizeof(double));
  if (HfaceYEnd) memcpy(HfaceYEnd, s->HfaceYEnd, (size_t)s->Nx * s->np * sizeof(double));
}

void or_set_bathymetry(or_ctx* s, const double* Hnod, const double* Hx, const double* Hy,
                       const double* HfaceX, const double* HfaceY, const double* HfaceXEnd,
                       const double* HfaceYEnd) {
  const size_t nf = (size_t)s->ne * s->np;
  if (Hnod) memcpy(s->Hnod, Hnod, s->Nd * sizeof(double));
  if (Hx) memcpy(s->Hx, Hx, s->Nd * sizeof(double));
  if (Hy) memcpy(s->Hy, Hy, s->Nd * sizeof(double));
  if (HfaceX) memcpy(s->HfaceX, HfaceX, nf * sizeof(double));
  if (HfaceY) memcpy(s->HfaceY, HfaceY, nf * sizeof(double));
  if (HfaceXEnd) memcpy(s->HfaceXEnd, HfaceXEnd, (size_t)s->Ny * s->np * sizeof(double));
  if (HfaceYEnd) memcpy(s->HfaceYEnd, HfaceYEnd, (size_t)s->Nx * s->np * sizeof(double));
}

/* ------------------------------------------------------------------------- */
/* rhs: src/solver/sgn2d.cpp:125-290                                          */
/* ------------------------------------------------------------------------- */

/* [not in the reference] mirror ghost of the element's own face trace across a wall
 * normal to direction dir: the normal momentum changes sign, written 0.0 + (-v). With
 * GLL points the trace is 0.0 + the edge node, and this is what the periodic reference
 * computes for the mirror-image element of the doubled domain. */
static void mirror_ghost(const double* own_trace, int dir, double* ghost) {
  for (int v = 0; v < NVAR; ++v) ghost[v] = 0.0 + own_trace[v];
  const int n = (dir == 0) ? IHU : IHV;
  ghost[n] = 0.0 + (-own_trace[n]);
}

int or_rhs(const or_ctx* s, const double* U, double* dU) {
  const int np = s->np, npp = s->npp, ne = s->ne, Nx = s->Nx, Ny = s->Ny;
  const long Nd = s->Nd;
  const double* D = s->D;
  const double *lL = s->lL, *lR = s->lR, *gLp = s->gLp, *gRp = s->gRp;
  const double Jx = s->Jx, Jy = s->Jy;
  memset(dU, 0, (size_t)NVAR * Nd * sizeof(double));

#define UIDX(e, a, b, var) ((long)(var) * Nd + (long)(e) * npp + (a) + np * (b))
  /* 1) face-extrapolated states (sgn2d.cpp:141-177) */
  const size_t nf = (size_t)ne * np * NVAR;
  double* xFaceL = (double*)malloc(nf * sizeof(double));
  double* xFaceR = (double*)malloc(nf * sizeof(double));
  double* yFaceB = (double*)malloc(nf * sizeof(double));
  double* yFaceT = (double*)malloc(nf * sizeof(double));
  for (int e = 0; e < ne; ++e)
    for (int var = 0; var < NVAR; ++var) {
      for (int b = 0; b < np; ++b) {
        double sL = 0.0, sR = 0.0;
        for (int a = 0; a < np; ++a) {
          const double val = U[UIDX(e, a, b, var)];
          sL += lL[a] * val;
          sR += lR[a] * val;
        }
        xFaceL[((size_t)e * np + b) * NVAR + var] = sL;
        xFaceR[((size_t)e * np + b) * NVAR + var] = sR;
      }
      for (int a = 0; a < np; ++a) {
        double sB = 0.0, sT = 0.0;
        for (int b = 0; b < np; ++b) {
          const double val = U[UIDX(e, a, b, var)];
          sB += lL[b] * val;
          sT += lR[b] * val;
        }
        yFaceB[((size_t)e * np + a) * NVAR + var] = sB;
        yFaceT[((size_t)e * np + a) * NVAR + var] = sT;
      }
    }

  /* 2..5) element loop (sgn2d.cpp:183-289) */
  double Fnod[25 * NVAR > 64 * NVAR ? 25 * NVAR : 64 * NVAR];
  double Gnod[25 * NVAR > 64 * NVAR ? 25 * NVAR : 64 * NVAR];
  double FxL[8 * NVAR], FxR[8 * NVAR], GyB[8 * NVAR], GyT[8 * NVAR];
  double hSxL[8], hSxR[8], hSyB[8], hSyT[8];
  double FdXL[8 * NVAR], FdXR[8 * NVAR], GdYB[8 * NVAR], GdYT[8 * NVAR];
  for (int e = 0; e < ne; ++e) {
    const int ex = e % Nx, ey = e / Nx;
    /* periodic neighbours (mesh2d.h:36-45) */
    const int eL = ((ex - 1 + Nx) % Nx) + Nx * ey, eR = ((ex + 1) % Nx) + Nx * ey;
    const int eB = ex + Nx * ((ey - 1 + Ny) % Ny), eT = ex + Nx * ((ey + 1) % Ny);
    const int wallL = (s->bcx == OR_BC_WALL && ex == 0);
    const int wallR = (s->bcx == OR_BC_WALL && ex == Nx - 1);
    const int wallB = (s->bcy == OR_BC_WALL && ey == 0);
    const int wallT = (s->bcy == OR_BC_WALL && ey == Ny - 1);

    /* 2) nodal fluxes (:188-196) */
    for (int b = 0; b < np; ++b)
      for (int a = 0; a < np; ++a) {
        double Un[NVAR];
        for (int var = 0; var < NVAR; ++var) Un[var] = U[UIDX(e, a, b, var)];
        const double Hl = s->Hnod[(long)e * npp + a + np * b];
        flux_x(s, Un, Hl, &Fnod[(a + np * b) * NVAR]);
        flux_y(s, Un, Hl, &Gnod[(a + np * b) * NVAR]);
      }

    /* 3) Rusanov fluxes and central depths on the four face lines (:198-227) */
    for (int b = 0; b < np; ++b) {
      double gL[NVAR], gR[NVAR];
      const double* uL = &xFaceR[((size_t)eL * np + b) * NVAR];
      const double* uMe = &xFaceL[((size_t)e * np + b) * NVAR];
      const double* uR = &xFaceL[((size_t)eR * np + b) * NVAR];
      const double* uMeR = &xFaceR[((size_t)e * np + b) * NVAR];
      if (wallL) {
        mirror_ghost(uMe, 0, gL);
        uL = gL;
      }
      if (wallR) {
        mirror_ghost(uMeR, 0, gR);
        uR = gR;
      }
      const double HxL = s->HfaceX[e * np + b];
      const double HxR = wallR ? s->HfaceXEnd[ey * np + b] : s->HfaceX[eR * np + b];
      rusanov(s, uL, uMe, 0, HxL, &FxL[b * NVAR]);
      rusanov(s, uMeR, uR, 0, HxR, &FxR[b * NVAR]);
      hSxL[b] = 0.5 * (uL[IH] + uMe[IH]);
      hSxR[b] = 0.5 * (uMeR[IH] + uR[IH]);
    }
    for (int a = 0; a < np; ++a) {
      double gB[NVAR], gT[NVAR];
      const double* uB = &yFaceT[((size_t)eB * np + a) * NVAR];
      const double* uMe = &yFaceB[((size_t)e * np + a) * NVAR];
      const double* uT = &yFaceB[((size_t)eT * np + a) * NVAR];
      const double* uMeT = &yFaceT[((size_t)e * np + a) * NVAR];
      if (wallB) {
        mirror_ghost(uMe, 1, gB);
        uB = gB;
      }
      if (wallT) {
        mirror_ghost(uMeT, 1, gT);
        uT = gT;
      }
      const double HyB = s->HfaceY[e * np + a];
      const double HyT = wallT ? s->HfaceYEnd[ex * np + a] : s->HfaceY[eT * np + a];
      rusanov(s, uB, uMe, 1, HyB, &GyB[a * NVAR]);
      rusanov(s, uMeT, uT, 1, HyT, &GyT[a * NVAR]);
      hSyB[a] = 0.5 * (uB[IH] + uMe[IH]);
      hSyT[a] = 0.5 * (uMeT[IH] + uT[IH]);
    }

    /* 4) the element's own face fluxes with the same face depth (:229-239) */
    for (int b = 0; b < np; ++b) {
      const double HxR = wallR ? s->HfaceXEnd[ey * np + b] : s->HfaceX[eR * np + b];
      flux_x(s, &xFaceL[((size_t)e * np + b) * NVAR], s->HfaceX[e * np + b], &FdXL[b * NVAR]);
      flux_x(s, &xFaceR[((size_t)e * np + b) * NVAR], HxR, &FdXR[b * NVAR]);
    }
    for (int a = 0; a < np; ++a) {
      const double HyT = wallT ? s->HfaceYEnd[ex * np + a] : s->HfaceY[eT * np + a];
      flux_y(s, &yFaceB[((size_t)e * np + a) * NVAR], s->HfaceY[e * np + a], &GdYB[a * NVAR]);
      flux_y(s, &yFaceT[((size_t)e * np + a) * NVAR], HyT, &GdYT[a * NVAR]);
    }

    /* 5) per-node update (:241-288) */
    for (int b = 0; b < np; ++b)
      for (int a = 0; a < np; ++a) {
        const int loc = a + np * b;
        double Un[NVAR];
        for (int var = 0; var < NVAR; ++var) Un[var] = U[UIDX(e, a, b, var)];
        double dF[NVAR], dG[NVAR];
        for (int var = 0; var < NVAR; ++var) {
          double dfx = 0.0, dgy = 0.0;
          for (int k = 0; k < np; ++k) {
            dfx += D[a * np + k] * Fnod[(k + np * b) * NVAR + var];
            dgy += D[b * np + k] * Gnod[(a + np * k) * NVAR + var];
          }
          const double cx = (FxL[b * NVAR + var] - FdXL[b * NVAR + var]) * gLp[a] +
                            (FxR[b * NVAR + var] - FdXR[b * NVAR + var]) * gRp[a];
          const double cy = (GyB[a * NVAR + var] - GdYB[a * NVAR + var]) * gLp[b] +
                            (GyT[a * NVAR + var] - GdYT[a * NVAR + var]) * gRp[b];
          dF[var] = (dfx + cx) / Jx;
          dG[var] = (dgy + cy) / Jy;
        }
        double dhx = 0.0, dhy = 0.0;
        for (int k = 0; k < np; ++k) {
          dhx += D[a * np + k] * U[UIDX(e, k, b, IH)];
          dhy += D[b * np + k] * U[UIDX(e, a, k, IH)];
        }
        dhx += (hSxL[b] - xFaceL[((size_t)e * np + b) * NVAR + IH]) * gLp[a] +
               (hSxR[b] - xFaceR[((size_t)e * np + b) * NVAR + IH]) * gRp[a];
        dhy += (hSyB[a] - yFaceB[((size_t)e * np + a) * NVAR + IH]) * gLp[b] +
               (hSyT[a] - yFaceT[((size_t)e * np + a) * NVAR + IH]) * gRp[b];
        const double hx = dhx / Jx, hy = dhy / Jy;
        double Bx[NVAR], By[NVAR], S[NVAR];
        ncp_x(s, Un, hx, Bx);
        ncp_y(s, Un, hy, By);
        source(s, Un, s->Hnod[(long)e * npp + loc], s->Hx[(long)e * npp + loc],
               s->Hy[(long)e * npp + loc], S);
        for (int var = 0; var < NVAR; ++var)
          dU[UIDX(e, a, b, var)] = -dF[var] - dG[var] - Bx[var] - By[var] + S[var];
      }
  }
#undef UIDX
  free(xFaceL); free(xFaceR); free(yFaceB); free(yFaceT);
  return 0;
}

/* ------------------------------------------------------------------------- */
/* Diagnostics: sgn2d.cpp:295-348                                             */
/* ------------------------------------------------------------------------- */

double or_max_wave_speed(const or_ctx* s, const double* U) {
  const long Nd = s->Nd;
  double lam = 0.0;
  for (long i = 0; i < Nd; ++i) {
    double Un[NVAR];
    for (int v = 0; v < NVAR; ++v) Un[v] = U[(long)v * Nd + i];
    lam = fmax(lam, fmax(max_wave_speed_pt(s, Un, 0), max_wave_speed_pt(s, Un, 1)));
  }
  return lam;
}

double or_cfl_time_step(const or_ctx* s, const double* U, double cfl) {
  const double lam = or_max_wave_speed(s, U);
  const double dxEff = fmin(s->hx, s->hy) / (2.0 * s->P + 1.0);
  return cfl * dxEff / (lam > 0.0 ? lam : 1e-300);
}

double or_mass(const or_ctx* s, const double* U) {
  const double JJ = s->Jx * s->Jy;
  double m = 0.0;
  for (int e = 0; e < s->ne; ++e)
    for (int b = 0; b < s->np; ++b)
      for (int a = 0; a < s->np; ++a)
        m += s->qw[a] * s->qw[b] * U[(long)e * s->npp + a + s->np * b];
  return m * JJ;
}

double or_energy(const or_ctx* s, const double* U) {
  const long Nd = s->Nd;
  const double JJ = s->Jx * s->Jy;
  double E = 0.0;
  for (int e = 0; e < s->ne; ++e)
    for (int b = 0; b < s->np; ++b)
      for (int a = 0; a < s->np; ++a) {
        const long loc = (long)e * s->npp + a + s->np * b;
        double Un[NVAR];
        for (int v = 0; v < NVAR; ++v) Un[v] = U[(long)v * Nd + loc];
        E += s->qw[a] * s->qw[b] * energy_density(s, Un, s->Hnod[loc]);
      }
  return E * JJ;
}

/* ------------------------------------------------------------------------- */
/* Integrators: src/solver/rk.cpp                                             */
/* ------------------------------------------------------------------------- */

/* rk4Step (rk.cpp:23-38) */
void or_rk4_step(const or_ctx* s, double t, double dt, double* u) {
  (void)t;
  const long n = NVAR * s->Nd;
  double* k1 = (double*)malloc(n * sizeof(double));
  double* k2 = (double*)malloc(n * sizeof(double));
  double* k3 = (double*)malloc(n * sizeof(double));
  double* k4 = (double*)malloc(n * sizeof(double));
  double* tmp = (double*)malloc(n * sizeof(double));
  or_rhs(s, u, k1);
  for (long i = 0; i < n; ++i) tmp[i] = u[i] + 0.5 * dt * k1[i];
  or_rhs(s, tmp, k2);
  for (long i = 0; i < n; ++i) tmp[i] = u[i] + 0.5 * dt * k2[i];
  or_rhs(s, tmp, k3);
  for (long i = 0; i < n; ++i) tmp[i] = u[i] + dt * k3[i];
  or_rhs(s, tmp, k4);
  for (long i = 0; i < n; ++i)
    u[i] += (dt / 6.0) * (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]);
  free(k1); free(k2); free(k3); free(k4); free(tmp);
}

/* bs3Step (rk.cpp:41-54) */
void or_bs3_step(const or_ctx* s, double t, double dt, double* u) {
  (void)t;
  const long n = NVAR * s->Nd;
  double* k1 = (double*)malloc(n * sizeof(double));
  double* k2 = (double*)malloc(n * sizeof(double));
  double* k3 = (double*)malloc(n * sizeof(double));
  double* tmp = (double*)malloc(n * sizeof(double));
  or_rhs(s, u, k1);
  for (long i = 0; i < n; ++i) tmp[i] = u[i] + 0.5 * dt * k1[i];
  or_rhs(s, tmp, k2);
  for (long i = 0; i < n; ++i) tmp[i] = u[i] + 0.75 * dt * k2[i];
  or_rhs(s, tmp, k3);
  for (long i = 0; i < n; ++i)
    u[i] += dt * (2.0 / 9.0 * k1[i] + 1.0 / 3.0 * k2[i] + 4.0 / 9.0 * k3[i]);
  free(k1); free(k2); free(k3); free(tmp);
}

static double dmax(double a, double b) { return (a < b) ? b : a; } /* std::max */
static double dmin(double a, double b) { return (b < a) ? b : a; } /* std::min */

/* integrateAdaptive (rk.cpp:67-164) */
long or_integrate_adaptive(const or_ctx* s, double* u, double t0, double tEnd, double dt0,
                           const double* opts, double* stats, double* log, long max_log) {
  const double atol = opts[0], rtol = opts[1], dtMin = opts[2], dtMax = opts[3];
  const double safety = opts[4], facMin = opts[5], facMax = opts[6];
  /* [not in the reference] opts[7] > 0 stops after that many accepted steps */
  const long stopAfter = (long)opts[7];
  const int orderLow = 2;
  const double expo = 1.0 / (orderLow + 1.0);
  const double alpha = 0.7 * expo;
  const double beta = 0.4 * expo;
  long accepted = 0, rejected = 0, rhsEvals = 0, attempts = 0;
  double tReached = t0, dtLast = 0.0, maxNormLast = 0.0;
  int aborted = 0;
  const long n = NVAR * s->Nd;

  double* k1 = (double*)malloc(n * sizeof(double));
  double* k2 = (double*)malloc(n * sizeof(double));
  double* k3 = (double*)malloc(n * sizeof(double));
  double* k4 = (double*)malloc(n * sizeof(double));
  double* tmp = (double*)malloc(n * sizeof(double));
  double* uNew = (double*)malloc(n * sizeof(double));
  double* ucur = u; /* the caller's buffer holds the state at return (see end) */

  double t = t0;
  double dt = dmin(dt0, dtMax);
  double errPrev = 1.0;
  or_rhs(s, ucur, k1);
  ++rhsEvals;
  while (t < tEnd - 1e-15 * dmax(1.0, fabs(tEnd))) {
    if (t + dt > tEnd) dt = tEnd - t;
    for (long i = 0; i < n; ++i) tmp[i] = ucur[i] + 0.5 * dt * k1[i];
    or_rhs(s, tmp, k2);
    for (long i = 0; i < n; ++i) tmp[i] = ucur[i] + 0.75 * dt * k2[i];
    or_rhs(s, tmp, k3);
    for (long i = 0; i < n; ++i)
      uNew[i] = ucur[i] + dt * (2.0 / 9.0 * k1[i] + 1.0 / 3.0 * k2[i] + 4.0 / 9.0 * k3[i]);
    or_rhs(s, uNew, k4);
    rhsEvals += 3;
    double errL2 = 0.0, errMax = 0.0;
    for (long i = 0; i < n; ++i) {
      const double uEmb = ucur[i] + dt * (7.0 / 24.0 * k1[i] + 0.25 * k2[i] +
                                          1.0 / 3.0 * k3[i] + 0.125 * k4[i]);
      const double e = uNew[i] - uEmb;
      const double sc = atol + rtol * dmax(fabs(ucur[i]), fabs(uNew[i]));
      const double r = e / sc;
      errL2 += r * r;
      errMax = dmax(errMax, fabs(r));
    }
    errL2 = sqrt(errL2 / (double)n);
    const double errNorm = dmax(errL2, 1e-300);
    const int acc = (errNorm <= 1.0);
    if (log && attempts < max_log) {
      log[4 * attempts + 0] = t;
      log[4 * attempts + 1] = dt;
      log[4 * attempts + 2] = errNorm;
      log[4 * attempts + 3] = acc;
    }
    ++attempts;
    if (acc) {
      t += dt;
      double* sw = ucur; ucur = uNew; uNew = sw;
      sw = k1; k1 = k4; k4 = sw;
      ++accepted;
      tReached = t;
      dtLast = dt;
      maxNormLast = errMax;
      errPrev = errNorm;
      if (stopAfter > 0 && accepted >= stopAfter) break;
    } else {
      ++rejected;
    }
    /* [not in the reference] NaN guard: stop instead of looping forever */
    if (errNorm != errNorm) { aborted = 2; break; }
    double fac = safety * pow(errNorm, -alpha) * pow(errPrev, beta);
    fac = (fac < facMin) ? facMin : (facMax < fac) ? facMax : fac; /* std::clamp */
    double dtNext = dt * fac;
    dtNext = dmin(dtNext, dtMax);
    if (dtNext < dtMin) {
      aborted = 1;
      dtLast = dtNext;
      break;
    }
    dt = dtNext;
  }
  if (ucur != u) { /* the accepted state lives in a work buffer: copy it back */
    memcpy(u, ucur, n * sizeof(double));
    uNew = ucur;
  }
  free(k1); free(k2); free(k3); free(k4); free(tmp); free(uNew);
  if (stats) {
    stats[0] = (double)accepted; stats[1] = (double)rejected; stats[2] = (double)rhsEvals;
    stats[3] = tReached; stats[4] = dtLast; stats[5] = maxNormLast; stats[6] = aborted;
  }
  return attempts;
}
