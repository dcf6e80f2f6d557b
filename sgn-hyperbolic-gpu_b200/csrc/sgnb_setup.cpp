// sgnb_setup.cpp -- host-side set-up of the FR discretisation: FR tables, node
// coordinates, and the bathymetry statics the kernels read.
//
// The arithmetic here must produce the same doubles as the reference's constructors
// (FROperators1D, src/core/fr_operators.cpp:134-200, and SGN2D, src/solver/sgn2d.cpp:30-84),
// because the exact mode promises bit-identical right-hand sides: each quantity is
// formed with the same published method in the same operation order.
#include "sgnb_setup.h"

#include <cmath>
#include <vector>

namespace sgnb {
namespace {

constexpr double kPi = 3.14159265358979323846;

// Legendre polynomial by the Bonnet recurrence (k+1) L_{k+1} = (2k+1) x L_k - k L_{k-1}.
double legendre(int n, double x) {
  if (n == 0) return 1.0;
  if (n == 1) return x;
  double prev = 1.0, cur = x;
  for (int k = 1; k < n; ++k) {
    const double next = ((2.0 * k + 1.0) * x * cur - k * prev) / (k + 1.0);
    prev = cur;
    cur = next;
  }
  return cur;
}

// L_n'(x) = n (x L_n - L_{n-1}) / (x^2 - 1); at x = +-1 the closed form
// L_n'(+-1) = (+-1)^(n-1) n (n+1) / 2.
double legendre_deriv(int n, double x) {
  if (n == 0) return 0.0;
  const double q = x * x - 1.0;
  if (std::fabs(q) < 1e-14) {
    const double sgn = (x > 0.0) ? 1.0 : ((n - 1) % 2 == 0 ? 1.0 : -1.0);
    return sgn * 0.5 * n * (n + 1.0);
  }
  return n * (x * legendre(n, x) - legendre(n - 1, x)) / q;
}

// Gauss-Lobatto points: +-1 and the roots of L_P', found by Newton's method from the
// Chebyshev-Lobatto points; L_P'' comes from Legendre's equation.
void gll_nodes(int P, FrTables& t) {
  t.nodes[0] = -1.0;
  t.nodes[P] = 1.0;
  for (int i = 1; i < P; ++i) {
    double x = -std::cos(kPi * i / (double)P);
    for (int it = 0; it < 100; ++it) {
      const double f = legendre_deriv(P, x);
      const double fpp = (2.0 * x * legendre_deriv(P, x) - P * (P + 1.0) * legendre(P, x)) /
                         (1.0 - x * x);
      const double step = f / fpp;
      x -= step;
      if (std::fabs(step) < 1e-15) break;
    }
    t.nodes[i] = x;
  }
}

// Gauss-Legendre points: the n = P + 1 roots of L_n by Newton's method from the
// asymptotic guesses -cos(pi (i + 3/4) / (n + 1/2)).
void gauss_nodes(int P, FrTables& t) {
  const int n = P + 1;
  for (int i = 0; i < n; ++i) {
    double x = -std::cos(kPi * (i + 0.75) / (n + 0.5));
    for (int it = 0; it < 100; ++it) {
      const double f = legendre(n, x);
      const double fp = legendre_deriv(n, x);
      const double step = f / fp;
      x -= step;
      if (std::fabs(step) < 1e-15) break;
    }
    t.nodes[i] = x;
  }
}

// Lagrange basis polynomial j of the nodes x (barycentric weights bw) at xq: the
// barycentric formula w_j / (xq - x_j) / sum_k w_k / (xq - x_k), and exactly the
// Kronecker delta where xq is a node.
double lagrange(int n, const double* x, const double* bw, int j, double xq) {
  for (int k = 0; k < n; ++k)
    if (std::fabs(xq - x[k]) < 1e-14) return (k == j) ? 1.0 : 0.0;
  const double num = bw[j] / (xq - x[j]);
  double den = 0.0;
  for (int k = 0; k < n; ++k) den += bw[k] / (xq - x[k]);
  return num / den;
}

}  // namespace

bool fr_tables(int P, FrTables& t, bool gauss) {
  if (P < 1 || P > 7) return false;
  const int n = P + 1;
  t.P = P;
  t.gauss = gauss;
  if (gauss) gauss_nodes(P, t);
  else gll_nodes(P, t);
  // barycentric weights 1 / prod_{k != j} (x_j - x_k)
  double bw[8];
  for (int j = 0; j < n; ++j) {
    double prod = 1.0;
    for (int k = 0; k < n; ++k)
      if (k != j) prod *= (t.nodes[j] - t.nodes[k]);
    bw[j] = 1.0 / prod;
  }
  // differentiation matrix (Berrut-Trefethen): off-diagonal (w_j/w_i)/(x_i-x_j), the
  // diagonal as minus the off-diagonal row sum so that D applied to a constant is 0
  for (int i = 0; i < n; ++i) {
    double diag = 0.0;
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      const double dij = (bw[j] / bw[i]) / (t.nodes[i] - t.nodes[j]);
      t.D[i * n + j] = dij;
      diag -= dij;
    }
    t.D[i * n + i] = diag;
  }
  // interpolation rows to the faces x = -1, +1 (unit rows for the end-point nodes of GLL)
  for (int j = 0; j < n; ++j) {
    t.lL[j] = lagrange(n, t.nodes, bw, j, -1.0);
    t.lR[j] = lagrange(n, t.nodes, bw, j, +1.0);
  }
  // Huynh's g_DG correction functions gL = (-1)^P (L_P - L_{P+1})/2,
  // gR = (L_P + L_{P+1})/2, differentiated at the nodes
  const double sgnP = (P % 2 == 0) ? 1.0 : -1.0;
  for (int i = 0; i < n; ++i) {
    const double a = legendre_deriv(P, t.nodes[i]);
    const double b = legendre_deriv(P + 1, t.nodes[i]);
    t.gLp[i] = 0.5 * sgnP * (a - b);
    t.gRp[i] = 0.5 * (a + b);
  }
  if (gauss) {
    // Gauss quadrature weights 2 / ((1 - x_i^2) L_{P+1}'(x_i)^2)
    for (int i = 0; i < n; ++i) {
      const double d = legendre_deriv(P + 1, t.nodes[i]);
      t.qw[i] = 2.0 / ((1.0 - t.nodes[i] * t.nodes[i]) * d * d);
    }
  } else {
    // Lobatto quadrature weights 2 / (P (P+1) L_P(x_i)^2)
    for (int i = 0; i < n; ++i) {
      const double lp = legendre(P, t.nodes[i]);
      t.qw[i] = 2.0 / (P * (P + 1.0) * lp * lp);
    }
  }
  return true;
}

double still_depth(int kind, const double* p, double x, double y) {
  switch (kind) {
    case 1:  // constant
      return p[0];
    case 2: {  // Gaussian bump: p0 - p1 exp(-((x-p2)^2 + (y-p3)^2) / p4)
      const double dx = x - p[2], dy = y - p[3];
      return p[0] - p[1] * std::exp(-(dx * dx + dy * dy) / p[4]);
    }
    case 3: {  // elliptic shoal: plane p0, crest depth p1 at (p2, p3), semi-axes p4, p5;
               // H = p0 - (p0 - p1)(1 - r^2)^3 inside the ellipse r < 1
      const double dx = (x - p[2]) / p[4], dy = (y - p[3]) / p[5];
      const double r2 = dx * dx + dy * dy;
      if (r2 >= 1.0) return p[0];
      const double q = 1.0 - r2;
      return p[0] - (p[0] - p[1]) * (q * q * q);
    }
    case 4: {  // p0 minus p1 Gaussian bumps (A, xc, yc, sigma)
      const int nb = (int)p[1];
      double s = 0.0;
      for (int k = 0; k < nb; ++k) {
        const double* b = p + 2 + 4 * k;
        const double dx = x - b[1], dy = y - b[2];
        s += b[0] * std::exp(-(dx * dx + dy * dy) / (2.0 * b[3] * b[3]));
      }
      return p[0] - s;
    }
    case 5: {  // bilinear interpolant of Mx x My cell means on [0,Lx] x [0,Ly], periodic
      const int Mx = (int)p[0], My = (int)p[1];
      const double cx = p[2] / Mx, cy = p[3] / My;
      const double sx = x / cx - 0.5, sy = y / cy - 0.5;
      const double fx0 = std::floor(sx), fy0 = std::floor(sy);
      const double tx = sx - fx0, ty = sy - fy0;
      int i0 = (int)fx0, j0 = (int)fy0;
      int i1 = i0 + 1, j1 = j0 + 1;
      i0 = ((i0 % Mx) + Mx) % Mx; i1 = ((i1 % Mx) + Mx) % Mx;
      j0 = ((j0 % My) + My) % My; j1 = ((j1 % My) + My) % My;
      const double* m = p + 4;
      const double v00 = m[i0 + Mx * j0], v10 = m[i1 + Mx * j0];
      const double v01 = m[i0 + Mx * j1], v11 = m[i1 + Mx * j1];
      const double lo = v00 + tx * (v10 - v00);
      const double hi = v01 + tx * (v11 - v01);
      return lo + ty * (hi - lo);
    }
    default:
      return 0.0;
  }
}

int bathy_param_count(int kind, const double* p, int n) {
  switch (kind) {
    case 0: return 0;
    case 1: return 1;
    case 2: return 5;
    case 3: return 6;
    case 4: return (n >= 2) ? 2 + 4 * (int)p[1] : 2;
    case 5: return (n >= 2) ? 4 + (int)p[0] * (int)p[1] : 4;
    default: return -1;
  }
}

void node_coords(const Mesh& m, const FrTables& t, double* x, double* y) {
  const int np = t.P + 1, npp = np * np;
  for (long long e = 0; e < (long long)m.Nx * m.Ny; ++e) {
    const int ex = (int)(e % m.Nx), ey = (int)(e / m.Nx);
    for (int b = 0; b < np; ++b)
      for (int a = 0; a < np; ++a) {
        const long long g = e * npp + a + np * b;
        x[g] = (m.ex0 + ex) * m.hx + 0.5 * m.hx * (t.nodes[a] + 1.0);
        y[g] = ey * m.hy + 0.5 * m.hy * (t.nodes[b] + 1.0);
      }
  }
}

void depth_gradients(const Mesh& m, const FrTables& t, const double* Hnod, double* Hx,
                     double* Hy) {
  // nodal gradients: the GLL derivative of H along each x-line and y-line, over J
  const int np = t.P + 1, npp = np * np;
  const long long ne = (long long)m.Nx * m.Ny;
  const double Jx = 0.5 * m.hx, Jy = 0.5 * m.hy;
  for (long long e = 0; e < ne; ++e) {
    const double* He = Hnod + e * npp;
    for (int b = 0; b < np; ++b)
      for (int a = 0; a < np; ++a) {
        double sx = 0.0, sy = 0.0;
        for (int k = 0; k < np; ++k) {
          sx += t.D[a * np + k] * He[k + np * b];
          sy += t.D[b * np + k] * He[a + np * k];
        }
        Hx[e * npp + a + np * b] = sx / Jx;
        Hy[e * npp + a + np * b] = sy / Jy;
      }
  }
}

void bathymetry(const Mesh& m, const FrTables& t, int kind, const double* p,
                Bathymetry& out) {
  const int np = t.P + 1, npp = np * np;
  const long long ne = (long long)m.Nx * m.Ny, Nd = ne * npp;
  out.Hnod.assign(Nd, 0.0);
  out.Hx.assign(Nd, 0.0);
  out.Hy.assign(Nd, 0.0);
  out.HfX.assign(ne * np, 0.0);
  out.HfY.assign(ne * np, 0.0);
  out.HfXEnd.assign((size_t)m.Ny * np, 0.0);
  out.HfYEnd.assign((size_t)m.Nx * np, 0.0);
  if (kind == 0) return;  // flat bottom at H = 0
  std::vector<double> x(Nd), y(Nd);
  node_coords(m, t, x.data(), y.data());
  for (long long i = 0; i < Nd; ++i) out.Hnod[i] = still_depth(kind, p, x[i], y[i]);
  depth_gradients(m, t, out.Hnod.data(), out.Hx.data(), out.Hy.data());
  // face depths sampled on the left / bottom element edges at the transverse nodes
  for (long long e = 0; e < ne; ++e) {
    const int ex = (int)(e % m.Nx), ey = (int)(e / m.Nx);
    for (int s = 0; s < np; ++s) {
      const double yt = ey * m.hy + 0.5 * m.hy * (t.nodes[s] + 1.0);
      const double xt = (m.ex0 + ex) * m.hx + 0.5 * m.hx * (t.nodes[s] + 1.0);
      out.HfX[e * np + s] = still_depth(kind, p, (m.ex0 + ex) * m.hx, yt);
      out.HfY[e * np + s] = still_depth(kind, p, xt, ey * m.hy);
    }
  }
  // right / top domain edges (walls), at x = Nx hx and y = Ny hy
  for (int ey = 0; ey < m.Ny; ++ey)
    for (int s = 0; s < np; ++s) {
      const double yt = ey * m.hy + 0.5 * m.hy * (t.nodes[s] + 1.0);
      out.HfXEnd[(size_t)ey * np + s] =
          still_depth(kind, p, m.wrapx ? 0.0 : (m.ex0 + m.Nx) * m.hx, yt);
    }
  for (int ex = 0; ex < m.Nx; ++ex)
    for (int s = 0; s < np; ++s) {
      const double xt = (m.ex0 + ex) * m.hx + 0.5 * m.hx * (t.nodes[s] + 1.0);
      out.HfYEnd[(size_t)ex * np + s] = still_depth(kind, p, xt, m.Ny * m.hy);
    }
}

namespace {
// The four cells and bilinear weights of the kind-5 interpolant at (x, y) (the same
// index arithmetic as still_depth).
void cell_weights(const double* p, double x, double y, int idx[4], double w[4]) {
  const int Mx = (int)p[0], My = (int)p[1];
  const double cx = p[2] / Mx, cy = p[3] / My;
  const double sx = x / cx - 0.5, sy = y / cy - 0.5;
  const double fx0 = std::floor(sx), fy0 = std::floor(sy);
  const double tx = sx - fx0, ty = sy - fy0;
  int i0 = (int)fx0, j0 = (int)fy0;
  int i1 = i0 + 1, j1 = j0 + 1;
  i0 = ((i0 % Mx) + Mx) % Mx; i1 = ((i1 % Mx) + Mx) % Mx;
  j0 = ((j0 % My) + My) % My; j1 = ((j1 % My) + My) % My;
  idx[0] = i0 + Mx * j0; w[0] = (1.0 - tx) * (1.0 - ty);
  idx[1] = i1 + Mx * j0; w[1] = tx * (1.0 - ty);
  idx[2] = i0 + Mx * j1; w[2] = (1.0 - tx) * ty;
  idx[3] = i1 + Mx * j1; w[3] = tx * ty;
}
}  // namespace

void cells_transpose(const Mesh& m, const FrTables& t, const double* p, const Bathymetry& bar,
                     double* means_bar) {
  const int np = t.P + 1, npp = np * np;
  const long long ne = (long long)m.Nx * m.Ny, Nd = ne * npp;
  const int Mx = (int)p[0], My = (int)p[1];
  for (long long i = 0; i < (long long)Mx * My; ++i) means_bar[i] = 0.0;
  // nodal gradients are D H / J along the element's lines: move their cotangents to H
  std::vector<double> Hn(bar.Hnod.begin(), bar.Hnod.end());
  const double Jx = 0.5 * m.hx, Jy = 0.5 * m.hy;
  for (long long e = 0; e < ne; ++e) {
    double* He = Hn.data() + e * npp;
    const double* gx = bar.Hx.data() + e * npp;
    const double* gy = bar.Hy.data() + e * npp;
    for (int b = 0; b < np; ++b)
      for (int a = 0; a < np; ++a)
        for (int k = 0; k < np; ++k) {
          He[k + np * b] += t.D[a * np + k] * gx[a + np * b] / Jx;
          He[a + np * k] += t.D[b * np + k] * gy[a + np * b] / Jy;
        }
  }
  auto add = [&](double x, double y, double g) {
    int idx[4];
    double w[4];
    cell_weights(p, x, y, idx, w);
    for (int q = 0; q < 4; ++q) means_bar[idx[q]] += w[q] * g;
  };
  std::vector<double> x(Nd), y(Nd);
  node_coords(m, t, x.data(), y.data());
  for (long long i = 0; i < Nd; ++i) add(x[i], y[i], Hn[i]);
  for (long long e = 0; e < ne; ++e) {
    const int ex = (int)(e % m.Nx), ey = (int)(e / m.Nx);
    for (int s = 0; s < np; ++s) {
      const double yt = ey * m.hy + 0.5 * m.hy * (t.nodes[s] + 1.0);
      const double xt = (m.ex0 + ex) * m.hx + 0.5 * m.hx * (t.nodes[s] + 1.0);
      add((m.ex0 + ex) * m.hx, yt, bar.HfX[e * np + s]);
      add(xt, ey * m.hy, bar.HfY[e * np + s]);
    }
  }
  for (int ey = 0; ey < m.Ny; ++ey)
    for (int s = 0; s < np; ++s)
      add(m.wrapx ? 0.0 : (m.ex0 + m.Nx) * m.hx, ey * m.hy + 0.5 * m.hy * (t.nodes[s] + 1.0),
          bar.HfXEnd[(size_t)ey * np + s]);
  for (int ex = 0; ex < m.Nx; ++ex)
    for (int s = 0; s < np; ++s)
      add((m.ex0 + ex) * m.hx + 0.5 * m.hx * (t.nodes[s] + 1.0), m.Ny * m.hy, bar.HfYEnd[(size_t)ex * np + s]);
}

}  // namespace sgnb
