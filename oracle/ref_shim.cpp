// ref_shim.cpp -- C entry points over the reference's own CPU solver sources.
//
// TEST INFRASTRUCTURE ONLY. Compiled by oracle/Makefile together with the
// reference's src/solver/sgn2d.cpp, src/solver/rk.cpp and src/core/fr_operators.cpp,
// read from where they lie (nothing is copied into this repository), into
// oracle/_ref/libsgnref.so. It exposes the same C interface as the restatement in
// sgn_oracle.c (sgn_oracle.h), so the tests can check one against the other.
//
// Reflective walls are not a reference feature. They are expressed here through the
// reference itself: the state is mirror-copied onto the doubled domain
// [0,2Lx] x [0,2Ly] (normal momentum negated in the mirror images), the periodic
// reference rhs runs there, and the first quadrant is returned. With GLL points the
// face traces are node values, so this is exactly the mirror-ghost wall. With Gauss
// points the mirror element's trace is interpolated with lR where the restatement
// mirrors the own trace formed with lL: equal to round-off, not bit for bit.
#include "sgn_oracle.h"
#include "or_bathy.h"

#include "solver/rk.h"
#include "solver/sgn1d.h"
#include "solver/sgn2d.h"
#include "io/vtk2d.h"

#include <cstring>
#include <memory>
#include <vector>

struct or_ctx {
  int Nx, Ny, np, npp;
  int bcx, bcy;
  int Nx2, Ny2;  // size of the simulated (possibly doubled) periodic domain
  std::unique_ptr<sgn::SGN2D> sys;  // the reference solver on the simulated domain
  std::vector<double> bpar;
  std::vector<double> Ubig, dUbig;  // doubled-domain work arrays (walls only)
  long ndof() const { return (long)Nx * Ny * npp; }
  bool doubled() const { return bcx == OR_BC_WALL || bcy == OR_BC_WALL; }

  // original node (ex, ey, a, b) -> index in the simulated domain state, per field
  long big_index(int ex, int ey, int a, int b) const {
    const long e = ex + (long)Nx2 * ey;
    return e * npp + a + np * b;
  }

  // mirror-copy a state on the original domain into the doubled periodic domain
  void expand(const double* U) {
    const long Nd = ndof(), Nd2 = (long)Nx2 * Ny2 * npp;
    Ubig.assign(5 * Nd2, 0.0);
    for (int ey2 = 0; ey2 < Ny2; ++ey2)
      for (int ex2 = 0; ex2 < Nx2; ++ex2) {
        const bool mx = ex2 >= Nx, my = ey2 >= Ny;
        const int ex = mx ? (2 * Nx - 1 - ex2) : ex2;
        const int ey = my ? (2 * Ny - 1 - ey2) : ey2;
        for (int b2 = 0; b2 < np; ++b2)
          for (int a2 = 0; a2 < np; ++a2) {
            const int a = mx ? (np - 1 - a2) : a2;
            const int b = my ? (np - 1 - b2) : b2;
            const long src = (long)(ex + Nx * ey) * npp + a + np * b;
            const long dst = big_index(ex2, ey2, a2, b2);
            for (int v = 0; v < 5; ++v) {
              double val = U[(long)v * Nd + src];
              if ((v == 1 && mx) || (v == 2 && my)) val = -val;
              Ubig[(long)v * Nd2 + dst] = val;
            }
          }
      }
  }
  void extract(const std::vector<double>& big, double* out) const {
    const long Nd = ndof(), Nd2 = (long)Nx2 * Ny2 * npp;
    for (int ey = 0; ey < Ny; ++ey)
      for (int ex = 0; ex < Nx; ++ex)
        for (int b = 0; b < np; ++b)
          for (int a = 0; a < np; ++a) {
            const long src = big_index(ex, ey, a, b);
            const long dst = (long)(ex + Nx * ey) * npp + a + np * b;
            for (int v = 0; v < 5; ++v) out[(long)v * Nd + dst] = big[(long)v * Nd2 + src];
          }
  }
  void rhs(const double* U, double* dU) {
    if (!doubled()) {
      const long n = 5 * ndof();
      sgn::State Us(U, U + n), R;
      sys->rhs(Us, R);
      std::memcpy(dU, R.data(), n * sizeof(double));
      return;
    }
    expand(U);
    sys->rhs(Ubig, dUbig);
    extract(dUbig, dU);
  }
};

extern "C" {

or_ctx* or_create(int P, int Nx, int Ny, double Lx, double Ly, double g, double c,
                  double gamma, double nManning, int bc_x, int bc_y, int bathy_kind,
                  const double* bp, int n_par) {
  return or_create_points(P, Nx, Ny, Lx, Ly, g, c, gamma, nManning, bc_x, bc_y, bathy_kind,
                          bp, n_par, OR_POINTS_GLL);
}

or_ctx* or_create_points(int P, int Nx, int Ny, double Lx, double Ly, double g, double c,
                         double gamma, double nManning, int bc_x, int bc_y, int bathy_kind,
                         const double* bp, int n_par, int points) {
  try {
    auto* s = new or_ctx();
    s->Nx = Nx; s->Ny = Ny; s->np = P + 1; s->npp = (P + 1) * (P + 1);
    s->bcx = bc_x; s->bcy = bc_y;
    s->Nx2 = (bc_x == OR_BC_WALL) ? 2 * Nx : Nx;
    s->Ny2 = (bc_y == OR_BC_WALL) ? 2 * Ny : Ny;
    const double Lx2 = (bc_x == OR_BC_WALL) ? 2.0 * Lx : Lx;
    const double Ly2 = (bc_y == OR_BC_WALL) ? 2.0 * Ly : Ly;
    s->bpar.assign(bp, bp + (n_par > 0 ? n_par : 0));
    sgn2d::Params par;
    par.g = g; par.c = c; par.gamma = gamma; par.nManning = nManning;
    std::function<double(double, double)> depth;
    if (bathy_kind != OR_BATHY_NONE) {
      const int kind = bathy_kind;
      const std::vector<double>* pv = &s->bpar;
      depth = [kind, pv](double x, double y) { return or_bathy_eval(kind, pv->data(), x, y); };
    }
    const sgn::PointSet ps =
        points == OR_POINTS_GAUSS ? sgn::PointSet::GaussLegendre : sgn::PointSet::GaussLobatto;
    s->sys.reset(new sgn::SGN2D(P, s->Nx2, s->Ny2, Lx2, Ly2, par, depth, ps));
    return s;
  } catch (...) {
    return nullptr;
  }
}

void or_destroy(or_ctx* s) { delete s; }

/* [reference only] the reference's 1D solver (src/solver/sgn1d.h:47-94) on N periodic
 * elements of length L with a flat bottom: dU1 = R1(U1), var-major (h, hu, hw, hp),
 * (P + 1) N nodes per field. The 2D <-> 1D embedding gates of test/test_sgn2d.cpp:79-157
 * compare the 2D right-hand side of x- or y-invariant states with it. Returns 0. */
int or_rhs_1d(int P, int N, double L, double g, double c, double gamma, const double* U1,
              double* dU1) {
  sgn::Params par;
  par.g = g; par.c = c; par.gamma = gamma;
  sgn::SGN1D s1(P, N, L, par);
  sgn::State U(U1, U1 + (size_t)s1.nTotal()), R;
  s1.rhs(U, R);
  std::memcpy(dU1, R.data(), R.size() * sizeof(double));
  return 0;
}

/* [reference only] the reference's VTK frame writer (src/io/vtk2d.h) on a periodic
 * domain; returns 0, or -1 when the domain has walls (mirror doubling would write the
 * doubled domain). */
int or_write_vtk(const or_ctx* s, const double* U, const char* path) {
  if (s->bcx || s->bcy) return -1;
  sgn::State Us(U, U + (size_t)sgn2d::NVAR * s->sys->nDof());
  sgn::writeVtk2D(*s->sys, Us, path);
  return 0;
}

long or_ndof(const or_ctx* s) { return s->ndof(); }

void or_tables(const or_ctx* s, double* nodes, double* D, double* lL, double* lR,
               double* gLp, double* gRp, double* qw) {
  const auto& op = s->sys->ops();
  auto cp = [](const std::vector<double>& v, double* o) {
    if (o) std::memcpy(o, v.data(), v.size() * sizeof(double));
  };
  cp(op.nodes(), nodes); cp(op.D(), D); cp(op.lL(), lL); cp(op.lR(), lR);
  cp(op.gLprime(), gLp); cp(op.gRprime(), gRp); cp(op.weights(), qw);
}

void or_bathymetry(const or_ctx* s, double* Hnod, double* Hx, double* Hy, double* HfaceX,
                   double* HfaceY, double* HfaceXEnd, double* HfaceYEnd) {
  const int np = s->np, npp = s->npp;
  const auto& sys = *s->sys;
  for (int ey = 0; ey < s->Ny; ++ey)
    for (int ex = 0; ex < s->Nx; ++ex) {
      const long e = ex + (long)s->Nx * ey, e2 = ex + (long)s->Nx2 * ey;
      for (int k = 0; k < npp; ++k) {
        if (Hnod) Hnod[e * npp + k] = sys.stillDepthNodal()[e2 * npp + k];
        if (Hx) Hx[e * npp + k] = sys.stillDepthGradX()[e2 * npp + k];
        if (Hy) Hy[e * npp + k] = sys.stillDepthGradY()[e2 * npp + k];
      }
      for (int t = 0; t < np; ++t) {
        if (HfaceX) HfaceX[e * np + t] = sys.stillDepthFaceX()[e2 * np + t];
        if (HfaceY) HfaceY[e * np + t] = sys.stillDepthFaceY()[e2 * np + t];
      }
    }
  // right / top domain edges: the left / bottom edge of the element just beyond the
  // original domain, which exists only in the doubled domain
  for (int ey = 0; ey < s->Ny; ++ey)
    for (int t = 0; t < np; ++t)
      if (HfaceXEnd)
        HfaceXEnd[ey * np + t] = (s->bcx == OR_BC_WALL)
                                     ? sys.stillDepthFaceX()[(s->Nx + (long)s->Nx2 * ey) * np + t]
                                     : 0.0;
  for (int ex = 0; ex < s->Nx; ++ex)
    for (int t = 0; t < np; ++t)
      if (HfaceYEnd)
        HfaceYEnd[ex * np + t] = (s->bcy == OR_BC_WALL)
                                     ? sys.stillDepthFaceY()[(ex + (long)s->Nx2 * s->Ny) * np + t]
                                     : 0.0;
}

void or_node_coords(const or_ctx* s, double* x, double* y) {
  std::vector<double> xb, yb;
  s->sys->nodeCoords(xb, yb);
  for (int ey = 0; ey < s->Ny; ++ey)
    for (int ex = 0; ex < s->Nx; ++ex)
      for (int k = 0; k < s->npp; ++k) {
        const long e = ex + (long)s->Nx * ey, e2 = ex + (long)s->Nx2 * ey;
        x[e * s->npp + k] = xb[e2 * s->npp + k];
        y[e * s->npp + k] = yb[e2 * s->npp + k];
      }
}

int or_rhs(const or_ctx* s, const double* U, double* dU) {
  const_cast<or_ctx*>(s)->rhs(U, dU);
  return 0;
}

double or_max_wave_speed(const or_ctx* s, const double* U) {
  const long n = 5 * s->ndof();
  if (!s->doubled()) return s->sys->maxWaveSpeed(sgn::State(U, U + n));
  auto* m = const_cast<or_ctx*>(s);
  m->expand(U);
  return s->sys->maxWaveSpeed(m->Ubig);
}

double or_cfl_time_step(const or_ctx* s, const double* U, double cfl) {
  const long n = 5 * s->ndof();
  if (!s->doubled()) return s->sys->cflTimeStep(sgn::State(U, U + n), cfl);
  auto* m = const_cast<or_ctx*>(s);
  m->expand(U);
  return s->sys->cflTimeStep(m->Ubig, cfl);
}

double or_mass(const or_ctx* s, const double* U) {
  const long n = 5 * s->ndof();
  if (!s->doubled()) return s->sys->mass(sgn::State(U, U + n));
  return 0.0; // mass on a walled domain is not a reference quantity
}

double or_energy(const or_ctx* s, const double* U) {
  const long n = 5 * s->ndof();
  if (!s->doubled()) return s->sys->energy(sgn::State(U, U + n));
  return 0.0;
}

static sgn::RhsFn make_fn(const or_ctx* s) {
  auto* m = const_cast<or_ctx*>(s);
  return [m](double, const sgn::State& U, sgn::State& dU) {
    dU.resize(U.size());
    m->rhs(U.data(), dU.data());
  };
}

void or_rk4_step(const or_ctx* s, double t, double dt, double* U) {
  const long n = 5 * s->ndof();
  sgn::State u(U, U + n);
  sgn::rk4Step(make_fn(s), t, dt, u);
  std::memcpy(U, u.data(), n * sizeof(double));
}

void or_bs3_step(const or_ctx* s, double t, double dt, double* U) {
  const long n = 5 * s->ndof();
  sgn::State u(U, U + n);
  sgn::bs3Step(make_fn(s), t, dt, u);
  std::memcpy(U, u.data(), n * sizeof(double));
}

long or_integrate_adaptive(const or_ctx* s, double* U, double t0, double tEnd, double dt0,
                           const double* opts, double* stats, double* log, long max_log) {
  (void)log; (void)max_log;  // the reference loop exposes no per-attempt record
  const long n = 5 * s->ndof();
  sgn::AdaptiveRKOptions opt;
  opt.atol = opts[0]; opt.rtol = opts[1]; opt.dtMin = opts[2]; opt.dtMax = opts[3];
  opt.safety = opts[4]; opt.facMin = opts[5]; opt.facMax = opts[6];
  sgn::State u(U, U + n);
  const auto st = sgn::integrateAdaptive(make_fn(s), u, t0, tEnd, dt0, opt);
  std::memcpy(U, u.data(), n * sizeof(double));
  if (stats) {
    stats[0] = (double)st.accepted; stats[1] = (double)st.rejected;
    stats[2] = (double)st.rhsEvals; stats[3] = st.tReached; stats[4] = st.dtLast;
    stats[5] = st.maxNormLast; stats[6] = st.aborted ? 1.0 : 0.0;
  }
  return st.accepted + st.rejected;
}

}  // extern "C"
