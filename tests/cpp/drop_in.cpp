// drop_in.cpp -- the reference's host solver driving libsgnb through sgnb.hpp.
//
// TEST INFRASTRUCTURE. Built against the reference sources (sgn::SGN2D, the rk.h
// integrators) by tests/cpp/Makefile into oracle/_ref/drop_in, and run on a GPU box by
// tests/test_drop_in_gpu.py. It shows a reference caller switching from
// sgn::SGN2DCuda to sgnb::SGN2DB200 with no other change, and checks, on the parity case
// of the reference's GPU test (8 x 6 elements over a Gaussian bump):
//   1. the device rhs equals SGN2D::rhs bit for bit (exact mode);
//   2. lake at rest: max |rhs| < 1e-12;
//   3. an adaptive run (tEnd 0.3, atol 1e-10, rtol 1e-8) takes the CPU's accepted /
//      rejected steps, ends within 1e-10 relative of the CPU state and conserves mass;
//   4. a host solver on Gauss-Legendre points (flat bottom): its tables reach the device
//      through the same constructor, and the device rhs equals SGN2D::rhs bit for bit;
//   5. three fixed steps: the device's rk4Steps / bs3Steps equal the reference's rk4Step /
//      bs3Step over host.rhsFn() bit for bit, and the reference's rk4Step over the device
//      right-hand side (dev.rhsFn()) equals it too.
// Prints one line per check and exits non-zero on any failure.
#include "sgnb.hpp"

#include "solver/rk.h"
#include "solver/sgn2d.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

static int failures = 0;
static void report(bool ok, const char* what, double value) {
  std::printf("%s %-52s %.3e\n", ok ? "PASS" : "FAIL", what, value);
  if (!ok) ++failures;
}

int main() {
  const double kPi = 3.14159265358979323846;
  sgn2d::Params par;
  par.g = 9.81;
  par.gamma = 1.5;
  par.c = 3.0 * std::sqrt(9.81);
  const double Lx = 10.0, Ly = 8.0;
  auto depth = [=](double x, double y) {
    const double dx = x - 0.5 * Lx, dy = y - 0.5 * Ly;
    return 1.0 - 0.4 * std::exp(-(dx * dx + dy * dy) / 6.0);
  };
  sgn::SGN2D host(4, 8, 6, Lx, Ly, par, depth);
  std::vector<double> x, y;
  host.nodeCoords(x, y);
  const int Nd = host.nDof();
  std::vector<double> h(Nd), u(Nd), v(Nd), w(Nd), p(Nd);
  for (int i = 0; i < Nd; ++i) {
    const double sx = std::sin(2 * kPi * x[i] / Lx), cy = std::cos(2 * kPi * y[i] / Ly);
    h[i] = depth(x[i], y[i]) + 0.04 * sx * cy;
    u[i] = 0.08 * std::cos(2 * kPi * x[i] / Lx);
    v[i] = -0.05 * std::sin(2 * kPi * y[i] / Ly);
    w[i] = 0.02 * sx;
    p[i] = 0.01 * cy;
  }
  const sgn::State U = host.makeState(h, u, v, w, p);

  {  // 1. rhs
    sgn::State Rc, Rg;
    host.rhs(U, Rc);
    sgnb::SGN2DB200 dev(host);
    dev.upload(U);
    dev.rhsOnce(Rg);
    const bool same = Rc.size() == Rg.size() &&
                      std::memcmp(Rc.data(), Rg.data(), Rc.size() * sizeof(double)) == 0;
    double diff = 0.0;
    for (size_t i = 0; i < Rc.size(); ++i) diff = std::fmax(diff, std::fabs(Rc[i] - Rg[i]));
    report(same, "device rhs == SGN2D::rhs bit for bit", diff);
  }
  {  // 2. lake at rest
    std::vector<double> z(Nd, 0.0);
    const sgn::State Ur = host.makeState(host.stillDepthNodal(), z, z, z, z);
    sgnb::SGN2DB200 dev(host);
    dev.upload(Ur);
    sgn::State R;
    dev.rhsOnce(R);
    double m = 0.0;
    for (double r : R) m = std::fmax(m, std::fabs(r));
    report(m < 1e-12, "lake at rest on the device: max |rhs|", m);
  }
  {  // 3. adaptive run
    sgn::AdaptiveRKOptions opt;
    opt.atol = 1e-10;
    opt.rtol = 1e-8;
    const double dt0 = host.cflTimeStep(U, 0.5);
    sgn::State Uh = U;
    const sgn::AdaptiveRKStats sh = sgn::integrateAdaptive(host.rhsFn(), Uh, 0.0, 0.3, dt0, opt);
    sgnb::SGN2DB200 dev(host);
    dev.upload(U);
    const sgn::AdaptiveRKStats sg = dev.integrateAdaptive(0.0, 0.3, dt0, opt);
    sgn::State Ug;
    dev.download(Ug);
    double diff = 0.0, scale = 0.0;
    for (size_t i = 0; i < Uh.size(); ++i) {
      diff = std::fmax(diff, std::fabs(Uh[i] - Ug[i]));
      scale = std::fmax(scale, std::fabs(Uh[i]));
    }
    report(sg.accepted == sh.accepted && sg.rejected == sh.rejected && !sg.aborted,
           "adaptive run: same accepted / rejected steps", (double)sg.accepted);
    report(diff / scale < 1e-10, "adaptive run: state vs CPU (relative)", diff / scale);
    const double dM = std::fabs(host.mass(Ug) - host.mass(U)) / std::fabs(host.mass(U));
    report(dM < 1e-13, "adaptive run: mass conserved", dM);
  }
  {  // 4. Gauss-Legendre points on a flat bottom (H = 0)
    sgn::SGN2D gauss(4, 7, 5, 8.75, 6.5, par, {}, sgn::PointSet::GaussLegendre);
    std::vector<double> xg, yg;
    gauss.nodeCoords(xg, yg);
    const int Ng = gauss.nDof();
    std::vector<double> hg(Ng), ug(Ng), vg(Ng), wg(Ng), pg(Ng);
    for (int i = 0; i < Ng; ++i) {
      hg[i] = 1.0 + 0.04 * std::sin(2 * kPi * xg[i] / 8.75) * std::cos(2 * kPi * yg[i] / 6.5);
      ug[i] = 0.08 * std::cos(2 * kPi * xg[i] / 8.75);
      vg[i] = -0.05 * std::sin(2 * kPi * yg[i] / 6.5);
      wg[i] = 0.02 * std::sin(xg[i]);
      pg[i] = 0.01 * std::cos(yg[i]);
    }
    const sgn::State Ug = gauss.makeState(hg, ug, vg, wg, pg);
    sgn::State Rc, Rg;
    gauss.rhs(Ug, Rc);
    sgnb::SGN2DB200 dev(gauss);
    dev.upload(Ug);
    dev.rhsOnce(Rg);
    const bool same = Rc.size() == Rg.size() &&
                      std::memcmp(Rc.data(), Rg.data(), Rc.size() * sizeof(double)) == 0;
    double diff = 0.0;
    for (size_t i = 0; i < Rc.size() && i < Rg.size(); ++i)
      diff = std::fmax(diff, std::fabs(Rc[i] - Rg[i]));
    report(same, "Gauss points: device rhs == SGN2D::rhs bit for bit", diff);
  }
  {  // 5. fixed steps: the reference's rk4Step and bs3Step over rhsFn() against the device's
    const double dt = host.cflTimeStep(U, 0.5);
    const std::vector<double> dts = {dt, 0.8 * dt, dt};
    sgn::State U4 = U, U3 = U;
    double t = 0.0;
    for (double d : dts) {
      sgn::rk4Step(host.rhsFn(), t, d, U4);
      sgn::bs3Step(host.rhsFn(), t, d, U3);
      t += d;
    }
    sgnb::SGN2DB200 dev(host);
    sgn::State G4, G3;
    dev.upload(U);
    dev.rk4Steps(0.0, dts);
    dev.download(G4);
    dev.upload(U);
    dev.bs3Steps(0.0, dts);
    dev.download(G3);
    auto maxdiff = [](const sgn::State& a, const sgn::State& b) {
      double d = 0.0;
      for (size_t i = 0; i < a.size() && i < b.size(); ++i) d = std::fmax(d, std::fabs(a[i] - b[i]));
      return d;
    };
    report(G4.size() == U4.size() && std::memcmp(G4.data(), U4.data(), U4.size() * sizeof(double)) == 0,
           "3 x rk4Step: device == reference bit for bit", maxdiff(G4, U4));
    report(G3.size() == U3.size() && std::memcmp(G3.data(), U3.data(), U3.size() * sizeof(double)) == 0,
           "3 x bs3Step: device == reference bit for bit", maxdiff(G3, U3));
    // the reference's own rk4Step driving the device right-hand side through rhsFn()
    sgn::State H4 = U;
    t = 0.0;
    for (double d : dts) {
      sgn::rk4Step(dev.rhsFn(), t, d, H4);
      t += d;
    }
    report(std::memcmp(H4.data(), U4.data(), U4.size() * sizeof(double)) == 0,
           "rk4Step over dev.rhsFn() == over host.rhsFn()", maxdiff(H4, U4));
  }
  std::printf(failures ? "%d FAILED\n" : "ALL PASSED\n", failures);
  return failures ? 1 : 0;
}
