// sgnb.hpp -- header-only C++ front end of libsgnb with the member signatures of the
// reference's single-GPU solver class sgn::SGN2DCuda (src/cuda/sgn2d_cuda.h:30-79).
//
// A reference caller switches by changing one include and one type name:
//
//   #include "cuda/sgn2d_cuda.h"          ->   #include "sgnb.hpp"
//   sgn::SGN2DCuda dev(host);             ->   sgnb::SGN2DB200 dev(host);
//   dev.upload(U); dev.rhsOnce(R);        (unchanged)
//   auto st = dev.integrateAdaptive(0.0, tEnd, dt0, opt);   (unchanged)
//
// The constructor takes the host solver object (a sgn::SGN2D or anything with the same
// accessors: order(), mesh(), params(), ops(), stillDepthNodal/GradX/GradY/FaceX/FaceY())
// and copies its FR tables and bathymetry arrays, exactly as the reference GPU solver
// builds itself from the host one (src/cuda/sgn2d_cuda.cu:318-400). State containers
// are any contiguous double container with data()/size()/resize() (sgn::State is
// std::vector<double>). Options and stats convert to and from the reference's
// sgn::AdaptiveRKOptions / AdaptiveRKStats by field name.
//
// Errors: the reference aborts the process on CUDA errors; this wrapper throws
// sgnb::Error carrying the status and the library's message instead.
#pragma once

#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "sgnb.h"

namespace sgnb {

class Error : public std::runtime_error {
 public:
  Error(int status, const std::string& msg)
      : std::runtime_error("sgnb: " + std::string(sgnb_status_string(status)) + ": " + msg),
        status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

// Field-for-field copy of sgn::AdaptiveRKOptions (src/solver/rk.h:53-61).
struct AdaptiveRKOptions {
  double atol = 1e-8, rtol = 1e-6, dtMin = 1e-13, dtMax = 1e30;
  double safety = 0.9, facMin = 0.2, facMax = 5.0;
  AdaptiveRKOptions() = default;
  template <class O>
  AdaptiveRKOptions(const O& o)  // NOLINT: implicit from the reference options
      : atol(o.atol), rtol(o.rtol), dtMin(o.dtMin), dtMax(o.dtMax), safety(o.safety),
        facMin(o.facMin), facMax(o.facMax) {}
};

// Field-for-field copy of sgn::AdaptiveRKStats (src/solver/rk.h:64-72), convertible to
// the reference type.
struct AdaptiveRKStats {
  long accepted = 0, rejected = 0, rhsEvals = 0;
  double tReached = 0.0, dtLast = 0.0, maxNormLast = 0.0;
  bool aborted = false;
  template <class S>
  operator S() const {  // NOLINT: implicit to the reference stats
    S s;
    s.accepted = accepted; s.rejected = rejected; s.rhsEvals = rhsEvals;
    s.tReached = tReached; s.dtLast = dtLast; s.maxNormLast = maxNormLast;
    s.aborted = aborted;
    return s;
  }
};

class SGN2DB200 {
 public:
  // Replaces SGN2DCuda(const SGN2D&): tables and bathymetry come from the host solver.
  template <class HostSolver>
  explicit SGN2DB200(const HostSolver& host, int precision = SGNB_FP64_EXACT, int device = 0,
                     int bc_x = SGNB_BC_PERIODIC, int bc_y = SGNB_BC_PERIODIC) {
    sgnb_desc d;
    sgnb_desc_init(&d);
    d.P = host.order();
    d.Nx = host.mesh().Nx;
    d.Ny = host.mesh().Ny;
    d.Lx = host.mesh().Lx;
    d.Ly = host.mesh().Ly;
    d.g = host.params().g;
    d.c = host.params().c;
    d.gamma = host.params().gamma;
    d.nManning = host.params().nManning;
    d.bc_x = bc_x;
    d.bc_y = bc_y;
    d.precision = precision;
    d.device = device;
    const auto& op = host.ops();
    d.nodes = op.nodes().data();
    d.D = op.D().data();
    d.lL = op.lL().data();
    d.lR = op.lR().data();
    d.gLp = op.gLprime().data();
    d.gRp = op.gRprime().data();
    d.qw = op.weights().data();
    d.bathy_kind = SGNB_BATHY_ARRAYS;
    d.Hnod = host.stillDepthNodal().data();
    d.Hx = host.stillDepthGradX().data();
    d.Hy = host.stillDepthGradY().data();
    d.HfaceX = host.stillDepthFaceX().data();
    d.HfaceY = host.stillDepthFaceY().data();
    check(sgnb_create(&d, &ctx_), nullptr);
  }
  // Built-in configuration (no host solver object).
  explicit SGN2DB200(const sgnb_desc& d) { check(sgnb_create(&d, &ctx_), nullptr); }
  ~SGN2DB200() { sgnb_destroy(ctx_); }
  SGN2DB200(const SGN2DB200&) = delete;
  SGN2DB200& operator=(const SGN2DB200&) = delete;

  int nDof() const { return (int)sgnb_ndof(ctx_); }
  int nTotal() const { return 5 * nDof(); }

  template <class State>
  void upload(const State& U) {
    if ((long long)U.size() != (long long)nTotal()) throw Error(SGNB_ERR_INVALID, "upload: size mismatch");
    check(sgnb_upload(ctx_, U.data()), ctx_);
  }
  template <class State>
  void download(State& U) const {
    U.resize(nTotal());
    check(sgnb_download(ctx_, U.data()), ctx_);
  }
  // One device RHS of the uploaded state, downloaded.
  template <class State>
  void rhsOnce(State& dU) {
    dU.resize(nTotal());
    check(sgnb_rhs_once(ctx_, dU.data()), ctx_);
  }
  // SGN2D::rhs for host states (the uploaded state is untouched).
  template <class State>
  void rhs(const State& U, State& dU) {
    if ((long long)U.size() != (long long)nTotal()) throw Error(SGNB_ERR_INVALID, "rhs: size mismatch");
    dU.resize(nTotal());
    check(sgnb_rhs_host(ctx_, U.data(), dU.data()), ctx_);
  }
  // rhs() in the shape of the reference's RhsFn, void(double t, const State&, State&)
  // (src/solver/rk.h:39), as SGN2D::rhsFn() offers it (src/solver/sgn2d.h:79-80): the
  // reference's host integrators (rk4Step, bs3Step, integrateAdaptive) then run with the
  // device right-hand side, each call copying the state in and the derivative out. t is
  // ignored. The returned callable refers to this object.
  std::function<void(double, const std::vector<double>&, std::vector<double>&)> rhsFn() {
    return [this](double, const std::vector<double>& U, std::vector<double>& dU) { rhs(U, dU); };
  }
  // rhs() for device pointers on a CUDA stream (0 = the context stream).
  void rhsDevice(const double* U, double* dU, void* stream = nullptr) {
    check(sgnb_rhs_device(ctx_, U, dU, stream), ctx_);
  }

  // Device-resident adaptive BS3(2) of the uploaded state (same controller as rk.cpp).
  AdaptiveRKStats integrateAdaptive(double t0, double tEnd, double dt0,
                                    const AdaptiveRKOptions& opt = AdaptiveRKOptions()) {
    sgnb_rk_opts o{opt.atol, opt.rtol, opt.dtMin, opt.dtMax, opt.safety, opt.facMin, opt.facMax};
    sgnb_rk_stats s{};
    const int rc = sgnb_integrate_adaptive(ctx_, t0, tEnd, dt0, &o, &s);
    if (rc != SGNB_OK && rc != SGNB_ERR_NAN) check(rc, ctx_);
    AdaptiveRKStats st;
    st.accepted = (long)s.accepted; st.rejected = (long)s.rejected; st.rhsEvals = (long)s.rhsEvals;
    st.tReached = s.tReached; st.dtLast = s.dtLast; st.maxNormLast = s.maxNormLast;
    st.aborted = s.aborted != 0;
    return st;
  }
  // Consecutive bs3Step calls with given step sizes (frozen-dt replay).
  void bs3Steps(double t0, const std::vector<double>& dts) {
    check(sgnb_bs3_steps(ctx_, t0, dts.data(), (long long)dts.size()), ctx_);
  }
  // Consecutive rk4Step calls with given step sizes (classical RK4; FP64 modes).
  void rk4Steps(double t0, const std::vector<double>& dts) {
    check(sgnb_rk4_steps(ctx_, t0, dts.data(), (long long)dts.size()), ctx_);
  }

  double mass() { return scalar(&sgnb_mass); }
  double energy() { return scalar(&sgnb_energy); }
  double maxWaveSpeed() { return scalar(&sgnb_max_wave_speed); }
  double cflTimeStep(double cfl) {
    double v = 0.0;
    check(sgnb_cfl_time_step(ctx_, cfl, &v), ctx_);
    return v;
  }
  sgnb_ctx* handle() { return ctx_; }

 private:
  static void check(int rc, const sgnb_ctx* c) {
    if (rc != SGNB_OK) throw Error(rc, sgnb_last_error(c));
  }
  double scalar(int (*fn)(sgnb_ctx*, double*)) {
    double v = 0.0;
    check(fn(ctx_, &v), ctx_);
    return v;
  }
  sgnb_ctx* ctx_ = nullptr;
};

}  // namespace sgnb
