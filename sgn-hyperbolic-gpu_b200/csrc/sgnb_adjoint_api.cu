// sgnb_adjoint_api.cu -- C ABI of the adjoint: gauge records of a frozen-dt BS3(2)
// trajectory and their vector-Jacobian product (no reference counterpart).
//
// Parameters: the bathymetry as element means (Nx * Ny, mapped to the depth statics by
// the bilinear cell interpolant, bathy kind 5 of sgnb_setup.cpp) and the initial free
// surface eta0 (Nd nodal values; h0 = H + eta0, zero velocity, w = p = 0).
// Forward: nsteps BS3(2) steps with the given step sizes (src/solver/rk.cpp:41-54 with
// the fused stage kernels of the solver context), recording eta = h - H at the gauge
// nodes after every step, with the state kept every `checkpoint_every` steps.
// Reverse: for each checkpoint segment, from the last to the first, the segment's
// states are recomputed from its checkpoint; then, step by step backwards, the stage
// derivatives k1, k2 are recomputed and the three right-hand-side VJPs of the step run
// (sgnb_adjoint.cu), carrying the state cotangent and accumulating the cotangents of
// the depth statics. The statics' cotangents map back to the element means through the
// transpose of the interpolant on the host.
#include "sgnb_ctx.h"

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

using namespace sgnb;

struct sgnb_adj {
  sgnb_ctx* c = nullptr;
  long long N = 0;
  int K = 0, ng = 0, nseg = 0;
  std::vector<double> dts;
  std::vector<long long> gnodes;
  std::vector<double> means;  // of the last forward
  bool haveForward = false;
  double* block = nullptr;    // every device buffer below lives in this allocation
  double* dts_dev = nullptr;
  long long* gnodes_dev = nullptr;
  double* ckpt = nullptr;     // nseg states
  double* seg = nullptr;      // K states
  double* u[2] = {nullptr, nullptr};
  double *k1 = nullptr, *k2 = nullptr, *k3 = nullptr;
  double *lam = nullptr, *acc = nullptr, *y3b = nullptr, *y2b = nullptr;
  double* eta_dev = nullptr;
  double* etab_dev = nullptr;
  CtrlState* ctrl = nullptr;
  VjpArgs V{};
  GatherArgs G{};
  size_t statBytes = 0;       // accumulators (contiguous from G.Hacc)
};

namespace {

int afail(sgnb_ctx* c, int code, const std::string& m) {
  if (c) c->err = m;
  return code;
}

#define SGNB_ACU(c, call)                                                                \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return afail(c, e_ == cudaErrorMemoryAllocation ? SGNB_ERR_NOMEM : SGNB_ERR_CUDA,  \
                   std::string(#call) + ": " + cudaGetErrorName(e_));                   \
  } while (0)

FrTablesDev tables_of(const sgnb_ctx* c) {
  FrTablesDev T{};
  for (int k = 0; k < 25; ++k) { T.D[k] = c->tab.D[k]; T.Df[k] = (float)c->tab.D[k]; }
  for (int k = 0; k < 5; ++k) {
    T.gLp[k] = c->tab.gLp[k]; T.gRp[k] = c->tab.gRp[k];
    T.gLpf[k] = (float)c->tab.gLp[k]; T.gRpf[k] = (float)c->tab.gRp[k];
  }
  return T;
}

cudaError_t fused(const sgnb_ctx* c, int mode, const StageArgs& A, cudaStream_t s) {
  return c->precision == SGNB_FP64_EXACT ? dev::launch_fused_exact(mode, c->C, A, s)
                                         : dev::launch_fused_fast(mode, c->C, A, s);
}

// Scratch of one right-hand-side VJP, carved from `p` (advanced past it).
size_t vjp_scratch_doubles(long long Nd, long long ne) {
  return 2 * 5 * (size_t)Nd + 2 * (size_t)Nd + 2 * (size_t)Nd + 4 * 25 * (size_t)ne + 4 * 5 * (size_t)ne;
}
void carve_vjp(VjpArgs& V, double*& p, long long Nd, long long ne) {
  for (int d = 0; d < 2; ++d) { V.Ub[d] = p; p += 5 * Nd; }
  for (int d = 0; d < 2; ++d) { V.Hb[d] = p; p += Nd; }
  V.Hxb = p; p += Nd;
  V.Hyb = p; p += Nd;
  for (int d = 0; d < 2; ++d)
    for (int f = 0; f < 2; ++f) { V.Sn[d][f] = p; p += 25 * ne; }
  for (int d = 0; d < 2; ++d)
    for (int f = 0; f < 2; ++f) { V.Hf[d][f] = p; p += 5 * ne; }
}
size_t stat_doubles(const sgnb_ctx* c) {
  const long long ne = (long long)c->desc.Nx * c->desc.Ny;
  return 3 * (size_t)c->Nd + 10 * (size_t)ne + 5 * (size_t)(c->desc.Nx + c->desc.Ny);
}
void carve_stats(GatherArgs& G, double*& p, const sgnb_ctx* c) {
  const long long ne = (long long)c->desc.Nx * c->desc.Ny;
  G.Hacc = p; p += c->Nd;
  G.Hxacc = p; p += c->Nd;
  G.Hyacc = p; p += c->Nd;
  G.HfXacc = p; p += 5 * ne;
  G.HfYacc = p; p += 5 * ne;
  G.HfXEndacc = p; p += 5 * c->desc.Ny;
  G.HfYEndacc = p; p += 5 * c->desc.Nx;
}
// device statics accumulators -> host Bathymetry of cotangents
cudaError_t download_stats(const sgnb_ctx* c, const GatherArgs& G, Bathymetry& bar) {
  const long long ne = (long long)c->desc.Nx * c->desc.Ny;
  bar.Hnod.resize(c->Nd); bar.Hx.resize(c->Nd); bar.Hy.resize(c->Nd);
  bar.HfX.resize(5 * ne); bar.HfY.resize(5 * ne);
  bar.HfXEnd.resize(5 * (size_t)c->desc.Ny); bar.HfYEnd.resize(5 * (size_t)c->desc.Nx);
  std::vector<double> all(stat_doubles(c));
  cudaError_t e = cudaMemcpy(all.data(), G.Hacc, all.size() * sizeof(double), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return e;
  const double* p = all.data();
  auto take = [&](std::vector<double>& v) { std::memcpy(v.data(), p, v.size() * sizeof(double)); p += v.size(); };
  take(bar.Hnod); take(bar.Hx); take(bar.Hy); take(bar.HfX); take(bar.HfY);
  take(bar.HfXEnd); take(bar.HfYEnd);
  return cudaSuccess;
}

// Replaces the context's depth statics.
cudaError_t upload_statics(sgnb_ctx* c, const Bathymetry& b) {
  auto put = [&](const std::vector<double>& v, const double* dst) {
    return cudaMemcpyAsync(const_cast<double*>(dst), v.data(), v.size() * sizeof(double),
                           cudaMemcpyHostToDevice, c->stream);
  };
  cudaError_t e = put(b.Hnod, c->C.Hnod);
  if (e == cudaSuccess) e = put(b.Hx, c->C.Hx);
  if (e == cudaSuccess) e = put(b.Hy, c->C.Hy);
  if (e == cudaSuccess) e = put(b.HfX, c->C.HfX);
  if (e == cudaSuccess) e = put(b.HfY, c->C.HfY);
  if (e == cudaSuccess) e = put(b.HfXEnd, c->C.HfXEnd);
  if (e == cudaSuccess) e = put(b.HfYEnd, c->C.HfYEnd);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  return e;
}

std::vector<double> cell_params(const sgnb_ctx* c, const double* means) {
  const long long nm = (long long)c->desc.Nx * c->desc.Ny;
  std::vector<double> p(4 + nm);
  p[0] = c->desc.Nx; p[1] = c->desc.Ny; p[2] = c->desc.Lx; p[3] = c->desc.Ly;
  std::memcpy(p.data() + 4, means, nm * sizeof(double));
  return p;
}

// One BS3(2) step u -> out at step index n (dt read from the device list).
int step(sgnb_adj* a, const double* u, double* out, long long n) {
  sgnb_ctx* c = a->c;
  cudaStream_t s = c->stream;
  SGNB_ACU(c, cudaMemcpyAsync(&a->ctrl->dt, a->dts_dev + n, sizeof(double), cudaMemcpyDeviceToDevice, s));
  StageArgs A{};
  A.U[0] = A.U[1] = const_cast<double*>(u);
  A.K1[0] = A.K1[1] = a->k1;
  A.K2 = a->k2;
  A.K3 = a->k3;
  A.ctrl = a->ctrl;
  A.partials = c->partials;
  A.in = u;
  A.out = a->k1;
  SGNB_ACU(c, fused(c, 0, A, s));
  A.kin_k2 = 0; A.coef = 0.5; A.out = a->k2;
  SGNB_ACU(c, fused(c, 1, A, s));
  A.kin_k2 = 1; A.coef = 0.75; A.out = a->k3;
  SGNB_ACU(c, fused(c, 1, A, s));
  SGNB_ACU(c, dev::launch_rk_update(u, a->k1, a->k2, a->k3, a->dts_dev, n, out, c->ntot, s));
  return SGNB_OK;
}

}  // namespace

extern "C" {

int sgnb_adj_create(sgnb_ctx* c, long long nsteps, const double* dts, int ngauges,
                    const long long* gauge_nodes, int checkpoint_every, sgnb_adj** out) {
  if (!c || !out || nsteps < 1 || !dts || ngauges < 0 || (ngauges > 0 && !gauge_nodes) ||
      checkpoint_every < 1)
    return afail(c, SGNB_ERR_INVALID, "sgnb_adj_create: bad arguments");
  *out = nullptr;
  if (c->mixed) return afail(c, SGNB_ERR_UNSUPPORTED, "the adjoint runs in FP64 modes");
  if (c->desc.Nx_global > 0 || c->C.ghostL || c->C.ghostR)
    return afail(c, SGNB_ERR_UNSUPPORTED, "the adjoint runs on whole meshes");
  if (c->tab.gauss) return afail(c, SGNB_ERR_UNSUPPORTED, "the adjoint runs on GLL points");
  for (int g = 0; g < ngauges; ++g)
    if (gauge_nodes[g] < 0 || gauge_nodes[g] >= c->Nd)
      return afail(c, SGNB_ERR_INVALID, "gauge node out of range");
  for (long long n = 0; n < nsteps; ++n)
    if (!(dts[n] > 0.0)) return afail(c, SGNB_ERR_INVALID, "step sizes must be > 0");
  SGNB_ACU(c, cudaSetDevice(c->device));
  sgnb_adj* a = new sgnb_adj();
  a->c = c;
  a->N = nsteps;
  a->K = checkpoint_every;
  a->ng = ngauges;
  a->nseg = (int)((nsteps + checkpoint_every - 1) / checkpoint_every);
  a->dts.assign(dts, dts + nsteps);
  a->gnodes.assign(gauge_nodes, gauge_nodes + ngauges);
  const long long S = c->ntot, Nd = c->Nd, ne = (long long)c->desc.Nx * c->desc.Ny;
  const long long segStates = (a->K < nsteps) ? a->K : nsteps;
  size_t total = nsteps + (size_t)ngauges + 2 * (size_t)nsteps * (ngauges > 0 ? ngauges : 1) +
                 ((size_t)a->nseg + segStates + 9) * S + vjp_scratch_doubles(Nd, ne) +
                 stat_doubles(c) + sizeof(CtrlState) / sizeof(double) + 8;
  cudaError_t e = cudaMalloc(&a->block, total * sizeof(double));
  if (e != cudaSuccess) { delete a; return afail(c, SGNB_ERR_NOMEM, "sgnb_adj_create: cudaMalloc"); }
  double* p = a->block;
  a->ctrl = reinterpret_cast<CtrlState*>(p); p += (sizeof(CtrlState) + 7) / 8 + 1;
  a->dts_dev = p; p += nsteps;
  a->gnodes_dev = reinterpret_cast<long long*>(p); p += ngauges;
  a->eta_dev = p; p += (size_t)nsteps * (ngauges > 0 ? ngauges : 1);
  a->etab_dev = p; p += (size_t)nsteps * (ngauges > 0 ? ngauges : 1);
  a->ckpt = p; p += (size_t)a->nseg * S;
  a->seg = p; p += (size_t)segStates * S;
  for (double** q : {&a->u[0], &a->u[1], &a->k1, &a->k2, &a->k3, &a->lam, &a->acc, &a->y3b, &a->y2b}) {
    *q = p;
    p += S;
  }
  carve_vjp(a->V, p, Nd, ne);
  carve_stats(a->G, p, c);
  e = cudaMemset(a->ctrl, 0, sizeof(CtrlState));
  if (e == cudaSuccess) e = cudaMemcpy(a->dts_dev, dts, nsteps * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && ngauges > 0)
    e = cudaMemcpy(a->gnodes_dev, gauge_nodes, ngauges * sizeof(long long), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(a->block);
    delete a;
    return afail(c, SGNB_ERR_CUDA, "sgnb_adj_create: upload");
  }
  *out = a;
  return SGNB_OK;
}

int sgnb_adj_destroy(sgnb_adj* a) {
  if (!a) return SGNB_OK;
  cudaSetDevice(a->c->device);
  cudaStreamSynchronize(a->c->stream);
  cudaFree(a->block);
  delete a;
  return SGNB_OK;
}

int sgnb_adj_forward(sgnb_adj* a, const double* means, const double* eta0, double* eta_out) {
  if (!a || !means || !eta0) return afail(a ? a->c : nullptr, SGNB_ERR_INVALID, "NULL argument");
  sgnb_ctx* c = a->c;
  SGNB_ACU(c, cudaSetDevice(c->device));
  cudaStream_t s = c->stream;
  const long long Nd = c->Nd, S = c->ntot;
  // statics from the element means (host set-up, as at context creation)
  a->means.assign(means, means + (long long)c->desc.Nx * c->desc.Ny);
  const std::vector<double> p = cell_params(c, means);
  Bathymetry b;
  bathymetry(c->mesh, c->tab, 5, p.data(), b);
  SGNB_ACU(c, upload_statics(c, b));
  // u0 = (H + eta0, 0, 0, 0, 0)
  std::vector<double> u0(S, 0.0);
  for (long long i = 0; i < Nd; ++i) u0[i] = b.Hnod[i] + eta0[i];
  SGNB_ACU(c, cudaMemcpyAsync(a->u[0], u0.data(), S * sizeof(double), cudaMemcpyHostToDevice, s));
  int cur = 0;
  for (long long n = 0; n < a->N; ++n) {
    if (n % a->K == 0)
      SGNB_ACU(c, cudaMemcpyAsync(a->ckpt + (n / a->K) * S, a->u[cur], S * sizeof(double),
                                  cudaMemcpyDeviceToDevice, s));
    if (int rc = step(a, a->u[cur], a->u[cur ^ 1], n)) return rc;
    cur ^= 1;
    if (a->ng > 0)
      SGNB_ACU(c, dev::launch_gauges(a->u[cur], c->C.Hnod, a->gnodes_dev, a->ng,
                                     a->eta_dev + n * a->ng, s));
  }
  // the context holds the final state
  SGNB_ACU(c, cudaMemcpyAsync(c->U[c->cur], a->u[cur], S * sizeof(double), cudaMemcpyDeviceToDevice, s));
  if (eta_out && a->ng > 0)
    SGNB_ACU(c, cudaMemcpyAsync(eta_out, a->eta_dev, a->N * a->ng * sizeof(double),
                                cudaMemcpyDeviceToHost, s));
  SGNB_ACU(c, cudaStreamSynchronize(s));
  a->haveForward = true;
  return SGNB_OK;
}

int sgnb_adj_vjp(sgnb_adj* a, const double* eta_bar, double* grad_means, double* grad_eta0) {
  if (!a || !eta_bar) return afail(a ? a->c : nullptr, SGNB_ERR_INVALID, "NULL argument");
  sgnb_ctx* c = a->c;
  if (!a->haveForward) return afail(c, SGNB_ERR_INVALID, "sgnb_adj_vjp before sgnb_adj_forward");
  SGNB_ACU(c, cudaSetDevice(c->device));
  cudaStream_t s = c->stream;
  const long long S = c->ntot, Nd = c->Nd;
  const int ng = a->ng;
  if (ng > 0)
    SGNB_ACU(c, cudaMemcpyAsync(a->etab_dev, eta_bar, a->N * ng * sizeof(double),
                                cudaMemcpyHostToDevice, s));
  SGNB_ACU(c, cudaMemsetAsync(a->G.Hacc, 0, stat_doubles(c) * sizeof(double), s));
  SGNB_ACU(c, cudaMemsetAsync(a->lam, 0, S * sizeof(double), s));
  if (ng > 0)
    SGNB_ACU(c, dev::launch_gauges_back(a->lam, a->gnodes_dev, ng, a->etab_dev + (a->N - 1) * ng, s));
  const FrTablesDev T = tables_of(c);
  double* lam = a->lam;
  double* acc = a->acc;
  for (int sg = a->nseg - 1; sg >= 0; --sg) {
    const long long n0 = (long long)sg * a->K;
    const long long n1 = (n0 + a->K < a->N) ? n0 + a->K : a->N;
    // recompute the segment's states u_n0 .. u_{n1-1}
    SGNB_ACU(c, cudaMemcpyAsync(a->seg, a->ckpt + sg * S, S * sizeof(double), cudaMemcpyDeviceToDevice, s));
    for (long long n = n0; n + 1 < n1; ++n)
      if (int rc = step(a, a->seg + (n - n0) * S, a->seg + (n + 1 - n0) * S, n)) return rc;
    for (long long n = n1 - 1; n >= n0; --n) {
      const double* u = a->seg + (n - n0) * S;
      const double dt = a->dts[n];
      // k1 = R(u), k2 = R(u + dt/2 k1)
      SGNB_ACU(c, cudaMemcpyAsync(&a->ctrl->dt, a->dts_dev + n, sizeof(double), cudaMemcpyDeviceToDevice, s));
      StageArgs A{};
      A.U[0] = A.U[1] = const_cast<double*>(u);
      A.K1[0] = A.K1[1] = a->k1;
      A.K2 = a->k2;
      A.K3 = a->k3;
      A.ctrl = a->ctrl;
      A.partials = c->partials;
      A.in = u;
      A.out = a->k1;
      SGNB_ACU(c, fused(c, 0, A, s));
      A.kin_k2 = 0; A.coef = 0.5; A.out = a->k2;
      SGNB_ACU(c, fused(c, 1, A, s));
      // u_{n+1} = u + dt (2/9 k1 + 1/3 k2 + 4/9 k3), k3 = R(u + 3dt/4 k2), k2 = R(u + dt/2 k1)
      VjpArgs V = a->V;
      GatherArgs G = a->G;
      V.u = u;
      V.k = a->k2; V.acoef = 0.75 * dt;
      V.ra = lam; V.rb = nullptr; V.alpha = (4.0 / 9.0) * dt; V.beta = 0.0;
      G.ybar = a->y3b; G.uacc = acc; G.lam = lam; G.init = 1;
      SGNB_ACU(c, dev::launch_vjp_rhs(c->C, T, V, G, s));
      V.k = a->k1; V.acoef = 0.5 * dt;
      V.ra = lam; V.rb = a->y3b; V.alpha = dt / 3.0; V.beta = 0.75 * dt;
      G.ybar = a->y2b; G.init = 0; G.lam = nullptr;
      SGNB_ACU(c, dev::launch_vjp_rhs(c->C, T, V, G, s));
      V.k = nullptr; V.acoef = 0.0;
      V.ra = lam; V.rb = a->y2b; V.alpha = (2.0 / 9.0) * dt; V.beta = 0.5 * dt;
      G.ybar = nullptr;
      SGNB_ACU(c, dev::launch_vjp_rhs(c->C, T, V, G, s));
      double* t = lam; lam = acc; acc = t;
      if (n >= 1 && ng > 0)
        SGNB_ACU(c, dev::launch_gauges_back(lam, a->gnodes_dev, ng, a->etab_dev + (n - 1) * ng, s));
    }
  }
  // lam = dL/du0; h0 = H + eta0
  std::vector<double> lh(Nd);
  SGNB_ACU(c, cudaMemcpyAsync(lh.data(), lam, Nd * sizeof(double), cudaMemcpyDeviceToHost, s));
  SGNB_ACU(c, cudaStreamSynchronize(s));
  if (grad_eta0) std::memcpy(grad_eta0, lh.data(), Nd * sizeof(double));
  if (grad_means) {
    Bathymetry bar;
    SGNB_ACU(c, download_stats(c, a->G, bar));
    for (long long i = 0; i < Nd; ++i) bar.Hnod[i] += lh[i];
    for (long long n = 0; n < a->N; ++n)
      for (int g = 0; g < ng; ++g) bar.Hnod[a->gnodes[g]] -= eta_bar[n * ng + g];  // eta = h - H
    const std::vector<double> p = cell_params(c, a->means.data());
    cells_transpose(c->mesh, c->tab, p.data(), bar, grad_means);
  }
  return SGNB_OK;
}

int sgnb_rhs_vjp(sgnb_ctx* c, const double* U, const double* Rbar, double* Ubar,
                 double* Hnod_bar, double* Hx_bar, double* Hy_bar, double* HfX_bar,
                 double* HfY_bar, double* HfXEnd_bar, double* HfYEnd_bar) {
  if (!c || !U || !Rbar || !Ubar) return afail(c, SGNB_ERR_INVALID, "NULL argument");
  if (c->mixed) return afail(c, SGNB_ERR_UNSUPPORTED, "the adjoint runs in FP64 modes");
  SGNB_ACU(c, cudaSetDevice(c->device));
  cudaStream_t s = c->stream;
  const long long S = c->ntot, Nd = c->Nd, ne = (long long)c->desc.Nx * c->desc.Ny;
  double* block = nullptr;
  const size_t total = 3 * (size_t)S + vjp_scratch_doubles(Nd, ne) + stat_doubles(c);
  SGNB_ACU(c, cudaMalloc(&block, total * sizeof(double)));
  double* p = block;
  double* Ud = p; p += S;
  double* Rd = p; p += S;
  double* Ubd = p; p += S;
  VjpArgs V{};
  GatherArgs G{};
  carve_vjp(V, p, Nd, ne);
  carve_stats(G, p, c);
  cudaError_t e = cudaMemcpyAsync(Ud, U, S * sizeof(double), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(Rd, Rbar, S * sizeof(double), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(G.Hacc, 0, stat_doubles(c) * sizeof(double), s);
  V.u = Ud; V.k = nullptr; V.acoef = 0.0;
  V.ra = Rd; V.rb = nullptr; V.alpha = 1.0; V.beta = 0.0;
  G.ybar = nullptr; G.uacc = Ubd; G.lam = nullptr; G.init = 1;
  if (e == cudaSuccess) e = dev::launch_vjp_rhs(c->C, tables_of(c), V, G, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(Ubar, Ubd, S * sizeof(double), cudaMemcpyDeviceToHost, s);
  Bathymetry bar;
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = download_stats(c, G, bar);
  cudaFree(block);
  if (e != cudaSuccess) return afail(c, SGNB_ERR_CUDA, std::string("sgnb_rhs_vjp: ") + cudaGetErrorName(e));
  auto out = [](const std::vector<double>& v, double* o) {
    if (o) std::memcpy(o, v.data(), v.size() * sizeof(double));
  };
  out(bar.Hnod, Hnod_bar); out(bar.Hx, Hx_bar); out(bar.Hy, Hy_bar); out(bar.HfX, HfX_bar);
  out(bar.HfY, HfY_bar); out(bar.HfXEnd, HfXEnd_bar); out(bar.HfYEnd, HfYEnd_bar);
  return SGNB_OK;
}

}  // extern "C"
