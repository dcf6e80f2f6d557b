// sgnb_ctx.h -- the solver context behind the C ABI's opaque sgnb_ctx (internal).
#pragma once

#include <string>

#include "sgnb.h"
#include "sgnb_device.h"
#include "sgnb_setup.h"

// One solver on one device: the bathymetry statics (one allocation, Hbuf: Hnod, Hx, Hy
// (Nd each), HfX, HfY (5 ne each), HfXEnd (5 Ny), HfYEnd (5 Nx); the RhsConsts C holds the
// pointers), the state ping-pong pair U[2], the FSAL pair K1[2] (k1 / k4), the stage
// derivatives K2, K3, the per-CTA error partials and the device-resident controller state.
struct sgnb_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  sgnb_desc desc{};
  int precision = SGNB_FP64_EXACT;
  sgnb::Mesh mesh;
  sgnb::FrTables tab;
  long long Nd = 0, ntot = 0;
  sgnb::RhsConsts C{};
  sgnb::TileMaps maps{};  // tensor maps of U, K1, K2, K3, Hnod (FP64 modes, whole tiles)
  sgnb::TileMapsM mapsM{};  // the mixed mode's (FP32 K1, K2, K3; Hnod)
  void* encode_tiled = nullptr;  // the driver's tensor-map encoder (set with the maps)
  double* Hbuf = nullptr;  // one allocation holding all statics
  double* trbuf = nullptr;  // Gauss points: face traces, 4 faces x 5 fields x 5 ne
  double* U[2] = {nullptr, nullptr};
  // stage derivatives: FP64 (exact / fast) or FP32 (mixed precision)
  void* K1[2] = {nullptr, nullptr};
  void* K2 = nullptr;
  void* K3 = nullptr;
  bool mixed = false;
  double* partials = nullptr;
  int nblk = 0;
  double* diag = nullptr;  // diagnostic partials
  int ndiag = 0;
  sgnb::CtrlState* dctrl = nullptr;
  sgnb::CtrlState* hctrl = nullptr;  // pinned mirror
  double* dtList = nullptr;
  long long dtCap = 0;
  double* alog = nullptr;  // device attempt log of the last integration
  static constexpr long long kLogCap = 1 << 16;
  cudaGraphExec_t chunk = nullptr;
  int chunkLen = 0;
  cudaEvent_t evRead = nullptr;
  long long launches = 0;  // kernels launched by the last integration
  long long pendingMaxAccepted = 0;  // set by sgnb_integrate_steps
  double* gauge = nullptr;  // gauge sampling: nodes then values, grown on demand
  int gaugeCap = 0;
  int cur = 0;
  std::string err;
};
