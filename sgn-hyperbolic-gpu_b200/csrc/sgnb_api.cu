// sgnb_api.cu -- implementation of the C ABI declared in include/sgnb.h.
//
// The context owns the device state of one solver: the bathymetry statics, the state
// ping-pong pair U[2], the FSAL pair K1[2] (k1 / k4), the stage derivatives K2, K3,
// the per-CTA error partials and the device-resident controller state. An adaptive
// integration is a device-side loop: a CUDA graph whose WHILE conditional node repeats one
// attempt (stage 2, stage 3, end-point stage, controller) until the controller clears the
// condition; the host reads the controller back once per graph launch instead of once per
// step (the reference copies error partials to the host every step,
// src/cuda/sgn2d_cuda.cu:506-516).
#include "sgnb_ctx.h"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace sgnb;


namespace {

thread_local std::string g_create_error;

int fail(sgnb_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg; else g_create_error = msg;
  return code;
}

int cuda_fail(sgnb_ctx* c, cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  return fail(c, e == cudaErrorMemoryAllocation ? SGNB_ERR_NOMEM : SGNB_ERR_CUDA, m);
}

#define SGNB_CU(ctx, call)                          \
  do {                                              \
    cudaError_t e_ = (call);                        \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
  } while (0)

// One fused launch: mode 0 rhs (in -> out), 1 stage (u + coef dt k -> K2 or K3),
// 2 end-point stage. Dispatches on the arithmetic mode of the context.
struct Launch {
  int mode = 0;
  const double* in = nullptr;  // mode 0
  double* out = nullptr;       // mode 0
  int stage = 2;               // mode 1: 2 (k1 -> K2) or 3 (k2 -> K3)
};

static bool encode_state_map(const sgnb_ctx* c, CUtensorMap* m, const void* p,
                             CUtensorMapDataType type, size_t elem, cuuint32_t nz);

cudaError_t launch(sgnb_ctx* c, const Launch& L, cudaStream_t s) {
  if (c->mixed) {
    StageArgsM A{};
    A.U[0] = c->U[0]; A.U[1] = c->U[1];
    A.K1[0] = (float*)c->K1[0]; A.K1[1] = (float*)c->K1[1];
    A.K2 = (float*)c->K2; A.K3 = (float*)c->K3;
    A.ctrl = c->dctrl;
    A.partials = c->partials;
    A.in = L.in;
    A.outd = L.out;
    A.kin_k2 = L.stage == 3;
    A.coef = L.stage == 3 ? 0.75 : 0.5;
    if (L.mode == 0) A.out = L.out ? nullptr : A.K1[c->cur];  // no FP64 output: the FSAL head
    else A.out = L.stage == 3 ? A.K3 : A.K2;
    return dev::launch_fused_mixed(L.mode, c->C, A, s, c->mapsM.ok ? &c->mapsM : nullptr);
  }
  StageArgs A{};
  A.U[0] = c->U[0]; A.U[1] = c->U[1];
  A.K1[0] = (double*)c->K1[0]; A.K1[1] = (double*)c->K1[1];
  A.K2 = (double*)c->K2; A.K3 = (double*)c->K3;
  A.ctrl = c->dctrl;
  A.partials = c->partials;
  A.in = L.in;
  A.kin_k2 = L.stage == 3;
  A.coef = L.stage == 3 ? 0.75 : 0.5;
  A.out = L.mode == 0 ? L.out : (L.stage == 3 ? A.K3 : A.K2);
  // tile copies by the tensor-memory accelerator: A names the context's buffers; the
  // right-hand side's input gets its own map, encoded for this launch
  const TileMaps* M = nullptr;
  TileMaps Mr;
  if (c->maps.ok) {
    if (L.mode != 0) {
      M = &c->maps;
    } else if (L.in != nullptr) {
      Mr = c->maps;
      if (encode_state_map(c, &Mr.In, L.in, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, 5)) {
        Mr.inOk = 1;
        M = &Mr;
      }
    }
  }
  return c->precision == SGNB_FP64_FAST ? dev::launch_fused_fast(L.mode, c->C, A, s, M)
                                        : dev::launch_fused_exact(L.mode, c->C, A, s, M);
}

Launch rhs_launch(const double* in, double* out) {
  Launch L;
  L.mode = 0; L.in = in; L.out = out;
  return L;
}
Launch stage_launch(int stage) {
  Launch L;
  if (stage == 4) { L.mode = 2; } else { L.mode = 1; L.stage = stage; }
  return L;
}

int set_device(sgnb_ctx* c) {
  SGNB_CU(c, cudaSetDevice(c->device));
  return SGNB_OK;
}

int check_desc(const sgnb_desc* d) {
  if (!d) return fail(nullptr, SGNB_ERR_INVALID, "desc is NULL");
  if (d->Nx < 2 || d->Ny < 2) return fail(nullptr, SGNB_ERR_INVALID, "SGN2D: Nx,Ny >= 2");
  if (d->P != 4) return fail(nullptr, SGNB_ERR_UNSUPPORTED, "only P = 4 is built");
  if (!(d->Lx > 0) || !(d->Ly > 0)) return fail(nullptr, SGNB_ERR_INVALID, "Lx, Ly must be > 0");
  if (!(d->nManning >= 0.0)) return fail(nullptr, SGNB_ERR_INVALID, "nManning must be >= 0");
  if (d->bc_x < 0 || d->bc_x > 1 || d->bc_y < 0 || d->bc_y > 1)
    return fail(nullptr, SGNB_ERR_INVALID, "bc must be SGNB_BC_PERIODIC or SGNB_BC_WALL");
  if (d->precision != SGNB_FP64_EXACT && d->precision != SGNB_FP64_FAST &&
      d->precision != SGNB_MIXED)
    return fail(nullptr, SGNB_ERR_UNSUPPORTED, "unknown precision mode");
  if (d->Nx_global < 0 || (d->Nx_global > 0 && (d->ex_offset < 0 || d->ex_offset + d->Nx > d->Nx_global)))
    return fail(nullptr, SGNB_ERR_INVALID, "slab: 0 <= ex_offset, ex_offset + Nx <= Nx_global");
  if ((long long)d->Nx * d->Ny > (1ll << 31) / 25)
    return fail(nullptr, SGNB_ERR_INVALID, "mesh too large");
  if (d->point_set != SGNB_POINTS_GLL && d->point_set != SGNB_POINTS_GAUSS)
    return fail(nullptr, SGNB_ERR_INVALID, "point_set must be SGNB_POINTS_GLL or SGNB_POINTS_GAUSS");
  if (d->bathy_kind == SGNB_BATHY_ARRAYS) {
    if (!d->Hnod || !d->Hx || !d->Hy || !d->HfaceX || !d->HfaceY)
      return fail(nullptr, SGNB_ERR_INVALID, "SGNB_BATHY_ARRAYS needs Hnod, Hx, Hy, HfaceX, HfaceY");
    if ((d->bc_x == SGNB_BC_WALL && !d->HfaceXEnd) || (d->bc_y == SGNB_BC_WALL && !d->HfaceYEnd))
      return fail(nullptr, SGNB_ERR_INVALID, "walls need HfaceXEnd / HfaceYEnd");
  } else {
    const int need = bathy_param_count(d->bathy_kind, d->bathy_par, d->n_bathy_par);
    if (need < 0) return fail(nullptr, SGNB_ERR_INVALID, "unknown bathy_kind");
    if (need > 0 && (!d->bathy_par || d->n_bathy_par < need))
      return fail(nullptr, SGNB_ERR_INVALID, "bathy_par too short for bathy_kind");
  }
  return SGNB_OK;
}

// FR tables: the caller's (copied from a reference FROperators1D) or built here.
int tables_for(const sgnb_desc* d, FrTables& t) {
  fr_tables(d->P, t, d->point_set == SGNB_POINTS_GAUSS);
  const int n = d->P + 1;
  if (d->nodes) std::memcpy(t.nodes, d->nodes, n * sizeof(double));
  if (d->D) std::memcpy(t.D, d->D, n * n * sizeof(double));
  if (d->lL) std::memcpy(t.lL, d->lL, n * sizeof(double));
  if (d->lR) std::memcpy(t.lR, d->lR, n * sizeof(double));
  if (d->gLp) std::memcpy(t.gLp, d->gLp, n * sizeof(double));
  if (d->gRp) std::memcpy(t.gRp, d->gRp, n * sizeof(double));
  if (d->qw) std::memcpy(t.qw, d->qw, n * sizeof(double));
  // unit face rows: the traces are the edge nodes (GLL); otherwise the Gauss-point kernels
  // interpolate them
  bool unit = true;
  for (int j = 0; j < n; ++j)
    unit = unit && t.lL[j] == (j == 0 ? 1.0 : 0.0) && t.lR[j] == (j == n - 1 ? 1.0 : 0.0);
  t.gauss = !unit;
  if (t.gauss) {
    // a flat bottom H = 0 (sgn2d.cpp:46-47): no profile, or arrays that are all zero (the
    // accessors of a reference SGN2D built with Gauss points)
    bool flat = d->bathy_kind == SGNB_BATHY_NONE;
    if (d->bathy_kind == SGNB_BATHY_ARRAYS) {
      const long long ne = (long long)d->Nx * d->Ny, Nd = 25 * ne;
      auto zero = [](const double* a, long long m) {
        for (long long i = 0; a && i < m; ++i)
          if (a[i] != 0.0) return false;
        return true;
      };
      flat = zero(d->Hnod, Nd) && zero(d->Hx, Nd) && zero(d->Hy, Nd) && zero(d->HfaceX, 5 * ne) &&
             zero(d->HfaceY, 5 * ne) && zero(d->HfaceXEnd, 5 * d->Ny) && zero(d->HfaceYEnd, 5 * d->Nx);
    }
    if (!flat) return fail(nullptr, SGNB_ERR_INVALID, "SGN2D: bathymetry requires GLL points");
    if (d->precision == SGNB_MIXED)
      return fail(nullptr, SGNB_ERR_UNSUPPORTED, "Gauss points run in the FP64 modes");
    if (d->Nx_global > 0)
      return fail(nullptr, SGNB_ERR_UNSUPPORTED, "Gauss points run on whole meshes");
  }
  return SGNB_OK;
}

Mesh mesh_for(const sgnb_desc* d) {
  Mesh m;
  m.Nx = d->Nx; m.Ny = d->Ny; m.Lx = d->Lx; m.Ly = d->Ly;
  m.hx = d->Lx / (d->Nx_global > 0 ? d->Nx_global : d->Nx); m.hy = d->Ly / d->Ny;  // mesh2d.h:27-28
  m.ex0 = d->Nx_global > 0 ? d->ex_offset : 0;
  m.wrapx = d->Nx_global > 0 && d->bc_x == SGNB_BC_PERIODIC && d->ex_offset + d->Nx == d->Nx_global;
  return m;
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// A map of one state-sized buffer as [field][element row][Nx * 25] elements of `type` with
// a [nz][4][200] box (nz = 5: one tile of every field; 1: one field).
static bool encode_state_map(const sgnb_ctx* c, CUtensorMap* m, const void* p,
                             CUtensorMapDataType type, size_t elem, cuuint32_t nz) {
  const EncodeTiled enc = reinterpret_cast<EncodeTiled>(c->encode_tiled);
  if (enc == nullptr || ((uintptr_t)p & 15) != 0) return false;
  const cuuint64_t W = (cuuint64_t)c->desc.Nx * 25;
  const cuuint64_t dim[3] = {W, (cuuint64_t)c->desc.Ny, 5};
  const cuuint64_t stride[2] = {W * elem, (cuuint64_t)c->Nd * elem};
  const cuuint32_t box[3] = {200, 4, nz};
  const cuuint32_t one[3] = {1, 1, 1};
  return enc(m, type, 3, const_cast<void*>(p), dim, stride, box, one,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor maps of the context's buffers for the fused kernels' tile loads (meshes that are
// a whole number of 8x4 tiles). The encoder comes from the driver through the runtime, so
// the library links no driver library; without it (or on any encoding error), or with
// SGNB_TMA=0 in the environment at creation, the kernels keep their per-thread
// asynchronous copies. Only the data movement differs: the exact mode gives the same bits;
// in the fast mode the TMA kernels are separate instantiations whose FMA contractions the
// compiler chooses on its own, so they agree to round-off (tests/test_tma_gpu.py finds
// the same bits for the whole-mesh kernels).
static void build_tile_maps(sgnb_ctx* c) {
  c->maps.ok = 0;
  c->maps.inOk = 0;
  c->mapsM.ok = 0;
  c->encode_tiled = nullptr;
  if (c->desc.Nx % 8 != 0 || c->desc.Ny % 4 != 0) return;
  const char* sw = std::getenv("SGNB_TMA");
  if (sw && sw[0] == '0') return;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
  if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault,
                                       &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || fn == nullptr) {
    cudaGetLastError();
    return;
  }
  c->encode_tiled = fn;
  const EncodeTiled enc = reinterpret_cast<EncodeTiled>(fn);
  // the nodal depth: [element row][Nx * 25] doubles, box [4][200]
  const cuuint64_t dim2[2] = {(cuuint64_t)c->desc.Nx * 25, (cuuint64_t)c->desc.Ny};
  const cuuint64_t stride2[1] = {dim2[0] * sizeof(double)};
  const cuuint32_t box2[2] = {200, 4};
  const cuuint32_t one[2] = {1, 1};
  auto mapH = [&](CUtensorMap* m) {
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(c->C.Hnod), dim2,
               stride2, box2, one, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
  };
  const auto F64 = CU_TENSOR_MAP_DATA_TYPE_FLOAT64, F32 = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  if (c->mixed) {
    const bool okm = encode_state_map(c, &c->mapsM.K1[0], c->K1[0], F32, 4, 1) &&
                     encode_state_map(c, &c->mapsM.K1[1], c->K1[1], F32, 4, 1) &&
                     encode_state_map(c, &c->mapsM.K2, c->K2, F32, 4, 1) &&
                     encode_state_map(c, &c->mapsM.K3, c->K3, F32, 4, 1) && mapH(&c->mapsM.H);
    c->mapsM.ok = okm ? 1 : 0;
    return;
  }
  const bool ok = encode_state_map(c, &c->maps.U[0], c->U[0], F64, 8, 5) &&
                  encode_state_map(c, &c->maps.U[1], c->U[1], F64, 8, 5) &&
                  encode_state_map(c, &c->maps.K1[0], c->K1[0], F64, 8, 5) &&
                  encode_state_map(c, &c->maps.K1[1], c->K1[1], F64, 8, 5) &&
                  encode_state_map(c, &c->maps.K2, c->K2, F64, 8, 5) &&
                  encode_state_map(c, &c->maps.K3, c->K3, F64, 8, 5) && mapH(&c->maps.H);
  c->maps.ok = ok ? 1 : 0;
}

void fill_consts(sgnb_ctx* c) {
  RhsConsts& C = c->C;
  const sgnb_desc& d = c->desc;
  C.Nx = d.Nx; C.Ny = d.Ny;
  C.bcx = d.bc_x; C.bcy = d.bc_y;
  C.Nd = c->Nd;
  C.g = d.g;
  C.halfg = 0.5 * d.g;
  C.gamma = d.gamma;
  C.c2 = d.c * d.c;
  C.mc2 = -d.c * d.c;
  C.m2c2 = -2.0 * C.c2;
  C.n2g = (d.nManning * d.nManning) * d.g;  // n2 * g as sgn_flux2d.h:137-139 multiplies
  C.manning = d.nManning != 0.0;
  C.Jx = 0.5 * c->mesh.hx;  // mesh2d.h:49-50
  C.Jy = 0.5 * c->mesh.hy;
  C.iJx = 1.0 / C.Jx;
  C.iJy = 1.0 / C.Jy;
  for (int k = 0; k < 25; ++k) {
    C.D[k] = c->tab.D[k];
    C.Df[k] = (float)c->tab.D[k];
  }
  for (int k = 0; k < 5; ++k) {
    C.gLp[k] = c->tab.gLp[k];
    C.gRp[k] = c->tab.gRp[k];
    C.gLpf[k] = (float)c->tab.gLp[k];
    C.gRpf[k] = (float)c->tab.gRp[k];
    C.lL[k] = c->tab.lL[k];
    C.lR[k] = c->tab.lR[k];
  }
  C.gauss = c->tab.gauss;
  C.tr = c->trbuf;
}

// The device-side loop: a CUDA graph whose one node is a WHILE conditional node; its body
// is one attempt (stages 2, 3, the end-point stage, the controller), and the controller
// sets the condition. One graph launch runs attempts until the run is done or attemptCap
// is reached, with no host round trip and no attempt launched after the end.
int build_loop_graph(sgnb_ctx* c) {
  if (c->chunk) return SGNB_OK;
  cudaGraph_t g = nullptr;
  SGNB_CU(c, cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle loop;
  cudaError_t e = cudaGraphConditionalHandleCreate(&loop, g, 1, cudaGraphCondAssignDefault);
  cudaGraphNodeParams p = {};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = loop;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, nullptr, 0, &p);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return cuda_fail(c, e, "conditional node of the device-side loop");
  }
  cudaGraph_t body = p.conditional.phGraph_out[0];
  e = cudaStreamBeginCaptureToGraph(c->stream, body, nullptr, nullptr, 0,
                                    cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    e = launch(c, stage_launch(2), c->stream);                 // k2 = R(u + dt/2 k1)
    if (e == cudaSuccess) e = launch(c, stage_launch(3), c->stream);  // k3 = R(u + 3dt/4 k2)
    if (e == cudaSuccess) e = launch(c, stage_launch(4), c->stream);  // uNew, k4, partials
    if (e == cudaSuccess)
      e = dev::launch_controller_loop(c->dctrl, c->partials, c->nblk, c->ntot, loop, c->stream);
    cudaError_t e2 = cudaStreamEndCapture(c->stream, &body);
    if (e == cudaSuccess) e = e2;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&c->chunk, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    c->chunk = nullptr;
    return cuda_fail(c, e, "device-side loop graph");
  }
  c->chunkLen = 1;
  return SGNB_OK;
}

// Drive the device-side loop until the controller reports done: each graph launch runs up
// to kAttemptsPerLaunch attempts (a bound on one launch's duration); the host reads the
// controller state between launches.
int run_loop(sgnb_ctx* c) {
  constexpr long long kAttemptsPerLaunch = 4096;
  // SGNB_HOST_LOOP=1: the same kernels launched from the host, 16 attempts between reads of
  // the controller (kernel-replay profilers do not see kernels inside conditional nodes)
  const char* hl = std::getenv("SGNB_HOST_LOOP");
  const bool host_loop = hl && hl[0] == '1';
  if (!host_loop) {
    int rc = build_loop_graph(c);
    if (rc) return rc;
  }
  CtrlState& h = *c->hctrl;
  h.attemptCap = h.attempts + kAttemptsPerLaunch;
  SGNB_CU(c, cudaMemcpyAsync(c->dctrl, c->hctrl, sizeof(CtrlState), cudaMemcpyHostToDevice, c->stream));
  // kernels per right-hand side: the fused kernel, after the trace pre-pass for Gauss points
  const long long per_rhs = c->tab.gauss ? 2 : 1, per_attempt = 3 * per_rhs + 1;
  const long long attempts0 = h.attempts;
  // FSAL head: k1 = R(u) into K1[cur] (FP32 in the mixed mode)
  SGNB_CU(c, launch(c, rhs_launch(c->U[c->cur], c->mixed ? nullptr : (double*)c->K1[c->cur]),
                    c->stream));
  long long host_attempts = 0;  // attempts launched by the host loop (finished runs' exit at entry)
  for (;;) {
    if (host_loop) {
      host_attempts += 16;
      for (int k = 0; k < 16; ++k) {
        SGNB_CU(c, launch(c, stage_launch(2), c->stream));
        SGNB_CU(c, launch(c, stage_launch(3), c->stream));
        SGNB_CU(c, launch(c, stage_launch(4), c->stream));
        SGNB_CU(c, dev::launch_controller(c->dctrl, c->partials, c->nblk, c->ntot, c->stream));
      }
    } else {
      SGNB_CU(c, cudaGraphLaunch(c->chunk, c->stream));
    }
    SGNB_CU(c, cudaMemcpyAsync(c->hctrl, c->dctrl, sizeof(CtrlState), cudaMemcpyDeviceToHost, c->stream));
    SGNB_CU(c, cudaStreamSynchronize(c->stream));
    if (h.done) break;
    h.attemptCap = h.attempts + kAttemptsPerLaunch;  // more attempts than one launch allows
    SGNB_CU(c, cudaMemcpyAsync(c->dctrl, c->hctrl, sizeof(CtrlState), cudaMemcpyHostToDevice, c->stream));
  }
  c->launches = per_rhs + per_attempt * (host_loop ? host_attempts : h.attempts - attempts0);
  c->cur = h.cur;
  return SGNB_OK;
}

void init_ctrl(sgnb_ctx* c, CtrlState& s, const sgnb_rk_opts& o) {
  std::memset(&s, 0, sizeof(s));
  s.log = c->alog;
  s.logCap = sgnb_ctx::kLogCap;
  s.atol = o.atol; s.rtol = o.rtol; s.dtMin = o.dtMin; s.dtMax = o.dtMax;
  s.safety = o.safety; s.facMin = o.facMin; s.facMax = o.facMax;
  const int orderLow = 2;                          // rk.cpp:71-76
  const double expo = 1.0 / (orderLow + 1.0);
  s.alpha = 0.7 * expo;
  s.beta = 0.4 * expo;
}

}  // namespace

extern "C" {

void sgnb_desc_init(sgnb_desc* d) {
  if (!d) return;
  std::memset(d, 0, sizeof(*d));
  d->P = 4; d->Nx = 2; d->Ny = 2; d->Lx = 1.0; d->Ly = 1.0;
  d->g = 9.81; d->c = 0.0; d->gamma = 1.5; d->nManning = 0.0;
  d->bc_x = SGNB_BC_PERIODIC; d->bc_y = SGNB_BC_PERIODIC;
  d->precision = SGNB_FP64_EXACT;
  d->bathy_kind = SGNB_BATHY_NONE;
}

void sgnb_rk_opts_init(sgnb_rk_opts* o) {
  if (!o) return;
  o->atol = 1e-8; o->rtol = 1e-6; o->dtMin = 1e-13; o->dtMax = 1e30;
  o->safety = 0.9; o->facMin = 0.2; o->facMax = 5.0;
}

int sgnb_fr_tables(int P, double* nodes, double* D, double* lL, double* lR, double* gLp,
                   double* gRp, double* qw) {
  FrTables t;
  if (!fr_tables(P, t)) return fail(nullptr, SGNB_ERR_UNSUPPORTED, "P out of range");
  const int n = P + 1;
  if (nodes) std::memcpy(nodes, t.nodes, n * sizeof(double));
  if (D) std::memcpy(D, t.D, n * n * sizeof(double));
  if (lL) std::memcpy(lL, t.lL, n * sizeof(double));
  if (lR) std::memcpy(lR, t.lR, n * sizeof(double));
  if (gLp) std::memcpy(gLp, t.gLp, n * sizeof(double));
  if (gRp) std::memcpy(gRp, t.gRp, n * sizeof(double));
  if (qw) std::memcpy(qw, t.qw, n * sizeof(double));
  return SGNB_OK;
}

int sgnb_fr_tables_points(int P, int point_set, double* nodes, double* D, double* lL,
                          double* lR, double* gLp, double* gRp, double* qw) {
  if (point_set != SGNB_POINTS_GLL && point_set != SGNB_POINTS_GAUSS)
    return fail(nullptr, SGNB_ERR_INVALID, "point_set must be SGNB_POINTS_GLL or SGNB_POINTS_GAUSS");
  FrTables t;
  if (!fr_tables(P, t, point_set == SGNB_POINTS_GAUSS))
    return fail(nullptr, SGNB_ERR_UNSUPPORTED, "P out of range");
  const int n = P + 1;
  if (nodes) std::memcpy(nodes, t.nodes, n * sizeof(double));
  if (D) std::memcpy(D, t.D, n * n * sizeof(double));
  if (lL) std::memcpy(lL, t.lL, n * sizeof(double));
  if (lR) std::memcpy(lR, t.lR, n * sizeof(double));
  if (gLp) std::memcpy(gLp, t.gLp, n * sizeof(double));
  if (gRp) std::memcpy(gRp, t.gRp, n * sizeof(double));
  if (qw) std::memcpy(qw, t.qw, n * sizeof(double));
  return SGNB_OK;
}

int sgnb_setup_bathymetry(const sgnb_desc* d, double* Hnod, double* Hx, double* Hy,
                          double* HfaceX, double* HfaceY, double* HfaceXEnd,
                          double* HfaceYEnd) {
  int rc = check_desc(d);
  if (rc) return rc;
  if (d->bathy_kind == SGNB_BATHY_ARRAYS) return fail(nullptr, SGNB_ERR_INVALID, "arrays given");
  FrTables t;
  if ((rc = tables_for(d, t))) return rc;
  const Mesh m = mesh_for(d);
  Bathymetry b;
  bathymetry(m, t, d->bathy_kind, d->bathy_par, b);
  auto cp = [](const std::vector<double>& v, double* o) {
    if (o) std::memcpy(o, v.data(), v.size() * sizeof(double));
  };
  cp(b.Hnod, Hnod); cp(b.Hx, Hx); cp(b.Hy, Hy); cp(b.HfX, HfaceX); cp(b.HfY, HfaceY);
  cp(b.HfXEnd, HfaceXEnd); cp(b.HfYEnd, HfaceYEnd);
  return SGNB_OK;
}

int sgnb_create(const sgnb_desc* d, sgnb_ctx** out) {
  if (!out) return fail(nullptr, SGNB_ERR_INVALID, "out is NULL");
  *out = nullptr;
  int rc = check_desc(d);
  if (rc) return rc;
  {  // argument errors (tables, point set against bathymetry) before device errors
    FrTables t;
    if ((rc = tables_for(d, t))) return rc;
  }
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return fail(nullptr, SGNB_ERR_NO_DEVICE, "no CUDA device visible");
  if (d->device < 0 || d->device >= ndev) return fail(nullptr, SGNB_ERR_INVALID, "bad device ordinal");

  sgnb_ctx* c = new sgnb_ctx();
  c->desc = *d;
  c->desc.nodes = c->desc.D = c->desc.lL = c->desc.lR = nullptr;
  c->desc.gLp = c->desc.gRp = c->desc.qw = nullptr;
  c->desc.bathy_par = nullptr;
  c->desc.Hnod = c->desc.Hx = c->desc.Hy = c->desc.HfaceX = c->desc.HfaceY = nullptr;
  c->desc.HfaceXEnd = c->desc.HfaceYEnd = nullptr;
  c->device = d->device;
  c->precision = d->precision;
  c->mixed = d->precision == SGNB_MIXED;
  if ((rc = tables_for(d, c->tab))) { delete c; return rc; }
  c->mesh = mesh_for(d);
  const long long ne = (long long)d->Nx * d->Ny;
  c->Nd = ne * 25;
  c->ntot = 5 * c->Nd;
  auto bail = [&](int code) { sgnb_destroy(c); return code; };
  if ((rc = set_device(c))) { g_create_error = c->err; delete c; return rc; }
  e = dev::prepare_fused_exact();
  if (e == cudaSuccess) e = dev::prepare_fused_fast();
  if (e == cudaSuccess) e = dev::prepare_fused_mixed();
  if (e == cudaSuccess) e = dev::prepare_fused_batch();
  if (e == cudaSuccess) e = dev::prepare_mixed_batch();
  if (e != cudaSuccess) { cuda_fail(c, e, "kernel attributes"); g_create_error = c->err; return bail(SGNB_ERR_CUDA); }

  // statics: Hnod, Hx, Hy (Nd each), HfX, HfY (5 ne each), HfXEnd (5 Ny), HfYEnd (5 Nx)
  Bathymetry b;
  if (d->bathy_kind == SGNB_BATHY_ARRAYS) {
    b.Hnod.assign(d->Hnod, d->Hnod + c->Nd);
    b.Hx.assign(d->Hx, d->Hx + c->Nd);
    b.Hy.assign(d->Hy, d->Hy + c->Nd);
    b.HfX.assign(d->HfaceX, d->HfaceX + 5 * ne);
    b.HfY.assign(d->HfaceY, d->HfaceY + 5 * ne);
    b.HfXEnd.assign(5 * (size_t)d->Ny, 0.0);
    b.HfYEnd.assign(5 * (size_t)d->Nx, 0.0);
    if (d->HfaceXEnd) b.HfXEnd.assign(d->HfaceXEnd, d->HfaceXEnd + 5 * d->Ny);
    if (d->HfaceYEnd) b.HfYEnd.assign(d->HfaceYEnd, d->HfaceYEnd + 5 * d->Nx);
    // the kernels form dH/dx, dH/dy from Hnod as SGN2D does; given arrays must agree
    std::vector<double> gx(c->Nd), gy(c->Nd);
    depth_gradients(c->mesh, c->tab, b.Hnod.data(), gx.data(), gy.data());
    if (std::memcmp(gx.data(), b.Hx.data(), c->Nd * sizeof(double)) != 0 ||
        std::memcmp(gy.data(), b.Hy.data(), c->Nd * sizeof(double)) != 0) {
      c->err = "SGNB_BATHY_ARRAYS: Hx, Hy must be the element-local GLL derivative of Hnod "
               "over the Jacobian, as SGN2D computes them (src/solver/sgn2d.cpp:54-71)";
      g_create_error = c->err;
      return bail(SGNB_ERR_UNSUPPORTED);
    }
  } else {
    bathymetry(c->mesh, c->tab, d->bathy_kind, d->bathy_par, b);
  }
  const size_t nstat = 3 * (size_t)c->Nd + 10 * (size_t)ne + 5 * (size_t)(d->Nx + d->Ny);
  e = cudaMalloc(&c->Hbuf, nstat * sizeof(double));
  if (e != cudaSuccess) { cuda_fail(c, e, "cudaMalloc(statics)"); g_create_error = c->err; return bail(SGNB_ERR_NOMEM); }
  double* p = c->Hbuf;
  auto put = [&](const std::vector<double>& v, const double*& dst) {
    dst = p;
    cudaError_t e2 = cudaMemcpy(p, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice);
    p += v.size();
    return e2;
  };
  e = put(b.Hnod, c->C.Hnod);
  if (e == cudaSuccess) e = put(b.Hx, c->C.Hx);
  if (e == cudaSuccess) e = put(b.Hy, c->C.Hy);
  if (e == cudaSuccess) e = put(b.HfX, c->C.HfX);
  if (e == cudaSuccess) e = put(b.HfY, c->C.HfY);
  if (e == cudaSuccess) e = put(b.HfXEnd, c->C.HfXEnd);
  if (e == cudaSuccess) e = put(b.HfYEnd, c->C.HfYEnd);
  if (e != cudaSuccess) { cuda_fail(c, e, "upload of statics"); g_create_error = c->err; return bail(SGNB_ERR_CUDA); }
  if (c->tab.gauss) {
    e = cudaMalloc(&c->trbuf, 100 * (size_t)ne * sizeof(double));
    if (e != cudaSuccess) { cuda_fail(c, e, "cudaMalloc(traces)"); g_create_error = c->err; return bail(SGNB_ERR_NOMEM); }
  }
  fill_consts(c);

  const size_t sbytes = (size_t)c->ntot * sizeof(double);
  // stage derivatives are FP32 in the mixed mode; K2 and K3 are allocated as one block so
  // that together they always hold an FP64 state (scratch for sgnb_rhs_host)
  const size_t kbytes = (size_t)c->ntot * (c->mixed ? sizeof(float) : sizeof(double));
  for (double** bp : {&c->U[0], &c->U[1]}) {
    e = cudaMalloc(bp, sbytes);
    if (e != cudaSuccess) { cuda_fail(c, e, "cudaMalloc(state)"); g_create_error = c->err; return bail(SGNB_ERR_NOMEM); }
  }
  for (void** bp : {&c->K1[0], &c->K1[1]}) {
    e = cudaMalloc(bp, kbytes);
    if (e != cudaSuccess) { cuda_fail(c, e, "cudaMalloc(stage)"); g_create_error = c->err; return bail(SGNB_ERR_NOMEM); }
  }
  e = cudaMalloc(&c->K2, 2 * kbytes);
  if (e != cudaSuccess) { cuda_fail(c, e, "cudaMalloc(stage)"); g_create_error = c->err; return bail(SGNB_ERR_NOMEM); }
  c->K3 = (char*)c->K2 + kbytes;
  build_tile_maps(c);
  e = cudaMemset(c->U[0], 0, sbytes);
  c->nblk = dev::fused_grid_blocks(d->Nx, d->Ny);
  c->ndiag = 592;
  if (e == cudaSuccess) e = cudaMalloc(&c->partials, 3 * (size_t)c->nblk * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&c->diag, (size_t)c->ndiag * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&c->dctrl, sizeof(CtrlState));
  if (e == cudaSuccess) e = cudaMalloc(&c->alog, 4 * sgnb_ctx::kLogCap * sizeof(double));
  if (e == cudaSuccess) e = cudaMallocHost(&c->hctrl, sizeof(CtrlState));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->evRead, cudaEventDisableTiming);
  if (e != cudaSuccess) { cuda_fail(c, e, "context buffers"); g_create_error = c->err; return bail(SGNB_ERR_CUDA); }
  sgnb_rk_opts o;
  sgnb_rk_opts_init(&o);
  init_ctrl(c, *c->hctrl, o);
  *out = c;
  return SGNB_OK;
}

int sgnb_destroy(sgnb_ctx* c) {
  if (!c) return SGNB_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->chunk) cudaGraphExecDestroy(c->chunk);
  if (c->evRead) cudaEventDestroy(c->evRead);
  cudaFree(c->Hbuf);
  cudaFree(c->trbuf);
  for (int k = 0; k < 2; ++k) { cudaFree(c->U[k]); cudaFree(c->K1[k]); }
  cudaFree(c->K2);  // K3 lives in the same block
  cudaFree(c->partials); cudaFree(c->diag); cudaFree(c->dctrl); cudaFree(c->dtList);
  cudaFree(c->alog);
  cudaFree(c->gauge);
  if (c->hctrl) cudaFreeHost(c->hctrl);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return SGNB_OK;
}

long long sgnb_ndof(const sgnb_ctx* c) { return c ? c->Nd : 0; }

int sgnb_upload(sgnb_ctx* c, const double* U) {
  if (!c || !U) return fail(c, SGNB_ERR_INVALID, "NULL argument");
  if (int rc = set_device(c)) return rc;
  SGNB_CU(c, cudaMemcpyAsync(c->U[c->cur], U, c->ntot * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  SGNB_CU(c, cudaStreamSynchronize(c->stream));
  return SGNB_OK;
}

int sgnb_download(sgnb_ctx* c, double* U) {
  if (!c || !U) return fail(c, SGNB_ERR_INVALID, "NULL argument");
  if (int rc = set_device(c)) return rc;
  SGNB_CU(c, cudaMemcpyAsync(U, c->U[c->cur], c->ntot * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  SGNB_CU(c, cudaStreamSynchronize(c->stream));
  return SGNB_OK;
}

int sgnb_rhs_device(sgnb_ctx* c, const double* Ud, double* dUd, void* stream) {
  if (!c || !Ud || !dUd) return fail(c, SGNB_ERR_INVALID, "NULL argument");
  if (Ud == dUd) return fail(c, SGNB_ERR_INVALID, "input and output must not alias");
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  SGNB_CU(c, launch(c, rhs_launch(Ud, dUd), s));
  return SGNB_OK;
}

int sgnb_rhs_once(sgnb_ctx* c, double* dU) {
  if (!c || !dU) return fail(c, SGNB_ERR_INVALID, "NULL argument");
  if (int rc = set_device(c)) return rc;
  if (int rc = sgnb_rhs_device(c, c->U[c->cur], c->U[c->cur ^ 1], c->stream)) return rc;
  SGNB_CU(c, cudaMemcpyAsync(dU, c->U[c->cur ^ 1], c->ntot * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  SGNB_CU(c, cudaStreamSynchronize(c->stream));
  return SGNB_OK;
}

int sgnb_rhs_host(sgnb_ctx* c, const double* U, double* dU) {
  if (!c || !U || !dU) return fail(c, SGNB_ERR_INVALID, "NULL argument");
  if (int rc = set_device(c)) return rc;
  // scratch: the spare state buffer holds the input; the output goes over it in place
  // is not allowed, so the input goes to U[cur ^ 1] and the output to the FP64 view of the
  // stage buffers (K2, K3 together hold one FP64 state in every precision mode)
  double* in = c->U[c->cur ^ 1];
  double* out = c->mixed ? (double*)c->K2 : (double*)c->K3;
  SGNB_CU(c, cudaMemcpyAsync(in, U, c->ntot * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (int rc = sgnb_rhs_device(c, in, out, c->stream)) return rc;
  SGNB_CU(c, cudaMemcpyAsync(dU, out, c->ntot * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  SGNB_CU(c, cudaStreamSynchronize(c->stream));
  return SGNB_OK;
}

int sgnb_integrate_adaptive(sgnb_ctx* c, double t0, double tEnd, double dt0,
                            const sgnb_rk_opts* opts, sgnb_rk_stats* st) {
  if (!c) return fail(c, SGNB_ERR_INVALID, "NULL context");
  if (c->C.ghostL || c->C.ghostR)
    return fail(c, SGNB_ERR_INVALID, "a slab integrates through the slab entries (sgnb_slab_*)");
  if (int rc = set_device(c)) return rc;
  sgnb_rk_opts o;
  if (opts) o = *opts; else sgnb_rk_opts_init(&o);
  CtrlState& h = *c->hctrl;
  init_ctrl(c, h, o);
  h.t = t0;
  h.tEnd = tEnd;
  h.dt = (o.dtMax < dt0) ? o.dtMax : dt0;  // std::min(dt0, dtMax), rk.cpp:87
  h.errPrev = 1.0;
  h.tReached = t0;
  h.cur = c->cur;
  h.rhsEvals = 1;  // FSAL head
  h.maxAccepted = c->pendingMaxAccepted;
  // loop test and end-time clip of the first attempt (rk.cpp:95-97)
  if (!(h.t < tEnd - 1e-15 * ((1.0 < std::fabs(tEnd)) ? std::fabs(tEnd) : 1.0))) h.done = 1;
  else if (h.t + h.dt > tEnd) h.dt = tEnd - h.t;
  if (c->ntot == 0) h.done = 1;
  if (int rc = run_loop(c)) return rc;
  if (st) {
    st->accepted = h.accepted; st->rejected = h.rejected; st->rhsEvals = h.rhsEvals;
    st->attempts = h.attempts; st->tReached = h.tReached; st->dtLast = h.dtLast;
    st->maxNormLast = h.maxNormLast;
    st->aborted = h.done == 2 ? 1 : (h.done == 3 ? 2 : 0);
    st->status = h.done == 3 ? SGNB_ERR_NAN : SGNB_OK;
    st->kernel_launches = c->launches;
  }
  if (h.done == 3) return fail(c, SGNB_ERR_NAN, "non-finite embedded error estimate");
  return SGNB_OK;
}

int sgnb_integrate_steps(sgnb_ctx* c, double t0, double dt0, long long nsteps,
                         const sgnb_rk_opts* opts, sgnb_rk_stats* st) {
  if (!c || nsteps < 1) return fail(c, SGNB_ERR_INVALID, "nsteps must be >= 1");
  c->hctrl->maxAccepted = 0;
  c->pendingMaxAccepted = nsteps;
  const int rc = sgnb_integrate_adaptive(c, t0, 1e300, dt0, opts, st);
  c->pendingMaxAccepted = 0;
  return rc;
}

int sgnb_launch_stage(sgnb_ctx* c, int stage, double dt, int count, void* stream) {
  if (!c || stage < 2 || stage > 4 || count < 1 || !(dt > 0))
    return fail(c, SGNB_ERR_INVALID, "stage in 2..4, count >= 1, dt > 0");
  if (int rc = set_device(c)) return rc;
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  CtrlState& h = *c->hctrl;
  sgnb_rk_opts o;
  sgnb_rk_opts_init(&o);
  init_ctrl(c, h, o);
  h.t = 0.0;
  h.tEnd = 1e300;
  h.dt = dt;
  h.cur = c->cur;
  h.log = nullptr;
  SGNB_CU(c, cudaMemcpyAsync(c->dctrl, c->hctrl, sizeof(CtrlState), cudaMemcpyHostToDevice, s));
  for (int k = 0; k < count; ++k) SGNB_CU(c, launch(c, stage_launch(stage), s));
  return SGNB_OK;
}

int sgnb_bs3_steps(sgnb_ctx* c, double t0, const double* dts, long long n) {
  if (!c || (n > 0 && !dts) || n < 0) return fail(c, SGNB_ERR_INVALID, "bad arguments");
  if (c->C.ghostL || c->C.ghostR)
    return fail(c, SGNB_ERR_INVALID, "a slab integrates through the slab entries (sgnb_slab_*)");
  if (n == 0) return SGNB_OK;
  if (int rc = set_device(c)) return rc;
  if (n > c->dtCap) {
    cudaFree(c->dtList);
    c->dtList = nullptr;
    SGNB_CU(c, cudaMalloc(&c->dtList, n * sizeof(double)));
    c->dtCap = n;
  }
  SGNB_CU(c, cudaMemcpy(c->dtList, dts, n * sizeof(double), cudaMemcpyHostToDevice));
  CtrlState& h = *c->hctrl;
  sgnb_rk_opts o;
  sgnb_rk_opts_init(&o);
  init_ctrl(c, h, o);
  h.t = t0;
  h.tEnd = 1e300;
  h.dt = dts[0];
  h.cur = c->cur;
  h.frozen = 1;
  h.dtList = c->dtList;
  h.nList = n;
  h.rhsEvals = 1;
  if (int rc = run_loop(c)) return rc;
  if (h.done == 3) return fail(c, SGNB_ERR_NAN, "non-finite state");
  return SGNB_OK;
}

// rk4Step (src/solver/rk.cpp:23-38) per given step size: k1 = R(u) into K1[cur], then the
// fused stage kernel three times with the stage coefficient 1/2 (k1 -> K2), 1/2 (K2 -> K3)
// and 1 (K3 -> K1[cur ^ 1]): its u + (c dt) k rounds as u + 0.5 * dt * k and u + dt * k
// do on the CPU (c dt is exact for c = 1/2 and 1). The update writes the state in place.
int sgnb_rk4_steps(sgnb_ctx* c, double t0, const double* dts, long long n) {
  (void)t0;  // R does not depend on t
  if (!c || (n > 0 && !dts) || n < 0) return fail(c, SGNB_ERR_INVALID, "bad arguments");
  if (c->C.ghostL || c->C.ghostR)
    return fail(c, SGNB_ERR_INVALID, "a slab integrates through the slab entries (sgnb_slab_*)");
  if (c->mixed) return fail(c, SGNB_ERR_UNSUPPORTED, "rk4 steps run in the FP64 modes");
  if (n == 0) return SGNB_OK;
  if (int rc = set_device(c)) return rc;
  if (n > c->dtCap) {
    cudaFree(c->dtList);
    c->dtList = nullptr;
    SGNB_CU(c, cudaMalloc(&c->dtList, n * sizeof(double)));
    c->dtCap = n;
  }
  SGNB_CU(c, cudaMemcpy(c->dtList, dts, n * sizeof(double), cudaMemcpyHostToDevice));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
  CtrlState& h = *c->hctrl;
  sgnb_rk_opts o;
  sgnb_rk_opts_init(&o);
  init_ctrl(c, h, o);  // done = 0: the stage kernels run
  h.cur = c->cur;
  h.log = nullptr;
  cudaStream_t s = c->stream;
  SGNB_CU(c, cudaMemcpyAsync(c->dctrl, c->hctrl, sizeof(CtrlState), cudaMemcpyHostToDevice, s));
  const int cur = c->cur;
  double* u = c->U[cur];
  double* k1 = (double*)c->K1[cur];
  double* k2 = (double*)c->K2;
  double* k3 = (double*)c->K3;
  double* k4 = (double*)c->K1[cur ^ 1];
  auto stage = [&](const double* kin, double coef, double* out) {
    StageArgs A{};
    A.U[0] = c->U[0]; A.U[1] = c->U[1];
    A.K1[0] = (double*)c->K1[0]; A.K1[1] = (double*)c->K1[1];
    A.K2 = const_cast<double*>(kin);  // the stage kernel adds A.K2 when kin_k2 is set
    A.K3 = k3;
    A.kin_k2 = 1;
    A.coef = coef;
    A.out = out;
    A.ctrl = c->dctrl;
    A.partials = c->partials;
    return c->precision == SGNB_FP64_FAST ? dev::launch_fused_fast(1, c->C, A, s)
                                          : dev::launch_fused_exact(1, c->C, A, s);
  };
  for (long long i = 0; i < n; ++i) {
    SGNB_CU(c, dev::launch_rk4_set_dt(c->dctrl, c->dtList, i, s));
    SGNB_CU(c, launch(c, rhs_launch(u, k1), s));  // k1 = R(u)
    SGNB_CU(c, stage(k1, 0.5, k2));                // k2 = R(u + 0.5 dt k1)
    SGNB_CU(c, stage(k2, 0.5, k3));                // k3 = R(u + 0.5 dt k2)
    SGNB_CU(c, stage(k3, 1.0, k4));                // k4 = R(u + dt k3)
    SGNB_CU(c, dev::launch_rk4_update(u, k1, k2, k3, k4, c->dctrl, c->ntot, sms, s));
  }
  SGNB_CU(c, cudaStreamSynchronize(s));
  return SGNB_OK;
}

static int diag(sgnb_ctx* c, int what, double* out) {
  if (!c || !out) return fail(c, SGNB_ERR_INVALID, "NULL argument");
  if (int rc = set_device(c)) return rc;
  SGNB_CU(c, dev::launch_reduce_diag(what, c->C, c->U[c->cur], c->tab.qw, c->diag, c->ndiag, c->stream));
  std::vector<double> part(c->ndiag);
  SGNB_CU(c, cudaMemcpyAsync(part.data(), c->diag, c->ndiag * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  SGNB_CU(c, cudaStreamSynchronize(c->stream));
  double acc = 0.0;
  for (double v : part) acc = (what == 0) ? std::fmax(acc, v) : acc + v;
  *out = acc;
  return SGNB_OK;
}

int sgnb_max_wave_speed(sgnb_ctx* c, double* out) { return diag(c, 0, out); }

int sgnb_cfl_time_step(sgnb_ctx* c, double cfl, double* out) {
  double lam = 0.0;
  if (int rc = diag(c, 0, &lam)) return rc;
  // SGN2D::cflTimeStep (sgn2d.cpp:310-314)
  const double dxEff = std::fmin(c->mesh.hx, c->mesh.hy) / (2.0 * c->desc.P + 1.0);
  *out = cfl * dxEff / (lam > 0.0 ? lam : 1e-300);
  return SGNB_OK;
}

int sgnb_mass(sgnb_ctx* c, double* out) {
  double m = 0.0;
  if (int rc = diag(c, 1, &m)) return rc;
  *out = m * (c->C.Jx * c->C.Jy);
  return SGNB_OK;
}

int sgnb_energy(sgnb_ctx* c, double* out) {
  double E = 0.0;
  if (int rc = diag(c, 2, &E)) return rc;
  *out = E * (c->C.Jx * c->C.Jy);
  return SGNB_OK;
}

int sgnb_node_coords(const sgnb_ctx* c, double* x, double* y) {
  if (!c || !x || !y) return SGNB_ERR_INVALID;
  node_coords(c->mesh, c->tab, x, y);
  return SGNB_OK;
}

int sgnb_attempt_log(sgnb_ctx* c, double* out, long long cap, long long* n) {
  if (!c || (cap > 0 && !out)) return fail(c, SGNB_ERR_INVALID, "bad arguments");
  if (int rc = set_device(c)) return rc;
  const long long have = c->hctrl->attempts < sgnb_ctx::kLogCap ? c->hctrl->attempts : sgnb_ctx::kLogCap;
  const long long m = have < cap ? have : cap;
  if (m > 0)
    SGNB_CU(c, cudaMemcpy(out, c->alog, 4 * m * sizeof(double), cudaMemcpyDeviceToHost));
  if (n) *n = have;
  return SGNB_OK;
}

int sgnb_state_device_ptr(sgnb_ctx* c, double** U, void** stream) {
  if (!c) return SGNB_ERR_INVALID;
  if (U) *U = c->U[c->cur];
  if (stream) *stream = (void*)c->stream;
  return SGNB_OK;
}

const char* sgnb_status_string(int s) {
  switch (s) {
    case SGNB_OK: return "ok";
    case SGNB_ERR_INVALID: return "invalid argument";
    case SGNB_ERR_UNSUPPORTED: return "unsupported configuration";
    case SGNB_ERR_CUDA: return "CUDA error";
    case SGNB_ERR_NAN: return "non-finite state";
    case SGNB_ERR_DTMIN: return "step size below dtMin";
    case SGNB_ERR_TIMEOUT: return "device wait timed out";
    case SGNB_ERR_NOMEM: return "out of device memory";
    case SGNB_ERR_NO_DEVICE: return "no CUDA device";
    default: return "unknown status";
  }
}

const char* sgnb_last_error(const sgnb_ctx* c) {
  return c ? c->err.c_str() : g_create_error.c_str();
}

}  // extern "C"

// ===========================================================================
// Batched sweep: many independent instances, one persistent launch per RK stage.
// ===========================================================================
// launch configurations the autotuner tries per tile shape: one CTA per tile (grid
// option 0), then persistent grids of 1..4 CTAs per SM (options 1..4)
constexpr int kTuneGrids = 5;

struct sgnb_batch {
  int n = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<sgnb_ctx*> ctx;          // per-instance buffers and statics
  RhsConsts* dconsts = nullptr;        // [n]
  bool mixed = false;                  // every instance SGNB_MIXED (else SGNB_FP64_FAST)
  StageArgs* dargs = nullptr;          // [n]
  StageArgs* hargs = nullptr;          // pinned host mirror
  StageArgsM* dargsM = nullptr;        // [n], mixed batches
  StageArgsM* hargsM = nullptr;
  CtrlState* dctrl = nullptr;          // [n]
  CtrlState* hctrl = nullptr;          // pinned host mirror
  double* dpartbuf = nullptr;          // error partials of every instance, 3 per tile
  std::vector<double*> hpart;          // instance i's partials within dpartbuf
  double** dpart = nullptr;            // [n] partial pointers
  int* dnblk[3] = {nullptr, nullptr, nullptr};  // [n] tiles per instance, per tile shape
  long long* dntot = nullptr;          // [n]
  int* dtile_inst[3] = {nullptr, nullptr, nullptr};        // per tile shape
  long long* dtile_start[3] = {nullptr, nullptr, nullptr};
  long long ntiles[3] = {0, 0, 0};
  int shape = 0;                       // tuned tile shape
  int blocks = 0;                      // tuned persistent grid
  cudaGraphExec_t chunk = nullptr;     // the device-side loop of the tuned configuration
  int chunkShape = -1, chunkBlocks = -1;
  int* dcount = nullptr;               // [2] running instances, finished controller blocks
  cudaEvent_t evRead = nullptr;
  long long launches = 0;
  std::string err;
};

namespace {

int bfail(sgnb_batch* b, int code, const std::string& msg) {
  if (b) b->err = msg; else g_create_error = msg;
  return code;
}

#define SGNB_BCU(b, call)                                                    \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess)                                                   \
      return bfail(b, e_ == cudaErrorMemoryAllocation ? SGNB_ERR_NOMEM : SGNB_ERR_CUDA, \
                   std::string(#call) + ": " + cudaGetErrorName(e_));       \
  } while (0)

// One batched stage launch of either arithmetic mode.
cudaError_t batch_launch(sgnb_batch* b, int mode, int shape, int blocks, int kin_k2, double coef);

BatchArgs batch_args(sgnb_batch* b, int shape, int kin_k2, double coef) {
  BatchArgs B{};
  const RhsConsts& C0 = b->ctx[0]->C;
  for (int k = 0; k < 25; ++k) { B.tables.D[k] = C0.D[k]; B.tables.Df[k] = C0.Df[k]; }
  for (int k = 0; k < 5; ++k) {
    B.tables.gLp[k] = C0.gLp[k]; B.tables.gRp[k] = C0.gRp[k];
    B.tables.gLpf[k] = C0.gLpf[k]; B.tables.gRpf[k] = C0.gRpf[k];
  }
  B.consts = b->dconsts;
  B.args = b->dargs;
  B.tile_inst = b->dtile_inst[shape];
  B.tile_start = b->dtile_start[shape];
  B.ntiles = b->ntiles[shape];
  B.kin_k2 = kin_k2;
  B.coef = coef;
  return B;
}

// The batch's device-side loop: a WHILE conditional node whose body is one attempt of
// every instance (three batched stage launches and the batched loop controller, which
// keeps the loop going while any instance runs).
int batch_build_graph(sgnb_batch* b) {
  if (b->chunk && b->chunkShape == b->shape && b->chunkBlocks == b->blocks) return SGNB_OK;
  if (b->chunk) { cudaGraphExecDestroy(b->chunk); b->chunk = nullptr; }
  cudaGraph_t g = nullptr;
  SGNB_BCU(b, cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle loop;
  cudaError_t e = cudaGraphConditionalHandleCreate(&loop, g, 1, cudaGraphCondAssignDefault);
  cudaGraphNodeParams p = {};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = loop;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, nullptr, 0, &p);
  if (e == cudaSuccess) {
    cudaGraph_t body = p.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(b->stream, body, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      e = batch_launch(b, 1, b->shape, b->blocks, 0, 0.5);
      if (e == cudaSuccess) e = batch_launch(b, 1, b->shape, b->blocks, 1, 0.75);
      if (e == cudaSuccess) e = batch_launch(b, 2, b->shape, b->blocks, 0, 0.0);
      if (e == cudaSuccess)
        e = dev::launch_controller_batch_loop(b->dctrl, b->dpart, b->dnblk[b->shape], b->dntot,
                                              b->n, b->dcount, loop, b->stream);
      cudaError_t e2 = cudaStreamEndCapture(b->stream, &body);
      if (e == cudaSuccess) e = e2;
    }
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->chunk, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    b->chunk = nullptr;
    return bfail(b, SGNB_ERR_CUDA, std::string("batch loop graph: ") + cudaGetErrorName(e));
  }
  b->chunkShape = b->shape;
  b->chunkBlocks = b->blocks;
  return SGNB_OK;
}

bool all_done(const sgnb_batch* b) {
  for (int i = 0; i < b->n; ++i)
    if (!b->hctrl[i].done) return false;
  return true;
}

// Stage arguments of every instance and the controllers (already initialised in
// b->hctrl) to the device.
cudaError_t batch_launch(sgnb_batch* b, int mode, int shape, int blocks, int kin_k2, double coef) {
  if (!b->mixed) return dev::launch_fused_batch(mode, shape, blocks, batch_args(b, shape, kin_k2, coef), b->stream);
  if (shape != 0) return cudaErrorInvalidValue;  // mixed batches use 8x4 tiles
  const BatchArgs B = batch_args(b, 0, kin_k2, coef);
  BatchArgsM M{};
  M.tables = B.tables;
  M.consts = B.consts;
  M.args = b->dargsM;
  M.tile_inst = B.tile_inst;
  M.tile_start = B.tile_start;
  M.ntiles = B.ntiles;
  M.kin_k2 = kin_k2;
  M.coef = coef;
  return dev::launch_mixed_batch(mode, blocks, M, b->stream);
}

int batch_prepare(sgnb_batch* b) {
  if (b->mixed) {
    for (int i = 0; i < b->n; ++i) {
      sgnb_ctx* c = b->ctx[i];
      StageArgsM& A = b->hargsM[i];
      A = StageArgsM{};
      A.U[0] = c->U[0]; A.U[1] = c->U[1];
      A.K1[0] = (float*)c->K1[0]; A.K1[1] = (float*)c->K1[1];
      A.K2 = (float*)c->K2; A.K3 = (float*)c->K3;
      A.ctrl = b->dctrl + i;
      A.partials = b->hpart[i];
      A.in = c->U[c->cur];               // FSAL head: R(u) into K1[cur] (FP32)
      A.outd = nullptr;
      A.out = (float*)c->K1[c->cur];
    }
    SGNB_BCU(b, cudaMemcpyAsync(b->dargsM, b->hargsM, b->n * sizeof(StageArgsM), cudaMemcpyHostToDevice, b->stream));
    SGNB_BCU(b, cudaMemcpyAsync(b->dctrl, b->hctrl, b->n * sizeof(CtrlState), cudaMemcpyHostToDevice, b->stream));
    return SGNB_OK;
  }
  for (int i = 0; i < b->n; ++i) {
    sgnb_ctx* c = b->ctx[i];
    StageArgs& A = b->hargs[i];
    A = StageArgs{};
    A.U[0] = c->U[0]; A.U[1] = c->U[1];
    A.K1[0] = (double*)c->K1[0]; A.K1[1] = (double*)c->K1[1];
    A.K2 = (double*)c->K2; A.K3 = (double*)c->K3;
    A.ctrl = b->dctrl + i;
    A.partials = b->hpart[i];
    A.in = c->U[c->cur];          // FSAL head input and output
    A.out = (double*)c->K1[c->cur];
  }
  SGNB_BCU(b, cudaMemcpyAsync(b->dargs, b->hargs, b->n * sizeof(StageArgs), cudaMemcpyHostToDevice, b->stream));
  SGNB_BCU(b, cudaMemcpyAsync(b->dctrl, b->hctrl, b->n * sizeof(CtrlState), cudaMemcpyHostToDevice, b->stream));
  return SGNB_OK;
}

// Controllers already initialised in b->hctrl; runs until every instance is done, each
// graph launch up to 4096 attempts (a bound on one launch; the host then relaunches).
int batch_run(sgnb_batch* b) {
  constexpr long long kAttemptsPerLaunch = 4096;
  if (int rc = batch_build_graph(b)) return rc;
  long long a0 = 0;
  for (int i = 0; i < b->n; ++i) {
    b->hctrl[i].attemptCap = b->hctrl[i].attempts + kAttemptsPerLaunch;
    a0 = std::max(a0, b->hctrl[i].attempts);
  }
  if (int rc = batch_prepare(b)) return rc;
  SGNB_BCU(b, batch_launch(b, 0, b->shape, b->blocks, 0, 0.0));
  for (;;) {
    SGNB_BCU(b, cudaGraphLaunch(b->chunk, b->stream));
    SGNB_BCU(b, cudaMemcpyAsync(b->hctrl, b->dctrl, b->n * sizeof(CtrlState), cudaMemcpyDeviceToHost, b->stream));
    SGNB_BCU(b, cudaStreamSynchronize(b->stream));
    if (all_done(b)) break;
    for (int i = 0; i < b->n; ++i) b->hctrl[i].attemptCap = b->hctrl[i].attempts + kAttemptsPerLaunch;
    SGNB_BCU(b, cudaMemcpyAsync(b->dctrl, b->hctrl, b->n * sizeof(CtrlState), cudaMemcpyHostToDevice, b->stream));
  }
  long long a1 = 0;
  for (int i = 0; i < b->n; ++i) a1 = std::max(a1, b->hctrl[i].attempts);
  b->launches = 1 + 4 * (a1 - a0);
  for (int i = 0; i < b->n; ++i) b->ctx[i]->cur = b->hctrl[i].cur;
  return SGNB_OK;
}

}  // namespace

extern "C" {

int sgnb_checked_oob(int device, long long* count, int reset) {
  if (!count) return fail(nullptr, SGNB_ERR_INVALID, "count is NULL");
  *count = 0;
#ifdef SGNB_CHECKED
  cudaError_t e = cudaSetDevice(device);
  unsigned long long a = 0, b = 0, m = 0, j = 0;
  if (e == cudaSuccess) e = dev::read_oob_exact(&a, reset != 0);
  if (e == cudaSuccess) e = dev::read_oob_fast(&b, reset != 0);
  if (e == cudaSuccess) e = dev::read_oob_mixed(&m, reset != 0);
  if (e == cudaSuccess) e = dev::read_oob_adjoint(&j, reset != 0);
  if (e != cudaSuccess) return fail(nullptr, SGNB_ERR_CUDA, cudaGetErrorString(e));
  *count = (long long)(a + b + m + j);
  return SGNB_OK;
#else
  (void)device; (void)reset;
  return fail(nullptr, SGNB_ERR_UNSUPPORTED, "not the checked build (libsgnb_checked.so)");
#endif
}

int sgnb_fast_math(int fn, const double* x, double* y, long long n, void* stream) {
  if ((fn != 0 && fn != 1) || n < 0 || (n > 0 && (!x || !y)))
    return fail(nullptr, SGNB_ERR_INVALID, "fn 0 or 1, device arrays x, y of n doubles");
  cudaError_t e = dev::launch_fast_math(fn, x, y, n, (cudaStream_t)stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return fail(nullptr, SGNB_ERR_CUDA, cudaGetErrorString(e));
  return SGNB_OK;
}

int sgnb_set_ghosts(sgnb_ctx* c, const double* ghostL, const double* ghostR) {
  if (!c) return fail(c, SGNB_ERR_INVALID, "NULL context");
  if (c->tab.gauss) return fail(c, SGNB_ERR_UNSUPPORTED, "Gauss points run on whole meshes");
  if (c->mixed) return fail(c, SGNB_ERR_UNSUPPORTED, "slab edges run in the FP64 modes");
  c->C.ghostL = ghostL;
  c->C.ghostR = ghostR;
  if (c->chunk) {  // captured launches hold the old constants
    cudaGraphExecDestroy(c->chunk);
    c->chunk = nullptr;
    c->chunkLen = 0;
  }
  return SGNB_OK;
}

int sgnb_slab_pack(sgnb_ctx* c, int stage, const double* in, double* sendL, double* sendR,
                   void* stream) {
  if (!c || !sendL || !sendR || !(stage == 0 || stage == 2 || stage == 3 || stage == 4))
    return fail(c, SGNB_ERR_INVALID, "stage 0, 2, 3 or 4; send buffers");
  if (c->mixed) return fail(c, SGNB_ERR_UNSUPPORTED, "slab edges run in the FP64 modes");
  if (int rc = set_device(c)) return rc;
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  StageArgs A{};
  A.U[0] = c->U[0]; A.U[1] = c->U[1];
  A.K1[0] = (double*)c->K1[0]; A.K1[1] = (double*)c->K1[1];
  A.K2 = (double*)c->K2; A.K3 = (double*)c->K3;
  A.ctrl = c->dctrl;
  A.in = in ? in : c->U[c->cur];
  A.kin_k2 = stage == 3;
  A.coef = stage == 3 ? 0.75 : 0.5;
  const int mode = stage == 0 ? 0 : (stage == 4 ? 2 : 1);
  SGNB_CU(c, dev::launch_pack_ghosts(mode, c->C, A, sendL, sendR, s));
  return SGNB_OK;
}

int sgnb_slab_begin(sgnb_ctx* c, double t0, double tEnd, double dt0, long long nsteps,
                    const double* dts, const sgnb_rk_opts* opts) {
  if (!c || nsteps < 0 || !(dt0 > 0) || (nsteps == 0 && !(tEnd < 1e300)) || (dts && nsteps < 1))
    return fail(c, SGNB_ERR_INVALID, "dt0 > 0; nsteps >= 1, or nsteps = 0 and a finite tEnd");
  if (int rc = set_device(c)) return rc;
  sgnb_rk_opts o;
  if (opts) o = *opts; else sgnb_rk_opts_init(&o);
  CtrlState& h = *c->hctrl;
  init_ctrl(c, h, o);
  h.log = nullptr;
  h.t = t0;
  h.tEnd = tEnd < 1e300 ? tEnd : 1e300;
  h.dt = (o.dtMax < dt0) ? o.dtMax : dt0;
  h.errPrev = 1.0;
  h.tReached = t0;
  h.cur = c->cur;
  h.rhsEvals = 1;  // the FSAL head
  h.maxAccepted = nsteps;
  // loop test and end-time clip of the first attempt (rk.cpp:95-97)
  if (!(h.t < h.tEnd - 1e-15 * ((1.0 < std::fabs(h.tEnd)) ? std::fabs(h.tEnd) : 1.0))) h.done = 1;
  else if (h.t + h.dt > h.tEnd) h.dt = h.tEnd - h.t;
  if (dts) {  // frozen step sizes (bs3Step replay)
    if (nsteps > c->dtCap) {
      cudaFree(c->dtList);
      c->dtList = nullptr;
      SGNB_CU(c, cudaMalloc(&c->dtList, nsteps * sizeof(double)));
      c->dtCap = nsteps;
    }
    SGNB_CU(c, cudaMemcpy(c->dtList, dts, nsteps * sizeof(double), cudaMemcpyHostToDevice));
    h.frozen = 1;
    h.dtList = c->dtList;
    h.nList = nsteps;
    h.dt = dts[0];
  }
  SGNB_CU(c, cudaMemcpy(c->dctrl, c->hctrl, sizeof(CtrlState), cudaMemcpyHostToDevice));
  return SGNB_OK;
}

int sgnb_slab_launch(sgnb_ctx* c, int stage, void* stream) {
  if (!c || stage < 1 || stage > 4) return fail(c, SGNB_ERR_INVALID, "stage 1..4");
  if (c->mixed) return fail(c, SGNB_ERR_UNSUPPORTED, "slab edges run in the FP64 modes");
  if (int rc = set_device(c)) return rc;
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  if (stage == 1)  // FSAL head: k1 = R(u)
    SGNB_CU(c, launch(c, rhs_launch(c->U[c->cur], (double*)c->K1[c->cur]), s));
  else
    SGNB_CU(c, launch(c, stage_launch(stage), s));
  return SGNB_OK;
}

int sgnb_slab_stage(sgnb_ctx* c, int stage, const double* ghostL, const double* ghostR,
                    double* edgeL, double* edgeR, void* stream) {
  if (!c || stage < 1 || stage > 4) return fail(c, SGNB_ERR_INVALID, "stage 1..4");
  if (c->mixed || c->tab.gauss)
    return fail(c, SGNB_ERR_UNSUPPORTED, "slab edges run in the FP64 modes on GLL points");
  if ((edgeL && !ghostL) || (edgeR && !ghostR))
    return fail(c, SGNB_ERR_INVALID, "an edge output needs the neighbour's ghost input");
  if (int rc = set_device(c)) return rc;
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  if (c->chunk) {  // captured launches hold other constants
    cudaGraphExecDestroy(c->chunk);
    c->chunk = nullptr;
    c->chunkLen = 0;
  }
  c->C.ghostL = ghostL;
  c->C.ghostR = ghostR;
  const bool fused = stage == 2 || stage == 3;  // the next stage's inputs are known
  c->C.edgeL = fused ? edgeL : nullptr;
  c->C.edgeR = fused ? edgeR : nullptr;
  cudaError_t e;
  if (stage == 1) e = launch(c, rhs_launch(c->U[c->cur], (double*)c->K1[c->cur]), s);
  else e = launch(c, stage_launch(stage), s);
  c->C.edgeL = c->C.edgeR = nullptr;
  SGNB_CU(c, e);
  return SGNB_OK;
}

int sgnb_slab_control_all(sgnb_ctx* c, const double* const* partials, const int* nblk, int nslab,
                          long long n_total, void* stream) {
  if (!c || !partials || !nblk || nslab < 1 || nslab > dev::kMaxSlabs || n_total < 1)
    return fail(c, SGNB_ERR_INVALID, "1..32 slabs, their partials and block counts");
  if (int rc = set_device(c)) return rc;
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  dev::SlabPartials L{};
  L.ns = nslab;
  L.start[0] = 0;
  for (int k = 0; k < nslab; ++k) {
    if (!partials[k] || nblk[k] < 1) return fail(c, SGNB_ERR_INVALID, "bad partials");
    L.p[k] = partials[k];
    L.start[k + 1] = L.start[k] + nblk[k];
  }
  SGNB_CU(c, dev::launch_controller_slabs(c->dctrl, L, n_total, s));
  return SGNB_OK;
}

int sgnb_enable_peer_access(int device, int peer) {
  if (device == peer) return SGNB_OK;
  int can = 0;
  cudaError_t e = cudaDeviceCanAccessPeer(&can, device, peer);
  if (e != cudaSuccess) return fail(nullptr, SGNB_ERR_CUDA, cudaGetErrorString(e));
  if (!can) return fail(nullptr, SGNB_ERR_UNSUPPORTED, "the devices cannot address each other");
  if ((e = cudaSetDevice(device)) != cudaSuccess) return fail(nullptr, SGNB_ERR_CUDA, cudaGetErrorString(e));
  e = cudaDeviceEnablePeerAccess(peer, 0);
  if (e == cudaErrorPeerAccessAlreadyEnabled) {
    cudaGetLastError();  // clear the sticky-free status of the repeated call
    e = cudaSuccess;
  }
  if (e != cudaSuccess) return fail(nullptr, SGNB_ERR_CUDA, cudaGetErrorString(e));
  return SGNB_OK;
}

int sgnb_slab_partials(sgnb_ctx* c, double** partials, int* nblk) {
  if (!c || !partials || !nblk) return fail(c, SGNB_ERR_INVALID, "NULL argument");
  *partials = c->partials;
  *nblk = c->nblk;
  return SGNB_OK;
}

int sgnb_slab_control(sgnb_ctx* c, const double* partials, int nblk, long long n_total,
                      void* stream) {
  if (!c || !partials || nblk < 1 || n_total < 1) return fail(c, SGNB_ERR_INVALID, "bad arguments");
  if (int rc = set_device(c)) return rc;
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  SGNB_CU(c, dev::launch_controller(c->dctrl, partials, nblk, n_total, s));
  return SGNB_OK;
}

int sgnb_slab_status(sgnb_ctx* c, sgnb_rk_stats* st, int* done, void* stream) {
  if (!c) return fail(c, SGNB_ERR_INVALID, "NULL context");
  if (int rc = set_device(c)) return rc;
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  SGNB_CU(c, cudaMemcpyAsync(c->hctrl, c->dctrl, sizeof(CtrlState), cudaMemcpyDeviceToHost, s));
  SGNB_CU(c, cudaStreamSynchronize(s));
  const CtrlState& h = *c->hctrl;
  c->cur = h.cur;
  if (done) *done = h.done;
  if (st) {
    st->accepted = h.accepted; st->rejected = h.rejected; st->rhsEvals = h.rhsEvals;
    st->attempts = h.attempts; st->tReached = h.tReached; st->dtLast = h.dtLast;
    st->maxNormLast = h.maxNormLast;
    st->aborted = h.done == 2 ? 1 : (h.done == 3 ? 2 : 0);
    st->status = h.done == 3 ? SGNB_ERR_NAN : SGNB_OK;
    st->kernel_launches = 0;
  }
  return SGNB_OK;
}

int sgnb_eta_max(sgnb_ctx* c, double x0, double x1, double y0, double y1, double* eta_max,
                 long long* node) {
  if (!c || !eta_max || !node) return fail(c, SGNB_ERR_INVALID, "NULL argument");
  if (int rc = set_device(c)) return rc;
  const int nblk = c->ndiag / 2;
  SGNB_CU(c, dev::launch_eta_max(c->C, c->U[c->cur], x0, x1, y0, y1, c->mesh.hx, c->mesh.hy,
                                 c->mesh.ex0, c->tab.nodes, c->diag, nblk, c->stream));
  std::vector<double> part(2 * (size_t)nblk);
  SGNB_CU(c, cudaMemcpyAsync(part.data(), c->diag, part.size() * sizeof(double),
                             cudaMemcpyDeviceToHost, c->stream));
  SGNB_CU(c, cudaStreamSynchronize(c->stream));
  double best = -HUGE_VAL;
  long long bi = -1;
  for (int b = 0; b < nblk; ++b) {
    const long long i = (long long)part[2 * b + 1];
    if (i < 0) continue;
    if (bi < 0 || part[2 * b] > best || (part[2 * b] == best && i < bi)) {
      best = part[2 * b];
      bi = i;
    }
  }
  *eta_max = best;
  *node = bi;
  return SGNB_OK;
}

int sgnb_sample_eta(sgnb_ctx* c, const long long* nodes, int n, double* eta) {
  if (!c || n < 0 || (n > 0 && (!nodes || !eta))) return fail(c, SGNB_ERR_INVALID, "bad arguments");
  if (n == 0) return SGNB_OK;
  for (int k = 0; k < n; ++k)
    if (nodes[k] < 0 || nodes[k] >= c->Nd) return fail(c, SGNB_ERR_INVALID, "node out of range");
  if (int rc = set_device(c)) return rc;
  if (n > c->gaugeCap) {
    cudaFree(c->gauge);
    c->gauge = nullptr;
    c->gaugeCap = 0;
    SGNB_CU(c, cudaMalloc(&c->gauge, 2 * (size_t)n * sizeof(double)));
    c->gaugeCap = n;
  }
  long long* dn = reinterpret_cast<long long*>(c->gauge);
  double* dv = c->gauge + c->gaugeCap;
  SGNB_CU(c, cudaMemcpyAsync(dn, nodes, n * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
  SGNB_CU(c, dev::launch_sample_eta(c->U[c->cur], c->C.Hnod, dn, n, dv, c->stream));
  SGNB_CU(c, cudaMemcpyAsync(eta, dv, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  SGNB_CU(c, cudaStreamSynchronize(c->stream));
  return SGNB_OK;
}

int sgnb_element_means(sgnb_ctx* c, double* out) {
  if (!c || !out) return fail(c, SGNB_ERR_INVALID, "NULL argument");
  if (int rc = set_device(c)) return rc;
  const size_t n = 5 * (size_t)c->desc.Nx * c->desc.Ny;
  double* d = nullptr;
  SGNB_CU(c, cudaMalloc(&d, n * sizeof(double)));
  cudaError_t e = dev::launch_elem_means(c->C, c->U[c->cur], c->tab.qw, d, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(c, e, "element means");
  return SGNB_OK;
}

int sgnb_write_vtk(sgnb_ctx* c, const char* path) {
  if (!c || !path) return fail(c, SGNB_ERR_INVALID, "NULL argument");
  const int Nx = c->desc.Nx, Ny = c->desc.Ny;
  const size_t ne = (size_t)Nx * Ny;
  std::vector<double> m(5 * ne);
  if (int rc = sgnb_element_means(c, m.data())) return rc;
  std::FILE* fp = std::fopen(path, "w");
  if (!fp) return fail(c, SGNB_ERR_INVALID, std::string("cannot open ") + path);
  // legacy VTK, one point per element centre (the format of src/io/vtk2d.h:46-82)
  std::fprintf(fp, "# vtk DataFile Version 3.0\nSGN2D element means\nASCII\n");
  std::fprintf(fp, "DATASET STRUCTURED_POINTS\nDIMENSIONS %d %d 1\n", Nx, Ny);
  std::fprintf(fp, "ORIGIN %.6f %.6f 0\nSPACING %.6f %.6f 1\n",
               c->mesh.ex0 * c->mesh.hx + 0.5 * c->mesh.hx,
               0.5 * c->mesh.hy, c->mesh.hx, c->mesh.hy);
  std::fprintf(fp, "POINT_DATA %d\n", Nx * Ny);
  static const char* names[5] = {"eta", "u", "v", "p", "H"};
  for (int f = 0; f < 5; ++f) {
    std::fprintf(fp, "SCALARS %s float 1\nLOOKUP_TABLE default\n", names[f]);
    for (int ey = 0; ey < Ny; ++ey) {
      for (int ex = 0; ex < Nx; ++ex) std::fprintf(fp, "%.5e ", m[f * ne + ex + (size_t)Nx * ey]);
      std::fprintf(fp, "\n");
    }
  }
  const bool ok = std::fclose(fp) == 0;
  return ok ? SGNB_OK : fail(c, SGNB_ERR_INVALID, std::string("write failed: ") + path);
}

int sgnb_nearest_node(const sgnb_ctx* c, double x, double y, long long* node) {
  if (!c || !node) return SGNB_ERR_INVALID;
  // the node coordinates of node_coords, scanned per element in index order
  const int Nx = c->desc.Nx, Ny = c->desc.Ny;
  double best = HUGE_VAL;
  long long bi = -1;
  for (long long e = 0; e < (long long)Nx * Ny; ++e) {
    const int ex = (int)(e % Nx), ey = (int)(e / Nx);
    for (int b = 0; b < 5; ++b)
      for (int a = 0; a < 5; ++a) {
        const double xn = (c->mesh.ex0 + ex) * c->mesh.hx + 0.5 * c->mesh.hx * (c->tab.nodes[a] + 1.0);
        const double yn = ey * c->mesh.hy + 0.5 * c->mesh.hy * (c->tab.nodes[b] + 1.0);
        const double d2 = (xn - x) * (xn - x) + (yn - y) * (yn - y);
        if (d2 < best) { best = d2; bi = e * 25 + a + 5 * b; }
      }
  }
  *node = bi;
  return SGNB_OK;
}

int sgnb_batch_create(const sgnb_desc* descs, int n, sgnb_batch** out) {
  if (!out || !descs || n < 1) return bfail(nullptr, SGNB_ERR_INVALID, "descs, n >= 1, out");
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    if (descs[i].precision != SGNB_FP64_FAST && descs[i].precision != SGNB_MIXED)
      return bfail(nullptr, SGNB_ERR_UNSUPPORTED, "batched instances run in SGNB_FP64_FAST or SGNB_MIXED");
    if (descs[i].precision != descs[0].precision)
      return bfail(nullptr, SGNB_ERR_INVALID, "all instances of a batch in one arithmetic mode");
    if (descs[i].nManning != 0.0)
      return bfail(nullptr, SGNB_ERR_UNSUPPORTED, "batched instances run without Manning friction");
    if (descs[i].Nx_global > 0)
      return bfail(nullptr, SGNB_ERR_UNSUPPORTED, "batched instances are whole meshes");
    if (descs[i].point_set != SGNB_POINTS_GLL ||
        (descs[i].lL && descs[i].lL[0] != 1.0))
      return bfail(nullptr, SGNB_ERR_UNSUPPORTED, "batched instances use GLL points");
    if (descs[i].device != descs[0].device)
      return bfail(nullptr, SGNB_ERR_INVALID, "all instances on one device");
  }
  sgnb_batch* b = new sgnb_batch();
  b->mixed = descs[0].precision == SGNB_MIXED;
  b->n = n;
  b->device = descs[0].device;
  b->ctx.assign(n, nullptr);
  for (int i = 0; i < n; ++i) {
    int rc = sgnb_create(&descs[i], &b->ctx[i]);
    if (rc) { sgnb_batch_destroy(b); return rc; }
  }
  cudaSetDevice(b->device);
  auto bail = [&](cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorName(e);
    sgnb_batch_destroy(b);
    return bfail(nullptr, e == cudaErrorMemoryAllocation ? SGNB_ERR_NOMEM : SGNB_ERR_CUDA, m);
  };
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->evRead, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc(&b->dconsts, n * sizeof(RhsConsts));
  if (e == cudaSuccess) e = cudaMalloc(&b->dargs, n * sizeof(StageArgs));
  if (e == cudaSuccess) e = cudaMallocHost(&b->hargs, n * sizeof(StageArgs));
  if (e == cudaSuccess) e = cudaMalloc(&b->dargsM, n * sizeof(StageArgsM));
  if (e == cudaSuccess) e = cudaMallocHost(&b->hargsM, n * sizeof(StageArgsM));
  if (e == cudaSuccess) e = cudaMalloc(&b->dctrl, n * sizeof(CtrlState));
  if (e == cudaSuccess) e = cudaMalloc(&b->dcount, 2 * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(b->dcount, 0, 2 * sizeof(int));
  if (e == cudaSuccess) e = cudaMallocHost(&b->hctrl, n * sizeof(CtrlState));
  if (e == cudaSuccess) e = cudaMalloc(&b->dpart, n * sizeof(double*));
  if (e == cudaSuccess) e = cudaMalloc(&b->dntot, n * sizeof(long long));
  if (e != cudaSuccess) return bail(e, "batch buffers");
  std::vector<RhsConsts> hc(n);
  std::vector<long long> ht(n);
  for (int i = 0; i < n; ++i) {
    hc[i] = b->ctx[i]->C;
    ht[i] = b->ctx[i]->ntot;
  }
  e = cudaMemcpy(b->dconsts, hc.data(), n * sizeof(RhsConsts), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->dntot, ht.data(), n * sizeof(long long), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return bail(e, "batch upload");
  std::vector<long long> maxTiles(n, 0);
  // work lists per tile shape: instance-major tiles (8x4 tiles also fix the per-instance
  // partial count, which the controllers reduce; other shapes have more or fewer tiles)
  for (int sh = 0; sh < 3; ++sh) {
    const int tx = dev::batch_tile_tx(sh), ty = 32 / tx;
    std::vector<int> inst;
    std::vector<long long> start(n + 1, 0);
    std::vector<int> nb(n);
    for (int i = 0; i < n; ++i) {
      const long long nt = (long long)((b->ctx[i]->desc.Nx + tx - 1) / tx) *
                           ((b->ctx[i]->desc.Ny + ty - 1) / ty);
      start[i + 1] = start[i] + nt;
      inst.insert(inst.end(), (size_t)nt, i);
      nb[i] = (int)nt;
      if (nt > maxTiles[i]) maxTiles[i] = nt;
    }
    b->ntiles[sh] = start[n];
    e = cudaMalloc(&b->dnblk[sh], n * sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(b->dnblk[sh], nb.data(), n * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&b->dtile_inst[sh], inst.size() * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->dtile_start[sh], (n + 1) * sizeof(long long));
    if (e == cudaSuccess) e = cudaMemcpy(b->dtile_inst[sh], inst.data(), inst.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->dtile_start[sh], start.data(), (n + 1) * sizeof(long long), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return bail(e, "batch work list");
  }
  long long totPart = 0;
  for (int i = 0; i < n; ++i) totPart += 3 * maxTiles[i];
  e = cudaMalloc(&b->dpartbuf, totPart * sizeof(double));
  if (e != cudaSuccess) return bail(e, "batch partials");
  b->hpart.resize(n);
  for (long long i = 0, off = 0; i < n; off += 3 * maxTiles[i], ++i) b->hpart[i] = b->dpartbuf + off;
  e = cudaMemcpy(b->dpart, b->hpart.data(), n * sizeof(double*), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return bail(e, "batch partials");
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  b->shape = 0;
  b->blocks = 0;
  *out = b;
  return SGNB_OK;
}

int sgnb_batch_destroy(sgnb_batch* b) {
  if (!b) return SGNB_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->chunk) cudaGraphExecDestroy(b->chunk);
  if (b->evRead) cudaEventDestroy(b->evRead);
  cudaFree(b->dconsts); cudaFree(b->dargs); cudaFree(b->dctrl); cudaFree(b->dpart);
  cudaFree(b->dcount);
  cudaFree(b->dntot); cudaFree(b->dpartbuf);
  if (b->hargs) cudaFreeHost(b->hargs);
  cudaFree(b->dargsM);
  if (b->hargsM) cudaFreeHost(b->hargsM);
  if (b->hctrl) cudaFreeHost(b->hctrl);
  for (int sh = 0; sh < 3; ++sh) {
    cudaFree(b->dtile_inst[sh]); cudaFree(b->dtile_start[sh]); cudaFree(b->dnblk[sh]);
  }
  if (b->stream) cudaStreamDestroy(b->stream);
  for (sgnb_ctx* c : b->ctx) sgnb_destroy(c);
  delete b;
  return SGNB_OK;
}

int sgnb_batch_size(const sgnb_batch* b) { return b ? b->n : 0; }

int sgnb_batch_stream(const sgnb_batch* b, void** stream) {
  if (!b || !stream) return SGNB_ERR_INVALID;
  *stream = (void*)b->stream;
  return SGNB_OK;
}

sgnb_ctx* sgnb_batch_instance(sgnb_batch* b, int i) {
  return (b && i >= 0 && i < b->n) ? b->ctx[i] : nullptr;
}

int sgnb_batch_set_config(sgnb_batch* b, int shape, int blocks) {
  if (!b || shape < 0 || shape > 2 || blocks < 0) return bfail(b, SGNB_ERR_INVALID, "shape 0..2, blocks >= 0");
  if (b->mixed && shape != 0) return bfail(b, SGNB_ERR_UNSUPPORTED, "mixed batches use 8x4 tiles");
  b->shape = shape;
  b->blocks = blocks;
  return SGNB_OK;
}

int sgnb_batch_get_config(const sgnb_batch* b, int* shape, int* blocks) {
  if (!b) return SGNB_ERR_INVALID;
  if (shape) *shape = b->shape;
  if (blocks) *blocks = b->blocks;
  return SGNB_OK;
}

}  // extern "C"

namespace {
int batch_init_ctrls(sgnb_batch* b, const double* dt0, long long nsteps, const sgnb_rk_opts& o) {
  for (int i = 0; i < b->n; ++i) {
    CtrlState& h = b->hctrl[i];
    init_ctrl(b->ctx[i], h, o);
    h.log = nullptr;
    h.t = 0.0;
    h.tEnd = 1e300;
    h.dt = (o.dtMax < dt0[i]) ? o.dtMax : dt0[i];
    h.errPrev = 1.0;
    h.cur = b->ctx[i]->cur;
    h.rhsEvals = 1;
    h.maxAccepted = nsteps;
  }
  // the instances' own uploads ran on their context streams
  for (sgnb_ctx* c : b->ctx) SGNB_BCU(b, cudaStreamSynchronize(c->stream));
  return SGNB_OK;
}
}  // namespace

extern "C" {

int sgnb_batch_integrate_steps(sgnb_batch* b, const double* dt0, long long nsteps,
                               const sgnb_rk_opts* opts, sgnb_rk_stats* stats) {
  if (!b || !dt0 || nsteps < 1) return bfail(b, SGNB_ERR_INVALID, "dt0, nsteps >= 1");
  SGNB_BCU(b, cudaSetDevice(b->device));
  sgnb_rk_opts o;
  if (opts) o = *opts; else sgnb_rk_opts_init(&o);
  if (int rc = batch_init_ctrls(b, dt0, nsteps, o)) return rc;
  if (int rc = batch_run(b)) return rc;
  int status = SGNB_OK;
  for (int i = 0; i < b->n; ++i) {
    const CtrlState& h = b->hctrl[i];
    if (stats) {
      sgnb_rk_stats& st = stats[i];
      st.accepted = h.accepted; st.rejected = h.rejected; st.rhsEvals = h.rhsEvals;
      st.attempts = h.attempts; st.tReached = h.tReached; st.dtLast = h.dtLast;
      st.maxNormLast = h.maxNormLast;
      st.aborted = h.done == 2 ? 1 : (h.done == 3 ? 2 : 0);
      st.status = h.done == 3 ? SGNB_ERR_NAN : SGNB_OK;
      st.kernel_launches = b->launches;
    }
    if (h.done == 3) status = SGNB_ERR_NAN;
  }
  if (status) return bfail(b, status, "non-finite error estimate in an instance");
  return SGNB_OK;
}

int sgnb_batch_autotune(sgnb_batch* b, const double* dt0, int reps, double* ms_out) {
  if (!b || !dt0 || reps < 1) return bfail(b, SGNB_ERR_INVALID, "dt0, reps >= 1");
  SGNB_BCU(b, cudaSetDevice(b->device));
  sgnb_rk_opts o;
  sgnb_rk_opts_init(&o);
  // One attempt's three stage launches per repetition. Without the controller the
  // ping-pong index never flips, so the state the instances hold is left as it was:
  // the launches only write k2, k3, the other state buffer and the error partials.
  if (int rc = batch_init_ctrls(b, dt0, 1, o)) return rc;
  if (int rc = batch_prepare(b)) return rc;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  cudaEvent_t e0, e1;
  SGNB_BCU(b, cudaEventCreate(&e0));
  SGNB_BCU(b, cudaEventCreate(&e1));
  double best = 1e300;
  int bestShape = 0, bestBlocks = 0;
  int rc = SGNB_OK;
  if (ms_out)
    for (int q = 0; q < 3 * kTuneGrids; ++q) ms_out[q] = -1.0;  // shapes not tried
  for (int sh = 0; sh < (b->mixed ? 1 : 3) && rc == SGNB_OK; ++sh) {
    for (int f = 0; f < kTuneGrids && rc == SGNB_OK; ++f) {
      const int blocks = f * sms;
      auto run = [&](int count) {
        cudaError_t e = cudaSuccess;
        for (int r = 0; r < count && e == cudaSuccess; ++r) {
          e = batch_launch(b, 1, sh, blocks, 0, 0.5);
          if (e == cudaSuccess) e = batch_launch(b, 1, sh, blocks, 1, 0.75);
          if (e == cudaSuccess) e = batch_launch(b, 2, sh, blocks, 0, 0.0);
        }
        return e;
      };
      cudaError_t e = run(1);
      if (e == cudaSuccess) e = cudaEventRecord(e0, b->stream);
      if (e == cudaSuccess) e = run(reps);
      if (e == cudaSuccess) e = cudaEventRecord(e1, b->stream);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e != cudaSuccess) { rc = bfail(b, SGNB_ERR_CUDA, std::string("autotune: ") + cudaGetErrorName(e)); break; }
      const double per = (double)ms / reps;
      if (ms_out) ms_out[sh * kTuneGrids + f] = per;
      if (per < best) { best = per; bestShape = sh; bestBlocks = blocks; }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  b->shape = bestShape;
  b->blocks = bestBlocks;
  return SGNB_OK;
}

const char* sgnb_batch_last_error(const sgnb_batch* b) {
  return b ? b->err.c_str() : g_create_error.c_str();
}

}  // extern "C"
