// sgnb_device.h -- parameter blocks shared by the host code and the sm_100a kernels.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

namespace sgnb {

// Everything the fused right-hand-side kernel needs besides the state: mesh size,
// boundary kinds, the physical constants in the exact forms the reference multiplies
// them in (src/physics/sgn_flux2d.h:89-161), the FR tables, and the bathymetry statics.
struct RhsConsts {
  int Nx, Ny;          // elements per direction
  int bcx, bcy;        // 0 periodic, 1 reflective wall
  long long Nd;        // nodes per field = 25 Nx Ny
  double g;            // gravity
  double halfg;        // 0.5 * g
  double gamma;        // dispersion parameter
  double c2;           // c * c
  double mc2;          // (-c) * c, the ncp coefficient
  double m2c2;         // -2.0 * c2, the relaxation-source coefficient
  double n2g;          // nManning^2 * g: Manning friction (sgn_flux2d.h:135-142)
  int manning;         // friction on (nManning != 0)
  int pad_;
  double Jx, Jy;       // affine Jacobians hx/2, hy/2
  double iJx, iJy;     // 1/Jx, 1/Jy (fast mode)
  double D[25];        // GLL differentiation matrix, row-major
  double gLp[5], gRp[5];  // g_DG correction derivatives
  // bathymetry statics (device pointers)
  const double* Hnod;    // nodal H, Nd
  const double* Hx;      // nodal dH/dx, Nd
  const double* Hy;      // nodal dH/dy, Nd
  const double* HfX;     // H at the left edge of each element, 5 per element
  const double* HfY;     // H at the bottom edge of each element
  const double* HfXEnd;  // H on the right domain edge (walls), 5 per row
  const double* HfYEnd;  // H on the top domain edge (walls), 5 per column
  // slab edges (x decomposition): the neighbours' trace nodes across the left and right
  // edge, [field][row][transverse node], stage inputs formed by the neighbours; NULL: the
  // edge follows bcx (periodic wrap or wall)
  const double* ghostL;
  const double* ghostR;
  // fused edge exchange of the intermediate stages: the next stage's inputs at the slab's
  // edge nodes, written by this launch into the neighbours' ghost arrays (the left
  // neighbour's right ghost, the right neighbour's left ghost; another device's memory in
  // a multi-device run); NULL: none
  double* edgeL;
  double* edgeR;
  // Gauss-Legendre points: face interpolation rows, and the face traces of every element
  // formed by a pre-pass, [face: 0 left, 1 right, 2 bottom, 3 top][field][element][node]
  double lL[5], lR[5];
  double* tr;
  int gauss;
  int pad2_;
  // the differentiation and correction tables rounded to FP32 (the mixed mode's FP32
  // contractions)
  float Df[25], gLpf[5], gRpf[5];
};

// Device-resident state of the adaptive integrator: the scalar loop variables of
// src/solver/rk.cpp:67-164 plus the index of the buffer pair that holds u and k1.
struct CtrlState {
  double t, dt, tEnd, errPrev;
  double tReached, dtLast, maxNormLast, errLast;
  long long accepted, rejected, rhsEvals, attempts;
  int cur;     // U[cur] holds u, K1[cur] holds k1
  int done;    // 0 running, 1 reached tEnd, 2 dt fell below dtMin, 3 non-finite error
  int frozen;  // 1: replay the dt list (every attempt accepted)
  int pad;
  double atol, rtol, dtMin, dtMax, safety, facMin, facMax, alpha, beta;
  const double* dtList;  // frozen-dt replay list
  long long nList;
  double* log;           // attempt log: (t, dt, errNorm, accepted) per attempt
  long long logCap;      // capacity of the log in attempts
  long long maxAccepted; // > 0: stop after this many accepted steps
  long long attemptCap;  // the device-side loop hands back to the host at this attempt count
};

#ifdef __CUDACC__
// The controller's per-launch values (buffer index, dt, tolerances) read again late in a
// stage kernel, through the read-only path: the controller state does not change while a
// stage kernel runs (the controller kernel writes it between launches), so after the
// first read on an SM the line comes from L1 instead of an L2 round trip. Asm statements,
// so the compiler neither merges them with the kernel's first read nor keeps that value
// live in registers in between.
struct CtrlReload {
  int cur;
  double dt, atol, rtol;
};
__device__ __forceinline__ CtrlReload ctrl_reload(const CtrlState* c) {
  CtrlReload r;
  asm volatile("ld.global.nc.s32 %0, [%1];" : "=r"(r.cur) : "l"(&c->cur));
  asm volatile("ld.global.nc.f64 %0, [%1];" : "=d"(r.dt) : "l"(&c->dt));
  asm volatile("ld.global.nc.f64 %0, [%1];" : "=d"(r.atol) : "l"(&c->atol));
  asm volatile("ld.global.nc.f64 %0, [%1];" : "=d"(r.rtol) : "l"(&c->rtol));
  return r;
}

// Block-wide copy of two parameter blocks (W1 and W2 32-bit words) from global to shared
// memory, by NT threads: every load of a thread is issued before its first store, so the
// copy costs one memory round trip however many words a thread moves.
template <int W1, int W2, int NT>
__device__ __forceinline__ void block_copy2(unsigned* d1, const unsigned* s1, unsigned* d2,
                                            const unsigned* s2) {
  constexpr int R1 = (W1 + NT - 1) / NT, R2 = (W2 + NT - 1) / NT;
  unsigned t1[R1], t2[R2];
  const int tid = threadIdx.x;
#pragma unroll
  for (int r = 0; r < R1; ++r)
    if (tid + r * NT < W1) t1[r] = s1[tid + r * NT];
#pragma unroll
  for (int r = 0; r < R2; ++r)
    if (tid + r * NT < W2) t2[r] = s2[tid + r * NT];
#pragma unroll
  for (int r = 0; r < R1; ++r)
    if (tid + r * NT < W1) d1[tid + r * NT] = t1[r];
#pragma unroll
  for (int r = 0; r < R2; ++r)
    if (tid + r * NT < W2) d2[tid + r * NT] = t2[r];
}

// Tile loads by the tensor-memory accelerator, completed on a shared-memory mbarrier
// (one elected thread initialises it and issues the copies; every thread waits on its
// phase with a bounded number of tries). Loads from this device's own buffers only, each
// into the issuing CTA's own shared memory.
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned mb) {
  asm volatile("mbarrier.init.shared.b64 [%0], 1;\n" ::"r"(mb) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned mb, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared.b64 _, [%0], %1;\n" ::"r"(mb), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned mb, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(mb), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void mbar_inval(unsigned mb) {
  asm volatile("mbarrier.inval.shared.b64 [%0];\n" ::"r"(mb) : "memory");
}
__device__ __forceinline__ void tma_load_3d(unsigned dst, const CUtensorMap* map, int x, int y,
                                            int z, unsigned mb) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(dst),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(mb)
      : "memory");
}
__device__ __forceinline__ void tma_load_2d(unsigned dst, const CUtensorMap* map, int x, int y,
                                            unsigned mb) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
      "l"(map), "r"(x), "r"(y), "r"(mb)
      : "memory");
}
// Tries before a tile-load wait gives up (each try waits a while in hardware): far more
// than any load takes, so a give-up means a fault, reported as a non-finite result.
constexpr int kTmaTries = 1 << 20;
#endif

// Tensor maps of a context's FP64 buffers for the fused kernels' tile loads on meshes that
// are a whole number of 8x4 tiles: each state-sized buffer as [field][element row]
// [Nx * 25 nodes] with an [5][4][200] box (one tile's 5 x 32 x 25 doubles, in the shared
// layout), the nodal depth as [element row][Nx * 25] with a [4][200] box. ok = 0: none.
// In: the right-hand-side mode's input (any 16-byte-aligned device state, encoded per
// launch); inOk = 0: none.
struct TileMaps {
  CUtensorMap U[2], K1[2], K2, K3, H, In;
  int ok, inOk;
};

// The mixed-precision mode's counterparts (intermediate stage): the FP32 stage buffers as
// [field][element row][Nx * 25] with a [1][4][200] box (one field of one tile per copy),
// the nodal depth as for the FP64 kernels.
struct TileMapsM {
  CUtensorMap K1[2], K2, K3, H;
  int ok;
};

// Buffers of one fused launch.
struct StageArgs {
  const double* in;   // MODE_RHS input state
  double* out;        // MODE_RHS / MODE_STAGE output derivative
  double* U[2];       // state ping-pong pair
  double* K1[2];      // k1 / k4 ping-pong pair
  double* K2;
  double* K3;
  int kin_k2;         // MODE_STAGE: add k2 (1) or k1 = K1[cur] (0) to u
  double coef;        // MODE_STAGE: 0.5 or 0.75
  const CtrlState* ctrl;
  double* partials;   // MODE_FSAL: 3 doubles per CTA (sum r^2, max |r|, NaN count)
};

// Buffers of one mixed-precision launch: FP64 state, FP32 stage derivatives.
struct StageArgsM {
  const double* in;   // MODE_RHS input state
  double* outd;       // MODE_RHS output derivative (FP64)
  float* out;         // MODE_STAGE output derivative
  double* U[2];
  float* K1[2];
  float* K2;
  float* K3;
  int kin_k2;
  double coef;
  const CtrlState* ctrl;
  double* partials;
};

// Work list of a batched launch: tile t belongs to instance tile_inst[t] and is that
// instance's local tile t - tile_start[inst]; per-instance constants and buffers.
struct FrTablesDev {
  double D[25], gLp[5], gRp[5];
  float Df[25], gLpf[5], gRpf[5];  // FP32 roundings (mixed mode)
};

struct BatchArgs {
  FrTablesDev tables;   // shared by every instance (P = 4 GLL)
  const RhsConsts* consts;
  const StageArgs* args;
  const int* tile_inst;
  const long long* tile_start;
  long long ntiles;
  int kin_k2;
  double coef;
};

// Vector-Jacobian product of R at a stage input y = u (k == nullptr) or u + acoef k,
// with the cotangent alpha ra + beta rb (rb optional). Scratch written by the line
// kernels and read by the gather kernel:
//   Ub[d]   [5 Nd]   cotangent of each node from its direction-d line
//   Hb[d]   [Nd]     nodal-depth cotangent from the direction-d lines
//   Hxb,Hyb [Nd]     cotangents of dH/dx, dH/dy (x lines: sources)
//   Sn[d][f][5 ne 5] cotangent of the neighbour's trace node across face f (0 low,
//                    1 high) of line (e, j), field-minor
//   Hf[d][f][5 ne]   cotangent of the face depth of face f of line (e, j)
struct VjpArgs {
  const double* u;
  const double* k;
  double acoef;
  const double* ra;
  const double* rb;
  double alpha, beta;
  double* Ub[2];
  double* Hb[2];
  double* Hxb;
  double* Hyb;
  double* Sn[2][2];
  double* Hf[2][2];
};

// Outputs of the gather: ybar (optional) = the node cotangent of R's input;
// uacc = lam + ybar (init; lam optional) or uacc += ybar; statics accumulators +=.
struct GatherArgs {
  double* ybar;
  double* uacc;
  const double* lam;
  int init;
  double* Hacc;
  double* Hxacc;
  double* Hyacc;
  double* HfXacc;
  double* HfYacc;
  double* HfXEndacc;
  double* HfYEndacc;
};

// Work list of a batched mixed-precision launch (8x4 tiles), as BatchArgs.
struct BatchArgsM {
  FrTablesDev tables;
  const RhsConsts* consts;
  const StageArgsM* args;
  const int* tile_inst;
  const long long* tile_start;
  long long ntiles;
  int kin_k2;
  double coef;
};

namespace dev {
// Batched mixed-precision launch: `blocks` persistent CTAs, or one CTA per tile (0).
cudaError_t launch_mixed_batch(int mode, int blocks, const BatchArgsM& B, cudaStream_t s);
cudaError_t prepare_mixed_batch();

// Out-of-range access counts of the checked build (exact and fast translation units).
cudaError_t read_oob_exact(unsigned long long* out, bool reset);
cudaError_t read_oob_fast(unsigned long long* out, bool reset);
cudaError_t read_oob_mixed(unsigned long long* out, bool reset);
cudaError_t read_oob_adjoint(unsigned long long* out, bool reset);

// The fast mode's reciprocal (fn 0) and square root (fn 1) elementwise, for tests.
cudaError_t launch_fast_math(int fn, const double* x, double* y, long long n, cudaStream_t s);

// Error partials of every slab of a decomposed mesh, in slab order: slab s holds blocks
// start[s] .. start[s+1]-1 at p[s] (3 doubles per block).
constexpr int kMaxSlabs = 32;
struct SlabPartials {
  const double* p[kMaxSlabs];
  long long start[kMaxSlabs + 1];
  int ns;
};
cudaError_t launch_controller_slabs(CtrlState* c, const SlabPartials& L, long long n,
                                    cudaStream_t s);

// Slab edges: the stage inputs of the first and last element columns' edge nodes
// (a = 0 / a = 4), [field][row][node], for the neighbours' ghosts. mode 0: rhs of in;
// 1: intermediate stage (kin_k2, coef of A); 2: end-point candidate.
cudaError_t launch_pack_ghosts(int mode, const RhsConsts& C, const StageArgs& A, double* sendL,
                               double* sendR, cudaStream_t s);

// Adjoint kernels (FP64, fast arithmetic).
cudaError_t launch_vjp_rhs(const RhsConsts& C, const FrTablesDev& T, const VjpArgs& A,
                           const GatherArgs& G, cudaStream_t s);
cudaError_t launch_rk_update(const double* u, const double* k1, const double* k2,
                             const double* k3, const double* dts, long long step, double* out,
                             long long n, cudaStream_t s);
cudaError_t launch_gauges(const double* U, const double* Hnod, const long long* nodes, int ng,
                          double* eta, cudaStream_t s);
cudaError_t launch_gauges_back(double* lam, const long long* nodes, int ng, const double* etab,
                               cudaStream_t s);

// Launchers (one translation unit per arithmetic mode).
// M: tensor maps of the buffers A names (the context's own), or nullptr (no tile loads
// by the tensor-memory accelerator).
cudaError_t launch_fused_exact(int mode, const RhsConsts& C, const StageArgs& A,
                               cudaStream_t s, const TileMaps* M = nullptr);
cudaError_t launch_fused_fast(int mode, const RhsConsts& C, const StageArgs& A,
                              cudaStream_t s, const TileMaps* M = nullptr);
cudaError_t prepare_fused_exact();
cudaError_t prepare_fused_fast();
cudaError_t launch_fused_mixed(int mode, const RhsConsts& C, const StageArgsM& A,
                               cudaStream_t s, const TileMapsM* M = nullptr);
cudaError_t prepare_fused_mixed();
int fused_grid_blocks(int Nx, int Ny);
// Batched launch (FP64 fast): tile shape shape_id (0: 8x4, 1: 16x2, 2: 4x8); `blocks`
// persistent CTAs looping over the work list, or one CTA per tile when blocks == 0.
cudaError_t launch_fused_batch(int mode, int shape_id, int blocks, const BatchArgs& B,
                               cudaStream_t s);
cudaError_t prepare_fused_batch();
int batch_tile_tx(int shape_id);
cudaError_t launch_controller_batch(CtrlState* ctrls, const double* const* partials,
                                    const int* nblk, const long long* n, int ninst,
                                    cudaStream_t s);
// rk4Step: c->dt = dts[i], and the final update u += dt/6 (k1 + 2 k2 + 2 k3 + k4) over n values
cudaError_t launch_rk4_set_dt(CtrlState* c, const double* dts, long long i, cudaStream_t s);
cudaError_t launch_rk4_update(double* u, const double* k1, const double* k2, const double* k3,
                              const double* k4, const CtrlState* c, long long n, int sms,
                              cudaStream_t s);
size_t fused_smem_bytes();

// Controller of one adaptive attempt: deterministic reduction of the per-CTA error
// partials, accept/reject, PI step-size update and the next attempt's dt.
// The controller as the last node of the body of a device-side WHILE loop (a conditional
// node of a CUDA graph): it also sets the loop condition, false once the run is done or
// the attempt count has reached attemptCap.
cudaError_t launch_controller_loop(CtrlState* c, const double* partials, int nblk, long long n,
                                   cudaGraphConditionalHandle loop, cudaStream_t s);
// Batched form of the loop controller: block i runs instance i's controller; every block
// counts whether its instance still runs, and the last block to finish (an atomic ticket,
// no waiting) sets the condition (any instance running) and clears the two counters.
cudaError_t launch_controller_batch_loop(CtrlState* ctrls, const double* const* partials,
                                         const int* nblk, const long long* n, int ninst,
                                         int* counters, cudaGraphConditionalHandle loop,
                                         cudaStream_t s);
cudaError_t launch_controller(CtrlState* c, const double* partials, int nblk,
                              long long n, cudaStream_t s);
// Largest eta = h - H inside a window, with its node: (value, index) per block.
cudaError_t launch_eta_max(const RhsConsts& C, const double* U, double x0, double x1, double y0,
                           double y1, double hx, double hy, int ex0, const double* xi,
                           double* out, int nblk, cudaStream_t s);
// Element means of eta, u, v, p, H (out[f * ne + e]), as the reference's VTK writer forms them.
cudaError_t launch_elem_means(const RhsConsts& C, const double* U, const double* qw, double* out,
                              cudaStream_t s);
// eta at the given nodes (gauges).
cudaError_t launch_sample_eta(const double* U, const double* Hnod, const long long* nodes, int n,
                              double* out, cudaStream_t s);
// Reductions over the uploaded state (diagnostics).
cudaError_t launch_reduce_diag(int what, const RhsConsts& C, const double* U,
                               const double* qw, double* out_partials, int nblk,
                               cudaStream_t s);
}  // namespace dev

}  // namespace sgnb
