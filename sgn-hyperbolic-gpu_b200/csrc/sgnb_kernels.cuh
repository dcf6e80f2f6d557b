// sgnb_kernels.cuh -- fused sm_100a kernels for the 2D hyperbolic-SGN FR right-hand side
// and the Bogacki-Shampine 3(2) stage loop.
//
// One launch evaluates the whole right-hand side R(U) of a tile of elements: the five
// phases of the reference CPU solver (face traces, nodal fluxes with per-direction GLL
// differentiation, Rusanov interface fluxes with central depths, the element's own
// face fluxes, FR correction lift + depth gradients + non-conservative products +
// sources; src/solver/sgn2d.cpp:125-290) run out of shared memory, and the only HBM
// traffic is the state in, the bathymetry statics in and dU out.
//
// The same kernel body also serves the three Runge-Kutta stages of one BS3(2) attempt
// (src/solver/rk.cpp:95-131): the stage input u + a dt k, or the third-order candidate
// uNew, is formed while the tile is loaded, and the end-point stage additionally
// writes uNew and reduces the scaled embedded error of its tile.
//
// Work decomposition. A CTA owns a tile of TX x TY elements (element-contiguous rows of
// the reference's variable-major layout U[v*Nd + e*25 + a + 5b], e = ex + Nx*ey) and
// runs 5 warps. Lane i of every warp is tile element i; warp j is the element's
// j-th GLL line:
//   column pass: warp j handles the y-line a = j (y-fluxes, bottom/top Rusanov,
//                y-derivatives, depth gradient h_y, ncpY) and hands dG, By over in
//                shared memory;
//   row pass:    warp j handles the x-line b = j (x-fluxes, left/right Rusanov,
//                x-derivatives, h_x, ncpX, sources) and assembles dU.
// Every 5-point contraction is thread-local (the line lives in registers), and the
// tables D, gL', gR' are warp-uniform kernel parameters.
//
// Two arithmetic modes, compiled as separate translation units:
//   EXACT (sgnb_kernels_exact.cu, -fmad=false): the reference CPU operation order,
//         IEEE division by the Jacobians, face traces formed as 0.0 + v exactly like the
//         reference's sum over unit GLL interpolation rows; bit-identical to the CPU;
//   FAST  (sgnb_kernels_fast.cu, -fmad=true): reciprocal of h and of the Jacobians,
//         FMA contraction, redundant work removed; agrees to round-off (<1e-13 rel).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "sgnb_device.h"
#include "sgnb_checked.cuh"
#include "sgnb_fastmath.cuh"

namespace sgnb {
namespace dev {

constexpr int NP = 5;          // GLL points per direction (P = 4)
constexpr int NPP = 25;        // nodes per element
constexpr int NV = 5;          // conserved fields h, hu, hv, hw, hp
constexpr int TE = 32;         // elements per tile = lanes per warp
constexpr int NWARP = 5;       // one warp per GLL line index
constexpr int NTHR = 32 * NWARP;
constexpr int NIT = TE * NPP / NTHR;                   // own-node items per thread
static_assert(TE * NPP == NIT * NTHR, "own nodes split evenly over the threads");

// Stage modes of the fused kernel.
enum : int {
  MODE_RHS = 0,    // dU = R(U)
  MODE_STAGE = 1,  // k_out = R(u + coef*dt*k_in)
  MODE_FSAL = 2    // uNew = u + dt(2/9 k1 + 1/3 k2 + 4/9 k3); k4 = R(uNew); error partials
};

// A tile of TX x TY = 32 elements (TX in 4, 8, 16) and its shared-memory layout.
template <int TX_, int TY_, bool EXACT_ = false>
struct Tile {
  static constexpr int TX = TX_, TY = TY_;
  static_assert(TX * TY == TE, "one tile element per lane");
  static constexpr int NHALO = 2 * TY + 2 * TX;                 // halo slots per field
  static constexpr int RUN = TX * NPP;                          // doubles per tile row and field
  static constexpr int NHIT = (NV * NHALO * NP + NTHR - 1) / NTHR;  // halo items per thread
  static constexpr int NFACE = (2 * TE + TY + TX) * NP;
  static constexpr int NFIT = (NFACE + NTHR - 1) / NTHR;        // face-depth items per thread
  struct Smem {
    double U[NV][TE][NPP];       // tile state (input of R)
    double H[TE][NPP];           // nodal still depth (its gradient is formed from it)
    // column-pass results dG (5 fields) and, in the exact mode, By on its own (the fast
    // mode adds By to the hp field's dG); then dU
    double G[NV + (EXACT_ ? 1 : 0)][TE][NPP];
    // halo node states, flat index q = t + NP * (slot + NHALO * v):
    //   slot 0..TY-1        node (4,t) of the element left of tile row slot
    //   slot TY..2TY-1      node (0,t) of the element right of tile row slot-TY
    //   slot 2TY..2TY+TX-1  node (t,4) of the element below tile column slot-2TY
    //   slot 2TY+TX..       node (t,0) of the element above tile column slot-2TY-TX
    double halo[NV * NHALO * NP];
    // face depths, flat: HfX[TE][NP] (left edges), HfY[TE][NP] (bottom edges),
    // HfXR[TY][NP] (right edge of the last tile column), HfYT[TX][NP] (top edge of the
    // last tile row)
    double Hf[NFACE];
    double red[NWARP][3];        // block reduction of the error partials
  };
  static __device__ __forceinline__ double& hf_x(Smem& S, int i, int t) { return S.Hf[i * NP + t]; }
  static __device__ __forceinline__ double& hf_y(Smem& S, int i, int t) { return S.Hf[(TE + i) * NP + t]; }
  static __device__ __forceinline__ double& hf_xr(Smem& S, int iy, int t) { return S.Hf[(2 * TE + iy) * NP + t]; }
  static __device__ __forceinline__ double& hf_yt(Smem& S, int ix, int t) { return S.Hf[(2 * TE + TY + ix) * NP + t]; }
  static __device__ __forceinline__ double& halo_at(Smem& S, int v, int slot, int t) {
    return S.halo[t + NP * (slot + NHALO * v)];
  }
};

// Resident CTAs per SM the fast-mode single-instance kernels are compiled for (the
// register budget per thread follows: 2 -> 168 registers, 3 -> 128).
#ifndef SGNB_FAST_MIN_CTAS
#define SGNB_FAST_MIN_CTAS 2
#endif

// Asynchronous global -> shared copy of one double (cp.async, no register staging), and
// the wait for all of this thread's outstanding copies.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}


// Read-only views of the stage inputs of one launch.
struct StageIn {
  const double* __restrict__ in;
  const double* __restrict__ u;
  const double* __restrict__ k;   // MODE_STAGE: the derivative added to u
  const double* __restrict__ k1;
  const double* __restrict__ k2;
  const double* __restrict__ k3;
  double acoef, dt;
};

// Stage combinations of src/solver/rk.cpp:100-108, with every product and sum rounded on
// its own in both arithmetic modes: a tile forms its own nodes in shared memory and its
// neighbours' halo nodes in registers, and the two must agree bit for bit.
__device__ __forceinline__ double stage_axpy(double u, double acoef, double k) {
  return __dadd_rn(u, __dmul_rn(acoef, k));  // u + (c dt) k
}
__device__ __forceinline__ double fsal_part(double k1, double k2) {
  return __dadd_rn(__dmul_rn(2.0 / 9.0, k1), __dmul_rn(1.0 / 3.0, k2));  // 2/9 k1 + 1/3 k2
}
__device__ __forceinline__ double fsal_finish(double u, double part, double k3, double dt) {
  return __dadd_rn(u, __dmul_rn(dt, __dadd_rn(part, __dmul_rn(4.0 / 9.0, k3))));
}

// Stage input of one value: plain, u + (coef dt) k, or the BS3 candidate.
template <int MODE>
__device__ __forceinline__ double stage_value(const StageIn& I, long long idx) {
  if constexpr (MODE == MODE_RHS) {
    return I.in[idx];
  } else if constexpr (MODE == MODE_STAGE) {
    return stage_axpy(I.u[idx], I.acoef, I.k[idx]);
  } else {
    return fsal_finish(I.u[idx], fsal_part(I.k1[idx], I.k2[idx]), I.k3[idx], I.dt);
  }
}

template <bool EXACT>
__device__ __forceinline__ double canon(double v) {
  // The reference forms face traces as sum_a lL[a] * U_a starting from 0.0 with unit
  // GLL rows (src/solver/sgn2d.cpp:157-161); the result is 0.0 + U_edge, which turns a
  // negative zero into a positive one. The exact mode reproduces that.
  if constexpr (EXACT) return v + 0.0; else return v;
}

// Primitive variables u, v, w, p of one point (src/physics/sgn_flux2d.h:92-93).
template <bool EXACT>
struct Prim {
  double u, v, w, p;
  __device__ __forceinline__ Prim() {}
  __device__ __forceinline__ explicit Prim(const double* U) {
    if constexpr (EXACT) {
      u = U[1] / U[0]; v = U[2] / U[0]; w = U[3] / U[0]; p = U[4] / U[0];
    } else {
      const double ih = fast_rcp(U[0]);
      u = U[1] * ih; v = U[2] * ih; w = U[3] * ih; p = U[4] * ih;
    }
  }
};

// Hydrostatic part 0.5 g (h^2 - H^2) of the normal momentum flux. h^2 - H^2 cancels
// where h ~ H; both modes round the two squares separately, as the CPU does, because
// the derivative amplifies this term's rounding by ~|D|/J.
template <class TC>
__device__ __forceinline__ double hydro(const TC& C, double h, double Hloc) {
  return C.halfg * (__dmul_rn(h, h) - __dmul_rn(Hloc, Hloc));
}

// Normal-momentum component of the directional flux (sgn_flux2d.h:94, 109).
template <bool EXACT, int DIR, class TC>
__device__ __forceinline__ double flux_normal(const TC& C, const double* U,
                                              const Prim<EXACT>& q, double Hloc) {
  const double hn = DIR == 0 ? U[1] : U[2];
  const double hp = EXACT ? U[0] * q.p : U[4];
  return hn * (DIR == 0 ? q.u : q.v) + hydro(C, U[0], Hloc) + hp;
}

// Directional flux: fluxX (DIR 0) or fluxY (DIR 1), src/physics/sgn_flux2d.h:89-116.
template <bool EXACT, int DIR, class TC>
__device__ __forceinline__ void flux(const TC& C, const double* U, const Prim<EXACT>& q,
                                     double Hloc, double* F) {
  const double hn = DIR == 0 ? U[1] : U[2];  // normal discharge
  F[0] = hn;
  if constexpr (DIR == 0) {
    F[1] = flux_normal<EXACT, DIR>(C, U, q, Hloc);
    F[2] = hn * q.v;
  } else {
    F[1] = hn * q.u;
    F[2] = flux_normal<EXACT, DIR>(C, U, q, Hloc);
  }
  F[3] = hn * q.w;
  F[4] = hn * (q.p + C.c2);
}

// |normal velocity| + sqrt(max(g h + p + c^2, 0)), src/physics/sgn_flux2d.h:73-86.
template <bool EXACT, int DIR, class TC>
__device__ __forceinline__ double wave_speed(const TC& C, const double* U,
                                             const Prim<EXACT>& q) {
  const double arg = C.g * U[0] + q.p + C.c2;
  const double ce = EXACT ? sqrt(arg > 0.0 ? arg : 0.0) : fast_sqrt(arg > 0.0 ? arg : 0.0);
  return fabs(DIR == 0 ? q.u : q.v) + ce;
}

// Field v of the directional flux from the per-node quantities: normal discharge hn,
// primitives q and the precomputed normal-momentum component fn (sgn_flux2d.h:89-116).
template <bool EXACT, int DIR, class TC>
__device__ __forceinline__ double flux_field(const TC& C, int v, double hn,
                                             const Prim<EXACT>& q, double fn) {
  switch (v) {
    case 0: return hn;
    case 1: return DIR == 0 ? fn : hn * q.u;
    case 2: return DIR == 0 ? hn * q.v : fn;
    case 3: return hn * q.w;
    default: return hn * (q.p + C.c2);
  }
}

// Face trace of one field along a line of solution points p[0], p[stride], ...:
// sum_k l[k] p[k] accumulated from 0.0 in the reference's order (sgn2d.cpp:141-177), each
// product and sum rounded on its own in both arithmetic modes, so that the trace an
// element forms of itself, the one its neighbour forms of it in the same tile and the
// one the trace pre-pass stores agree bit for bit.
__device__ __forceinline__ double face_trace(const double* l, const double* p, int stride) {
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < NP; ++k) s = __dadd_rn(s, __dmul_rn(l[k], p[k * stride]));
  return s;
}

// Mirror ghost of a face trace across a wall normal to DIR, written 0.0 + v and
// 0.0 + (-v) for the normal discharge (the mirror element's trace in the reference's
// doubled-domain picture).
template <int DIR>
__device__ __forceinline__ void mirror_trace(const double* own, double* ghost) {
#pragma unroll
  for (int v = 0; v < NV; ++v) ghost[v] = __dadd_rn(0.0, own[v]);
  ghost[DIR == 0 ? 1 : 2] = __dadd_rn(0.0, -own[DIR == 0 ? 1 : 2]);
}

// The line computation shared by the row (DIR 0) and column (DIR 1) passes: nodal
// fluxes, both Rusanov face fluxes with central depths, the element's own face fluxes,
// the 5-point differentiation and the correction lift (src/solver/sgn2d.cpp:188-275
// restricted to one line).
//   Un[k]   raw node states along the line, k = 0..4 (low face at k = 0)
//   Hn[k]   nodal still depth
//   nLo/nHi raw node state of the neighbour across the low/high face (or the mirror
//           ghost at a wall)
//   HfLo/HfHi still depth at the two faces
// Results go out through two callbacks: emit_dh(m, dh, q) with the FR-corrected depth
// derivative of node m, then emit(m, v, d, q) with the FR-corrected derivative of flux
// field v at node m (both already divided by J). The flux of each field is rebuilt from
// per-node quantities inside the contraction, which keeps the live set small.
// GAUSS (Gauss-Legendre points): the own traces are interpolated with the rows lL / lR
// of Tb, nLo / nHi are the neighbours' traces, and a wall (mirLo / mirHi) mirrors the own
// trace.
template <bool EXACT, int DIR, bool GAUSS = false, class TC, class TB, class EmitH, class Emit>
__device__ __forceinline__ void line_pass(const TC& C, const TB& Tb, const double (&Un)[NP][NV],
                                          const double (&Hn)[NP], const double* nLo,
                                          const double* nHi, double HfLo, double HfHi,
                                          EmitH&& emit_dh, Emit&& emit, bool mirLo = false,
                                          bool mirHi = false) {
  Prim<EXACT> q[NP];
  double hn[NP], fn[NP];
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    q[k] = Prim<EXACT>(Un[k]);
    hn[k] = DIR == 0 ? Un[k][1] : Un[k][2];
    fn[k] = flux_normal<EXACT, DIR>(C, Un[k], q[k], Hn[k]);
  }
  // face traces: own side t*, neighbour side s*
  double tLo[NV], tHi[NV], sLo[NV], sHi[NV];
  if constexpr (GAUSS) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      tLo[v] = face_trace(Tb.lL, &Un[0][v], NV);
      tHi[v] = face_trace(Tb.lR, &Un[0][v], NV);
    }
    if (mirLo) {
      mirror_trace<DIR>(tLo, sLo);
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) sLo[v] = nLo[v];
    }
    if (mirHi) {
      mirror_trace<DIR>(tHi, sHi);
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) sHi[v] = nHi[v];
    }
  } else {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      tLo[v] = canon<EXACT>(Un[0][v]);
      tHi[v] = canon<EXACT>(Un[NP - 1][v]);
      sLo[v] = canon<EXACT>(nLo[v]);
      sHi[v] = canon<EXACT>(nHi[v]);
    }
  }
  double jLo[NV], jHi[NV];  // common flux minus own face flux
  {
    const Prim<EXACT> qsLo(sLo), qsHi(sHi);
    Prim<EXACT> qtLo, qtHi;
    if constexpr (EXACT || GAUSS) {
      qtLo = Prim<EXACT>(tLo);
      qtHi = Prim<EXACT>(tHi);
    } else {
      qtLo = q[0];
      qtHi = q[NP - 1];
    }
    const double fnLo_t = flux_normal<EXACT, DIR>(C, tLo, qtLo, HfLo);
    const double fnHi_t = flux_normal<EXACT, DIR>(C, tHi, qtHi, HfHi);
    const double fnLo_s = flux_normal<EXACT, DIR>(C, sLo, qsLo, HfLo);
    const double fnHi_s = flux_normal<EXACT, DIR>(C, sHi, qsHi, HfHi);
    const double hnLo_t = tLo[1 + DIR], hnHi_t = tHi[1 + DIR];
    const double hnLo_s = sLo[1 + DIR], hnHi_s = sHi[1 + DIR];
    // Rusanov (sgn_flux2d.h:169-179); the low face has the neighbour on its left
    const double lamLo = fmax(wave_speed<EXACT, DIR>(C, sLo, qsLo), wave_speed<EXACT, DIR>(C, tLo, qtLo));
    const double lamHi = fmax(wave_speed<EXACT, DIR>(C, tHi, qtHi), wave_speed<EXACT, DIR>(C, sHi, qsHi));
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      // own face flux Fd (sgn2d.cpp:229-239) and the neighbour's flux at the face
      const double FdLo = flux_field<EXACT, DIR>(C, v, hnLo_t, qtLo, fnLo_t);
      const double FdHi = flux_field<EXACT, DIR>(C, v, hnHi_t, qtHi, fnHi_t);
      const double FnLo = flux_field<EXACT, DIR>(C, v, hnLo_s, qsLo, fnLo_s);
      const double FnHi = flux_field<EXACT, DIR>(C, v, hnHi_s, qsHi, fnHi_s);
      const double fsLo = 0.5 * (FnLo + FdLo) - 0.5 * lamLo * (tLo[v] - sLo[v]);
      const double fsHi = 0.5 * (FdHi + FnHi) - 0.5 * lamHi * (sHi[v] - tHi[v]);
      jLo[v] = fsLo - FdLo;
      jHi[v] = fsHi - FdHi;
    }
  }
  // FR-corrected depth derivative with the central common depth h* (sgn2d.cpp:265-275)
  {
    const double jhLo = 0.5 * (sLo[0] + tLo[0]) - tLo[0];
    const double jhHi = 0.5 * (tHi[0] + sHi[0]) - tHi[0];
#pragma unroll
    for (int m = 0; m < NP; ++m) {
      double dh;
      if constexpr (EXACT) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) s += Tb.D[m * NP + k] * Un[k][0];
        s += jhLo * Tb.gLp[m] + jhHi * Tb.gRp[m];
        dh = s / (DIR == 0 ? C.Jx : C.Jy);
      } else {
        double s = jhLo * Tb.gLp[m];
        s = fma(jhHi, Tb.gRp[m], s);
#pragma unroll
        for (int k = 0; k < NP; ++k) s = fma(Tb.D[m * NP + k], Un[k][0], s);
        dh = s * (DIR == 0 ? C.iJx : C.iJy);
      }
      emit_dh(m, dh, q[m]);
    }
  }
  // FR-corrected flux divergence, field by field (sgn2d.cpp:248-263)
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double F[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) F[k] = flux_field<EXACT, DIR>(C, v, hn[k], q[k], fn[k]);
#pragma unroll
    for (int m = 0; m < NP; ++m) {
      double d;
      if constexpr (EXACT) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) s += Tb.D[m * NP + k] * F[k];
        const double c = jLo[v] * Tb.gLp[m] + jHi[v] * Tb.gRp[m];
        d = (s + c) / (DIR == 0 ? C.Jx : C.Jy);
      } else {
        // accumulate with the unscaled tables, one rounding for 1/J at the end
        double s = jLo[v] * Tb.gLp[m];
        s = fma(jHi[v], Tb.gRp[m], s);
#pragma unroll
        for (int k = 0; k < NP; ++k) s = fma(Tb.D[m * NP + k], F[k], s);
        d = s * (DIR == 0 ? C.iJx : C.iJy);
      }
      emit(m, v, d, q[m]);
    }
  }
}

// Nodal still-depth gradient at node (a, b) of one element from its nodal depths He:
// the element-local GLL derivative over the Jacobian, dH/dx (DIR 0) or dH/dy (DIR 1), as
// the solver's set-up defines it (src/solver/sgn2d.cpp:54-71). The exact mode repeats the
// set-up's operation order (sum from 0.0, then a division), so it reproduces the
// precomputed arrays bit for bit; reading them would cost 3.2 bytes per DOF.
template <bool EXACT, int DIR, class TC, class TB>
__device__ __forceinline__ double depth_grad(const TC& C, const TB& Tb, const double* He, int a,
                                             int b) {
  const int m = DIR == 0 ? a : b;
  if constexpr (EXACT) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < NP; ++k)
      s += Tb.D[m * NP + k] * He[DIR == 0 ? k + NP * b : a + NP * k];
    return s / (DIR == 0 ? C.Jx : C.Jy);
  } else {
    double s = Tb.D[m * NP] * He[DIR == 0 ? NP * b : a];
#pragma unroll
    for (int k = 1; k < NP; ++k)
      s = fma(Tb.D[m * NP + k], He[DIR == 0 ? k + NP * b : a + NP * k], s);
    return s * (DIR == 0 ? C.iJx : C.iJy);
  }
}

// Mirror ghost across a wall normal to DIR: the normal discharge changes sign.
template <int DIR>
__device__ __forceinline__ void mirror(const double* own, double* ghost) {
#pragma unroll
  for (int v = 0; v < NV; ++v) ghost[v] = own[v];
  ghost[DIR == 0 ? 1 : 2] = -own[DIR == 0 ? 1 : 2];
}


// One tile of the fused right-hand side / stage kernel: tile (bx, by) of the mesh whose
// constants are C, error partial slot blk. Shared by the single-instance kernel and the
// batched kernel. Returns early (uniformly over the CTA) when the instance's run is done.
// FULL: the mesh is a whole number of tiles, so every tile is full and the per-item range
// checks and their branches are compiled out (8 % off the end-point stage at 2048 x 1024).
// TMA: the own-node tiles (state or stage derivatives, nodal depth) arrive by
// tensor-memory-accelerator copies described by M (full tiles of the single-instance
// kernel only).
template <int MODE, bool EXACT, int TX_, int TY_, class TC, class TB, class TA, bool FRIC = false,
          bool GHOST = false, bool GAUSS = false, bool FULL = false, bool TMA = false>
__device__ __forceinline__ void fused_tile(const TC& C, const TB& Tb, const TA& A,
                                           int bx, int by, long long blk,
                                           typename Tile<TX_, TY_, EXACT>::Smem& S,
                                           const TileMaps* M = nullptr) {
  static_assert(!TMA || (FULL && !GAUSS && TX_ == 8 && TY_ == 4),
                "tile loads by the tensor-memory accelerator: full 8x4 tiles");
  using T = Tile<TX_, TY_, EXACT>;
  constexpr int TX = T::TX, TY = T::TY, NHALO = T::NHALO, RUN = T::RUN;
  constexpr int NHIT = T::NHIT, NFACE = T::NFACE, NFIT = T::NFIT;

  // ---- controller state (stage modes only) ---------------------------------
  int cur = 0;
  double atol = 0.0, rtol = 0.0;
  StageIn I;
  I.in = A.in;
  I.dt = 0.0;
  I.acoef = 0.0;
  if constexpr (MODE != MODE_RHS) {
    if (A.ctrl->done) return;  // uniform across the grid
    cur = A.ctrl->cur;
    I.dt = A.ctrl->dt;
    I.acoef = A.coef * I.dt;  // 0.5 * dt or 0.75 * dt as in rk.cpp:100-103
    atol = A.ctrl->atol;
    rtol = A.ctrl->rtol;
  }
  I.u = A.U[cur];
  I.k = A.kin_k2 ? A.K2 : A.K1[cur];
  I.k1 = A.K1[cur];
  I.k2 = A.K2;
  I.k3 = A.K3;

  // the thread index read through an opaque move: in the persistent batched kernel this
  // keeps the compiler from hoisting the per-thread item and halo descriptors out of the
  // tile loop (they would stay live, in registers, across every tile's passes)
  int tid;
  asm volatile("mov.u32 %0, %%tid.x;" : "=r"(tid));
  const int warp = tid >> 5, lane = tid & 31;
  const int Nx = C.Nx, Ny = C.Ny;
  const long long Nd = C.Nd;
  const int ex0 = bx * TX, ey0 = by * TY;
  const int TXv = FULL ? TX : min(TX, Nx - ex0), TYv = FULL ? TY : min(TY, Ny - ey0);
  // the element columns and rows across the tile's edges, wrapped periodically (a compare
  // instead of an integer remainder by the mesh size)
  const int exL = ex0 == 0 ? Nx - 1 : ex0 - 1, exR = ex0 + TXv == Nx ? 0 : ex0 + TXv;
  const int eyB = ey0 == 0 ? Ny - 1 : ey0 - 1, eyT = ey0 + TYv == Ny ? 0 : ey0 + TYv;
  // slab edges: the trace nodes across come from the neighbours' ghost arrays
  bool ghostL = false, ghostR = false;
  if constexpr (GHOST) {
    ghostL = C.ghostL != nullptr && ex0 == 0;
    ghostR = C.ghostR != nullptr && ex0 + TXv == Nx;
  }
  const bool wallL = C.bcx && ex0 == 0 && !ghostL, wallR = C.bcx && ex0 + TXv == Nx && !ghostR;
  const bool wallB = C.bcy && ey0 == 0, wallT = C.bcy && ey0 + TYv == Ny;

  // ---- own-node item map: NIT items per thread, shared by every array -------
  // item u of a thread is double k of tile row iy: global (e_row*25 + k), shared
  // iy*RUN + k (the [TE][NPP] layout of one field). The stage modes on full tiles keep a
  // thread's items in one tile row, NTHR / TY doubles apart (one base address and
  // immediate offsets: the end-point stage 1.3 % faster); the rhs-only mode and partial
  // tiles (the batched kernels) take q = tid + NTHR*u in tile-row order (1 % and 0.3 %
  // faster there). Recomputed after the passes rather than kept live through them.
  int gof[NIT];  // node offset within one field (Nd <= 2^31 by the mesh-size limit)
  int sof[NIT];
  bool okk[NIT];
  auto item_map = [&]() {
#pragma unroll
    for (int u = 0; u < NIT; ++u) {
      constexpr int PER_ROW = NTHR / TY;
      static_assert(NTHR % TY == 0 && RUN == NIT * PER_ROW, "items split evenly over the rows");
      int iy, k;
      if constexpr (MODE != MODE_RHS && FULL) {
        iy = tid / PER_ROW;
        k = tid - iy * PER_ROW + PER_ROW * u;
      } else {
        const int q = tid + NTHR * u;
        iy = q / RUN;
        k = q - iy * RUN;
      }
      okk[u] = FULL || (iy < TYv && k < TXv * NPP);
      gof[u] = (int)(((long long)ex0 + (long long)Nx * (ey0 + iy)) * NPP + k);
      sof[u] = iy * RUN + k;
    }
  };
  item_map();

  // ---- load phase --------------------------------------------------------------
  // TMA: one thread issues the tile's copies (rhs: the input; stage: u and k; end point: k1
  // and k2; each [5][4][200] doubles; and the [4][200] nodal depths) on an mbarrier that
  // aliases the (not yet used) reduction slots.
  const unsigned mbar = smem_addr(&S.red[0][0]);
  if constexpr (TMA) {
    if (tid == 0) mbar_init(mbar);
    __syncthreads();
    if (tid == 0) {
      const int x = ex0 * NPP;  // 16-byte aligned: 1600 bytes per tile column
      constexpr int narr = MODE == MODE_RHS ? 1 : 2;
      mbar_expect_tx(mbar, (unsigned)((narr * NV + 1) * TE * NPP * sizeof(double)));
      const CUtensorMap* mu = MODE == MODE_RHS ? &M->In : (MODE == MODE_STAGE ? &M->U[cur] : &M->K1[cur]);
      tma_load_3d(smem_addr(&S.U[0][0][0]), mu, x, ey0, 0, mbar);
      if constexpr (MODE != MODE_RHS) {
        const CUtensorMap* mg = MODE == MODE_STAGE ? (A.kin_k2 ? &M->K2 : &M->K1[cur]) : &M->K2;
        tma_load_3d(smem_addr(&S.G[0][0][0]), mg, x, ey0, 0, mbar);
      }
      tma_load_2d(smem_addr(&S.H[0][0]), &M->H, x, ey0, mbar);
    }
  }
  {
    // Otherwise the statics, and the state of the rhs and stage modes, arrive by
    // per-thread asynchronous copies straight into shared memory: a tile's loads are all in
    // flight at once without holding registers. The stage mode stages k in the (still
    // unused) G area and forms u + (c dt) k in shared memory once the copies have landed.
    if constexpr (!TMA) {
#pragma unroll
      for (int u = 0; u < NIT; ++u)
        if (okk[u]) {
          if (SGNB_INB(gof[u], Nd) && SGNB_INB(sof[u], TE * NPP)) cp_async8(&(&S.H[0][0])[sof[u]], C.Hnod + gof[u]);
        }
    }
    if constexpr (TMA) {
      // the tile copies above
    } else if constexpr (MODE == MODE_RHS || MODE == MODE_STAGE) {
      const double* __restrict__ src = MODE == MODE_RHS ? I.in : I.u;
#pragma unroll
      for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int u = 0; u < NIT; ++u)
          if (okk[u] && SGNB_INB(gof[u], Nd) && SGNB_INB(sof[u], TE * NPP)) {
            cp_async8(&(&S.U[v][0][0])[sof[u]], (src + (long long)v * Nd) + gof[u]);
            if constexpr (MODE == MODE_STAGE)
              cp_async8(&(&S.G[v][0][0])[sof[u]], (I.k + (long long)v * Nd) + gof[u]);
          }
    } else {
      // end-point stage, round 1: k1 and k2 into the U and G areas
#pragma unroll
      for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int u = 0; u < NIT; ++u)
          if (okk[u] && SGNB_INB(gof[u], Nd) && SGNB_INB(sof[u], TE * NPP)) {
            cp_async8(&(&S.U[v][0][0])[sof[u]], (I.k1 + (long long)v * Nd) + gof[u]);
            cp_async8(&(&S.G[v][0][0])[sof[u]], (I.k2 + (long long)v * Nd) + gof[u]);
          }
    }
    // halo items: descriptors, then loads
    double hv[NHIT];
    int hq[NHIT];
    int hs[NHIT];  // source: 0 the state, 1 the left ghost, 2 the right ghost
    long long hg[NHIT];
#pragma unroll
    for (int u = 0; u < NHIT; ++u) {
      const int q = tid + NTHR * u;
      const int t = q % NP, r = q / NP;
      const int slot = r % NHALO, v = r / NHALO;
      bool ok = q < NV * NHALO * NP;
      long long e = 0;
      int node = 0;
      hs[u] = 0;
      if (slot < TY) {
        if (GHOST && ghostL) hs[u] = 1;
        ok = ok && slot < TYv && !wallL;
        e = (long long)(exL) + (long long)Nx * (ey0 + slot);
        node = (NP - 1) + NP * t;
      } else if (slot < 2 * TY) {
        if (GHOST && ghostR) hs[u] = 2;
        ok = ok && slot - TY < TYv && !wallR;
        e = (long long)(exR) + (long long)Nx * (ey0 + slot - TY);
        node = NP * t;
      } else if (slot < 2 * TY + TX) {
        ok = ok && slot - 2 * TY < TXv && !wallB;
        e = (long long)(ex0 + slot - 2 * TY) + (long long)Nx * (eyB);
        node = t + NP * (NP - 1);
      } else {
        ok = ok && slot - 2 * TY - TX < TXv && !wallT;
        e = (long long)(ex0 + slot - 2 * TY - TX) + (long long)Nx * (eyT);
        node = t;
      }
      hq[u] = ok ? q : -1;
      hg[u] = (GHOST && hs[u]) ? (long long)v * Ny * NP + (long long)(ey0 + (slot < TY ? slot : slot - TY)) * NP + t
                               : (long long)v * Nd + e * NPP + node;
      if constexpr (GAUSS) {
        // the neighbour's trace on the shared face: the left neighbour's right face (1),
        // the right neighbour's left face (0), the bottom one's top face (3), the top
        // one's bottom face (2)
        const int f = slot < TY ? 1 : (slot < 2 * TY ? 0 : (slot < 2 * TY + TX ? 3 : 2));
        hg[u] = ((long long)(f * NV + v) * (Nd / NPP) + e) * NP + t;
      }
    }
#pragma unroll
    for (int u = 0; u < NHIT; ++u)
      if (hq[u] >= 0) {
        if constexpr (GAUSS)
          hv[u] = SGNB_INB(hg[u], 4 * Nd) ? C.tr[hg[u]] : 0.0;
        else if constexpr (GHOST)
          hv[u] = hs[u] == 0 ? (SGNB_INB(hg[u], NV * Nd) ? stage_value<MODE>(I, hg[u]) : 0.0)
                             : (SGNB_INB(hg[u], (long long)NV * Ny * NP) ? (hs[u] == 1 ? C.ghostL : C.ghostR)[hg[u]] : 0.0);
        else
          hv[u] = SGNB_INB(hg[u], NV * Nd) ? stage_value<MODE>(I, hg[u]) : 0.0;
      }
    // face depths
    double fv[NFIT];
    int fq[NFIT];
#pragma unroll
    for (int u = 0; u < NFIT; ++u) {
      const int q = tid + NTHR * u;
      fq[u] = -1;
      if (q < 2 * TE * NP) {
        const int t = q % NP, i = (q / NP) % TE, s = q / (NP * TE);
        const int ix = i % TX, iy = i / TX;
        if (ix < TXv && iy < TYv) {
          const long long e = (long long)(ex0 + ix) + (long long)Nx * (ey0 + iy);
          fv[u] = SGNB_INB(e * NP + t, Nd / NP) ? (s == 0 ? C.HfX : C.HfY)[e * NP + t] : 0.0;
          fq[u] = q;
        }
      } else if (q < NFACE) {
        const int r = q - 2 * TE * NP;
        const int t = r % NP, slot = r / NP;
        if (slot < TY) {
          if (slot < TYv) {
            const int ey = ey0 + slot;
#ifdef SGNB_CHECKED
            const long long fe = (long long)ey * NP + t;
            const long long fx = ((long long)(exR) + (long long)Nx * ey) * NP + t;
            fv[u] = (wallR || ghostR) ? (SGNB_INB(fe, (long long)Ny * NP) ? C.HfXEnd[fe] : 0.0)
                                      : (SGNB_INB(fx, Nd / NP) ? C.HfX[fx] : 0.0);
#else
            fv[u] = (wallR || ghostR) ? C.HfXEnd[(long long)ey * NP + t]
                          : C.HfX[((long long)(exR) + (long long)Nx * ey) * NP + t];
#endif
            fq[u] = q;
          }
        } else if (slot - TY < TXv) {
          const int ex = ex0 + slot - TY;
#ifdef SGNB_CHECKED
          const long long fe = (long long)ex * NP + t;
          const long long fy = ((long long)ex + (long long)Nx * (eyT)) * NP + t;
          fv[u] = wallT ? (SGNB_INB(fe, (long long)Nx * NP) ? C.HfYEnd[fe] : 0.0)
                        : (SGNB_INB(fy, Nd / NP) ? C.HfY[fy] : 0.0);
#else
          fv[u] = wallT ? C.HfYEnd[(long long)ex * NP + t]
                        : C.HfY[((long long)ex + (long long)Nx * (eyT)) * NP + t];
#endif
          fq[u] = q;
        }
      }
    }
#pragma unroll
    for (int u = 0; u < NHIT; ++u)
      if (hq[u] >= 0 && SGNB_INB(hq[u], NV * NHALO * NP)) S.halo[hq[u]] = hv[u];
#pragma unroll
    for (int u = 0; u < NFIT; ++u)
      if (fq[u] >= 0 && SGNB_INB(fq[u], NFACE)) S.Hf[fq[u]] = fv[u];
    cp_async_wait_all();
    if constexpr (TMA) {
      bool landed = false;
      for (int it = 0; it < kTmaTries && !landed; ++it) landed = mbar_try_wait(mbar, 0);
      if (!landed) {
        // the copies did not complete: this thread's items become NaN, so the launch's
        // results are non-finite and the controller ends the run with that error
        const double nan = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
        for (int v = 0; v < NV; ++v)
#pragma unroll
          for (int u = 0; u < NIT; ++u) {
            (&S.U[v][0][0])[sof[u]] = nan;
            (&S.G[v][0][0])[sof[u]] = nan;
          }
      }
    }
    if constexpr (MODE == MODE_STAGE) {
      // u + (c dt) k for this thread's own items (rk.cpp:100-103), in shared memory
#pragma unroll
      for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int u = 0; u < NIT; ++u)
          if (okk[u]) {
            double& y = (&S.U[v][0][0])[sof[u]];
            y = stage_axpy(y, I.acoef, (&S.G[v][0][0])[sof[u]]);
          }
    } else if constexpr (MODE == MODE_FSAL) {
      // round 2: 2/9 k1 + 1/3 k2 in place, k3 into the G area while u comes through
      // registers, then uNew = u + dt ((2/9 k1 + 1/3 k2) + 4/9 k3) (rk.cpp:106-108),
      // written to shared memory and out as the candidate state
      // every u load of the tile is issued first, so that they are in flight together
      // with the k3 copies (one memory round trip for the round, not one per field)
      double ux[NV][NIT];
#pragma unroll
      for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int u = 0; u < NIT; ++u)
          if (okk[u] && SGNB_INB(gof[u], Nd)) ux[v][u] = (I.u + (long long)v * Nd)[gof[u]];
#pragma unroll
      for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int u = 0; u < NIT; ++u)
          if (okk[u]) {
            double& y = (&S.U[v][0][0])[sof[u]];
            y = fsal_part(y, (&S.G[v][0][0])[sof[u]]);
            if (SGNB_INB(gof[u], Nd) && SGNB_INB(sof[u], TE * NPP))
              cp_async8(&(&S.G[v][0][0])[sof[u]], (I.k3 + (long long)v * Nd) + gof[u]);
          }
      double* __restrict__ unew = A.U[cur ^ 1];  // stored evict-first (see the copy-out)
      cp_async_wait_all();
#pragma unroll
      for (int v = 0; v < NV; ++v) {
#pragma unroll
        for (int u = 0; u < NIT; ++u)
          if (okk[u]) {
            double& y = (&S.U[v][0][0])[sof[u]];
            const double un = fsal_finish(ux[v][u], y, (&S.G[v][0][0])[sof[u]], I.dt);
            y = un;
            if (SGNB_INB(gof[u], Nd)) __stcs(&(unew + (long long)v * Nd)[gof[u]], un);
          }
      }
    }
  }
  __syncthreads();
  if constexpr (TMA) {
    if (tid == 0) mbar_inval(mbar);  // its slots serve the error reduction later
  }

  const int i = lane;  // tile element of this lane
  const int ix = i % TX, iy = i / TX;
  const bool valid = FULL || (ix < TXv && iy < TYv);
  const int j = warp;  // GLL line index of this warp

  // ---- column pass: y-line a = j ---------------------------------------------
  if (valid) {
    double Un[NP][NV], Hn[NP];
#pragma unroll
    for (int b = 0; b < NP; ++b) {
#pragma unroll
      for (int v = 0; v < NV; ++v) Un[b][v] = S.U[v][i][j + NP * b];
      Hn[b] = S.H[i][j + NP * b];
    }
    double nLo[NV], nHi[NV];
    if (iy > 0) {
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        if constexpr (GAUSS) nLo[v] = face_trace(Tb.lR, &S.U[v][i - TX][j], NP);
        else nLo[v] = S.U[v][i - TX][j + NP * (NP - 1)];
      }
    } else if (wallB) {
      if constexpr (!GAUSS) mirror<1>(Un[0], nLo);
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) nLo[v] = T::halo_at(S, v, 2 * TY + ix, j);
    }
    if (iy + 1 < TYv) {
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        if constexpr (GAUSS) nHi[v] = face_trace(Tb.lL, &S.U[v][i + TX][j], NP);
        else nHi[v] = S.U[v][i + TX][j];
      }
    } else if (wallT) {
      if constexpr (!GAUSS) mirror<1>(Un[NP - 1], nHi);
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) nHi[v] = T::halo_at(S, v, 2 * TY + TX + ix, j);
    }
    const double HfLo = T::hf_y(S, i, j);
    const double HfHi = (iy + 1 < TYv) ? T::hf_y(S, i + TX, j) : T::hf_yt(S, ix, j);
    double by[NP];  // ncpY, -c^2 v h_y (sgn_flux2d.h:156-161)
    line_pass<EXACT, 1, GAUSS>(
        C, Tb, Un, Hn, nLo, nHi, HfLo, HfHi,
        [&](int b, double dh, const Prim<EXACT>& q) {
          if constexpr (EXACT) S.G[NV][i][j + NP * b] = C.mc2 * q.v * dh;
          else by[b] = C.mc2 * q.v * dh;
        },
        [&](int b, int v, double d, const Prim<EXACT>&) {
          if constexpr (EXACT) S.G[v][i][j + NP * b] = d;
          else S.G[v][i][j + NP * b] = v == NV - 1 ? d + by[b] : d;
        },
        iy == 0 && wallB, iy + 1 >= TYv && wallT);
  }
  __syncthreads();

  // ---- row pass: x-line b = j, then assembly ---------------------------------
  // dU of node (a, j) replaces that node's column-pass results in S.G; only this
  // thread touches those slots in this phase.
  if (valid) {
    double Un[NP][NV], Hn[NP];
#pragma unroll
    for (int a = 0; a < NP; ++a) {
#pragma unroll
      for (int v = 0; v < NV; ++v) Un[a][v] = S.U[v][i][a + NP * j];
      Hn[a] = S.H[i][a + NP * j];
    }
    double nLo[NV], nHi[NV];
    if (ix > 0) {
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        if constexpr (GAUSS) nLo[v] = face_trace(Tb.lR, &S.U[v][i - 1][NP * j], 1);
        else nLo[v] = S.U[v][i - 1][(NP - 1) + NP * j];
      }
    } else if (wallL) {
      if constexpr (!GAUSS) mirror<0>(Un[0], nLo);
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) nLo[v] = T::halo_at(S, v, iy, j);
    }
    if (ix + 1 < TXv) {
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        if constexpr (GAUSS) nHi[v] = face_trace(Tb.lL, &S.U[v][i + 1][NP * j], 1);
        else nHi[v] = S.U[v][i + 1][NP * j];
      }
    } else if (wallR) {
      if constexpr (!GAUSS) mirror<0>(Un[NP - 1], nHi);
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) nHi[v] = T::halo_at(S, v, TY + iy, j);
    }
    const double HfLo = T::hf_x(S, i, j);
    const double HfHi = (ix + 1 < TXv) ? T::hf_x(S, i + 1, j) : T::hf_xr(S, iy, j);
    double dhx[NP];
    line_pass<EXACT, 0, GAUSS>(
        C, Tb, Un, Hn, nLo, nHi, HfLo, HfHi,
        [&](int a, double dh, const Prim<EXACT>&) { dhx[a] = dh; },
        [&](int a, int v, double d, const Prim<EXACT>& q) {
          const int loc = a + NP * j;
          const double g = S.G[v][i][loc];
          double res;
          // dU = -dF - dG - Bx - By + S (sgn2d.cpp:285-287) with the source of
          // sgn_flux2d.h:122-134 (Manning off); Bx, By vanish except in hp
          if (v == 0) {
            res = EXACT ? (-d - g) + 0.0 : -(d + g);
          } else if (v == 3) {
            const double S3 = C.gamma * q.p;
            res = EXACT ? (-d - g) + S3 : S3 - (d + g);
          } else if (v == 1 || v == 2) {
            const double bath = C.g * (Un[a][0] - Hn[a]) + C.gamma * q.p;
            double Sv = bath * (v == 1 ? depth_grad<EXACT, 0>(C, Tb, S.H[i], a, j)
                                       : depth_grad<EXACT, 1>(C, Tb, S.H[i], a, j));
            if constexpr (FRIC) {
              // Manning friction along the velocity, n^2 g |vel| vel / h^(1/3)
              // (sgn_flux2d.h:135-142)
              const double vmag = sqrt(q.u * q.u + q.v * q.v);
              const double cf = C.n2g * vmag / cbrt(Un[a][0]);
              Sv = Sv - cf * (v == 1 ? q.u : q.v);
            }
            res = EXACT ? (-d - g) + Sv : Sv - (d + g);
          } else {
            const double Hxl = depth_grad<EXACT, 0>(C, Tb, S.H[i], a, j);
            const double Hyl = depth_grad<EXACT, 1>(C, Tb, S.H[i], a, j);
            const double S4 = C.m2c2 * (q.w + q.u * Hxl + q.v * Hyl);
            const double Bx = C.mc2 * q.u * dhx[a];  // ncpX (sgn_flux2d.h:150-155)
            if constexpr (EXACT) {
              const double By = S.G[NV][i][loc];
              res = (((-d - g) - Bx) - By) + S4;
            } else {
              res = S4 - (d + g) - Bx;  // g holds dG + By
            }
          }
          S.G[v][i][loc] = res;
        },
        ix == 0 && wallL, ix + 1 >= TXv && wallR);
  }
  __syncthreads();

  // ---- copy-out (and the embedded error of the FSAL stage) ------------------
  double esum = 0.0, emax = 0.0;
  int enan = 0;
  item_map();
  {
    // reload the controller values and stage pointers instead of keeping them live
    // through the passes
    if constexpr (MODE == MODE_FSAL) {
      const CtrlReload rc = ctrl_reload(A.ctrl);
      cur = rc.cur;
      I.dt = rc.dt;
      atol = rc.atol;
      rtol = rc.rtol;
      I.u = A.U[cur];
      I.k1 = A.K1[cur];
      I.k2 = A.K2;
      I.k3 = A.K3;
    }
    // L2 use: every result (dU, k2, k3, uNew, k4) is next read by another launch, after
    // gigabytes of other traffic, so it is stored with the streaming (evict-first) hint;
    // the end-point stage's second reads of u, k1, k2, k3 below are their last use in the
    // launch and are loaded the same way. The lines the launch still reads (its inputs,
    // which the epilogue and the neighbour tiles' halos read again) keep L2 to themselves:
    // 5.01 -> 4.73 ms for the end-point stage at 2048 x 1024.
    double* __restrict__ outp;
    if constexpr (MODE == MODE_RHS || MODE == MODE_STAGE) outp = A.out;
    else outp = A.K1[cur ^ 1];
    if constexpr (MODE != MODE_FSAL) {
#pragma unroll 1
      for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int u = 0; u < NIT; ++u)
          if (okk[u] && SGNB_INB(gof[u], Nd)) __stcs(&(outp + (long long)v * Nd)[gof[u]], (&S.G[v][0][0])[sof[u]]);
    } else {
      // One field at a time, with the next field's four arrays prefetched while the
      // current field's error is formed: hoisting every field's loads at once would
      // overflow the register budget.
      double uu[NIT], c1[NIT], c2[NIT], c3[NIT];
      double nu[NIT], n1[NIT], n2[NIT], n3[NIT];
#pragma unroll
      for (int u = 0; u < NIT; ++u)
        if (okk[u]) {
          const int g = gof[u];
          if (SGNB_INB(g, Nd)) { uu[u] = __ldcs(&I.u[g]); c1[u] = __ldcs(&I.k1[g]); c2[u] = __ldcs(&I.k2[g]); c3[u] = __ldcs(&I.k3[g]); }
        }
#pragma unroll 1
      for (int v = 0; v < NV; ++v) {
        if (v + 1 < NV) {
#pragma unroll
          for (int u = 0; u < NIT; ++u)
            if (okk[u]) {
              const long long o = (long long)(v + 1) * Nd;  // per-field base, 32-bit item offset
              const int g = gof[u];
              if (SGNB_INB(o + g, NV * Nd)) { nu[u] = __ldcs(&(I.u + o)[g]); n1[u] = __ldcs(&(I.k1 + o)[g]); n2[u] = __ldcs(&(I.k2 + o)[g]); n3[u] = __ldcs(&(I.k3 + o)[g]); }
            }
        }
#pragma unroll
        for (int u = 0; u < NIT; ++u)
          if (okk[u]) {
            const double k4 = (&S.G[v][0][0])[sof[u]];
            if (SGNB_INB(gof[u], Nd)) __stcs(&(outp + (long long)v * Nd)[gof[u]], k4);
            // scaled embedded error, src/solver/rk.cpp:118-128; the candidate uNew is
            // still in the tile (the passes only read S.U)
            const double dt = I.dt;
            const double un = (&S.U[v][0][0])[sof[u]];
            const double uEmb = uu[u] + dt * (7.0 / 24.0 * c1[u] + 0.25 * c2[u] + 1.0 / 3.0 * c3[u] +
                                              0.125 * k4);
            const double e = un - uEmb;
            const double au = fabs(uu[u]), an = fabs(un);
            const double sc = atol + rtol * (au < an ? an : au);
            double rr;
            if constexpr (EXACT) {
              rr = e / sc;
            } else {
              // the fast mode's reciprocal (a few ulp) where sc is a normal number
              rr = sc >= 2.2250738585072014e-308 ? e * fast_rcp(sc) : e / sc;
            }
            esum += rr * rr;
            const double ar = fabs(rr);
            emax = emax < ar ? ar : emax;
            enan |= (rr != rr);
          }
#pragma unroll
        for (int u = 0; u < NIT; ++u) {
          uu[u] = nu[u]; c1[u] = n1[u]; c2[u] = n2[u]; c3[u] = n3[u];
        }
      }
    }
  }
  if constexpr (GHOST && MODE == MODE_STAGE) {
    // Fused edge exchange: the slab-edge tiles form the next stage's input at their edge
    // nodes (a = 0 of the first column, a = 4 of the last) from this launch's result and
    // store it straight into the neighbours' ghost arrays, [field][row][node], while the
    // other tiles still compute. After stage 2 (k1 added) that is u + 3/4 dt k2, the next
    // launch's own stage input; after stage 3 the end-point candidate. Both with the
    // explicitly rounded combinations of the stage inputs, so the neighbour sees the bits
    // this slab's own next launch forms.
    const bool outLo = C.edgeL != nullptr && ex0 == 0, outHi = C.edgeR != nullptr && ex0 + TXv == Nx;
    if (outLo || outHi) {
      const CtrlReload rc = ctrl_reload(A.ctrl);
      const int cr = rc.cur;
      const double dt = rc.dt;
      const double* __restrict__ u0 = A.U[cr];
      const double* __restrict__ k1 = A.K1[cr];
      const double* __restrict__ k2 = A.K2;
      const int per = NV * TYv * NP;
      for (int q = tid; q < 2 * per; q += NTHR) {
        const int side = q / per;
        if (side == 0 ? !outLo : !outHi) continue;
        const int r = q - side * per;
        const int t = r % NP, iy = (r / NP) % TYv, v = r / (NP * TYv);
        const int ixe = side == 0 ? 0 : TXv - 1;
        const int node = (side == 0 ? 0 : NP - 1) + NP * t;
        const long long g = (long long)v * Nd + ((long long)(ex0 + ixe) + (long long)Nx * (ey0 + iy)) * NPP + node;
        const double kout = S.G[v][TX * iy + ixe][node];
        const long long ge = (long long)v * Ny * NP + (long long)(ey0 + iy) * NP + t;
        if (!SGNB_INB(g, NV * Nd) || !SGNB_INB(ge, (long long)NV * Ny * NP)) continue;
        const double val = A.kin_k2 == 0 ? stage_axpy(u0[g], 0.75 * dt, kout)
                                          : fsal_finish(u0[g], fsal_part(k1[g], k2[g]), kout, dt);
        (side == 0 ? C.edgeL : C.edgeR)[ge] = val;
      }
    }
  }
  if constexpr (MODE == MODE_FSAL) {
    // deterministic block reduction: fixed shuffle tree, then warps in order
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      esum += __shfl_down_sync(0xffffffffu, esum, off);
      const double om = __shfl_down_sync(0xffffffffu, emax, off);
      emax = emax < om ? om : emax;
      enan |= __shfl_down_sync(0xffffffffu, enan, off);
    }
    if (lane == 0) {
      S.red[warp][0] = esum;
      S.red[warp][1] = emax;
      S.red[warp][2] = (double)enan;
    }
    __syncthreads();
    if (tid == 0) {
      double s = 0.0, m = 0.0, n = 0.0;
      for (int w = 0; w < NWARP; ++w) {
        s += S.red[w][0];
        m = m < S.red[w][1] ? S.red[w][1] : m;
        n += S.red[w][2];
      }
      A.partials[3 * blk + 0] = s;
      A.partials[3 * blk + 1] = m;
      A.partials[3 * blk + 2] = n;
    }
  }
}


// FRIC: Manning friction compiled in (instantiated only for contexts that use it, so the
// frictionless kernels carry none of its code).
// GHOST: slab edges compiled in (only contexts with ghost arrays launch these variants).
// GAUSS: Gauss-Legendre points (after k_traces of the same stage).
// FULL: Nx a multiple of 8 and Ny of 4 (every tile full).
template <int MODE, bool EXACT, bool FRIC = false, bool GHOST = false, bool GAUSS = false,
          bool FULL = false>
__global__ void __launch_bounds__(NTHR, EXACT ? 2 : SGNB_FAST_MIN_CTAS) k_fused(const RhsConsts C, const StageArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  using T = Tile<8, 4, EXACT>;
  typename T::Smem& S = *reinterpret_cast<typename T::Smem*>(smem_raw);
  fused_tile<MODE, EXACT, 8, 4, RhsConsts, RhsConsts, StageArgs, FRIC, GHOST, GAUSS, FULL>(C, C, A, blockIdx.x, blockIdx.y,
                                (long long)blockIdx.y * gridDim.x + blockIdx.x, S);
}

// A mesh of whole tiles, with the own-node tiles loaded by the tensor-memory accelerator
// from the buffers that M describes. GHOST: slab edges compiled in (x-slab contexts).
template <int MODE, bool EXACT, bool GHOST = false>
__global__ void __launch_bounds__(NTHR, EXACT ? 2 : SGNB_FAST_MIN_CTAS)
    k_fused_tma(const RhsConsts C, const StageArgs A, const __grid_constant__ TileMaps M) {
  extern __shared__ __align__(128) unsigned char smem_tiles[];  // the copies' destinations
  using T = Tile<8, 4, EXACT>;
  typename T::Smem& S = *reinterpret_cast<typename T::Smem*>(smem_tiles);
  fused_tile<MODE, EXACT, 8, 4, RhsConsts, RhsConsts, StageArgs, false, GHOST, false, true, true>(
      C, C, A, blockIdx.x, blockIdx.y, (long long)blockIdx.y * gridDim.x + blockIdx.x, S, &M);
}

// Face traces of every element for Gauss-Legendre points (sgn2d.cpp:141-177), of the
// stage input the fused kernel of the same MODE reads: one thread per (direction,
// element, transverse node), five fields, both faces. Writes C.tr. The traces are
// explicitly rounded, so both arithmetic modes (EXACT) form the same bits.
template <int MODE, bool EXACT>
__global__ void __launch_bounds__(256) k_traces(const RhsConsts C, const StageArgs A) {
  const long long ne = (long long)C.Nx * C.Ny;
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 2 * ne * NP) return;
  StageIn I;
  I.in = A.in;
  I.dt = 0.0;
  I.acoef = 0.0;
  int cur = 0;
  if constexpr (MODE != MODE_RHS) {
    if (A.ctrl->done) return;
    cur = A.ctrl->cur;
    I.dt = A.ctrl->dt;
    I.acoef = A.coef * I.dt;
  }
  I.u = A.U[cur];
  I.k = A.kin_k2 ? A.K2 : A.K1[cur];
  I.k1 = A.K1[cur];
  I.k2 = A.K2;
  I.k3 = A.K3;
  const int dir = (int)(q / (ne * NP));
  const long long r = q - dir * ne * NP;
  const long long e = r / NP;
  const int t = (int)(r % NP);
  const int fl = dir == 0 ? 0 : 2;  // left / bottom face; the right / top one is fl + 1
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double line[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k)
      line[k] = stage_value<MODE>(I, (long long)v * C.Nd + e * NPP + (dir == 0 ? k + NP * t : t + NP * k));
    const long long lo = ((long long)(fl * NV + v) * ne + e) * NP + t;
    const long long hi = ((long long)((fl + 1) * NV + v) * ne + e) * NP + t;
    if (SGNB_INB(lo, 100 * ne)) C.tr[lo] = face_trace(C.lL, line, 1);
    if (SGNB_INB(hi, 100 * ne)) C.tr[hi] = face_trace(C.lR, line, 1);
  }
}

// Batched form: one launch per stage walks the tiles of many independent instances
// (the work list tile_inst / tile_start), each with its own constants, buffers and
// controller. The instance's constants and buffer pointers are copied into shared
// memory once per tile. PERSIST: a fixed grid of CTAs loops over the work list;
// otherwise one CTA per tile (no loop: the compiler then keeps nothing live from one tile
// to the next, which the loop costs in spilled registers).
template <int MODE, bool EXACT, int TX_, int TY_>
__device__ __forceinline__ void batch_tile(const BatchArgs& B, long long t,
                                           typename Tile<TX_, TY_, EXACT>::Smem& S, RhsConsts& Cs,
                                           StageArgs& As) {
  const int inst = B.tile_inst[t];
  const long long lt = t - B.tile_start[inst];
  __syncthreads();  // the previous tile is done with Cs / As
  {
    // both blocks' loads in flight before the first store (one round trip per tile)
    block_copy2<(int)(sizeof(RhsConsts) / 4), (int)(sizeof(StageArgs) / 4), NTHR>(
        reinterpret_cast<unsigned*>(&Cs), reinterpret_cast<const unsigned*>(B.consts + inst),
        reinterpret_cast<unsigned*>(&As), reinterpret_cast<const unsigned*>(B.args + inst));
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    As.kin_k2 = B.kin_k2;
    As.coef = B.coef;
    if (MODE == MODE_STAGE) As.out = B.kin_k2 ? As.K3 : As.K2;
  }
  __syncthreads();
  const int ntx = (Cs.Nx + TX_ - 1) / TX_;
  // volatile views: per-instance values are re-read from shared memory at each use
  // rather than held in registers through the passes
  fused_tile<MODE, EXACT, TX_, TY_>(static_cast<const volatile RhsConsts&>(Cs), B.tables,
                                    static_cast<const volatile StageArgs&>(As),
                                    (int)(lt % ntx), (int)(lt / ntx), lt, S);
}

template <int MODE, bool EXACT, int TX_, int TY_, bool PERSIST>
__global__ void __launch_bounds__(NTHR, 2) k_fused_batch(const BatchArgs B) {
  // FR tables come from the kernel parameters (constant bank): the same for every
  // instance (P = 4 GLL)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  using T = Tile<TX_, TY_, EXACT>;
  typename T::Smem& S = *reinterpret_cast<typename T::Smem*>(smem_raw);
  __shared__ RhsConsts Cs;
  __shared__ StageArgs As;
  if constexpr (PERSIST) {
    for (long long t = blockIdx.x; t < B.ntiles; t += gridDim.x)
      batch_tile<MODE, EXACT, TX_, TY_>(B, t, S, Cs, As);
  } else {
    if ((long long)blockIdx.x < B.ntiles) batch_tile<MODE, EXACT, TX_, TY_>(B, blockIdx.x, S, Cs, As);
  }
}

}  // namespace dev
}  // namespace sgnb
