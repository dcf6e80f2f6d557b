// sgnb_kernels_mixed.cuh -- mixed-precision variant of the fused right-hand side and
// BS3(2) stage kernels.
//
// Precision split (every term of src/physics/sgn_flux2d.h appears in exactly one part):
//   FP64  the well-balanced hydrostatic flux 0.5 g (h^2 - H^2) of the normal momentum, its
//         Rusanov central average, its FR-corrected derivative, and the bathymetry source
//         g (h - H) grad H. These two cancel to O(g h grad eta); the cancellation happens
//         in FP64 and only the result is rounded to FP32. The terms linear in the
//         discharges hu, hv: the mass flux hn and the c^2 hn part of the hp flux, their
//         central face averages and FR-corrected derivatives, and the Rusanov jumps of h,
//         hu and hv (formed in FP64, then rounded). hu and hv stay FP64 in shared memory:
//         a 5-point derivative of FP32-rounded discharges puts grid-scale noise of
//         relative size 2^-24 |D| / J into dh/dt, which the adaptive step sequence of
//         configuration 1 amplifies past an eta error of 1e-6 (rounding only hw and hp, or
//         only the stored k, stays near 1e-7). For the same reason the FR derivative of
//         eta = h - H and the depth gradient D eta + grad H of the non-conservative
//         products are FP64, and the 5-point derivatives of the momentum fluxes (which
//         carry hp linearly) accumulate their FP32 flux values in FP64; each is rounded
//         once, after the sum. The state, the RK stage combinations, the embedded error
//         estimate and the controller are FP64 too.
//   FP32  the remaining deviations from the lake at rest: the advective (quadratic)
//         fluxes, the hw and hp fluxes apart from c^2 hn, the Rusanov dissipation
//         lam/2 (U_R - U_L) of hw and hp, wave speeds, the FR derivatives of these fluxes,
//         the products c^2 u h_x of the non-conservative terms, and the sources
//         gamma p grad H, gamma p, -2 c^2 (w + u H_x + v H_y).
// At rest every FP32 term is exactly zero, so the lake-at-rest residual is the FP64 one.
// Stage derivatives k are stored in FP32 (the RK accumulation u + dt sum b_i k_i and the
// error estimate promote them to FP64).
//
// Layout and work decomposition are those of sgnb_kernels.cuh (8 x 4 element tiles, 5 warps,
// lane = element, warp = GLL line); shared memory is 56.3 KB, so 3 CTAs fit per SM.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "sgnb_device.h"
#include "sgnb_checked.cuh"
#include "sgnb_fastmath.cuh"

namespace sgnb {
namespace mix {

constexpr int NP = 5, NPP = 25, NV = 5;
constexpr int TX = 8, TY = 4, TE = TX * TY;
constexpr int NWARP = 5, NTHR = 32 * NWARP;
constexpr int NHALO = 2 * TY + 2 * TX;
constexpr int RUN = TX * NPP;
constexpr int NIT = TY * RUN / NTHR;
constexpr int NHIT = (NV * NHALO * NP + NTHR - 1) / NTHR;
constexpr int NFACE = (2 * TE + TY + TX) * NP;
constexpr int NFIT = (NFACE + NTHR - 1) / NTHR;

enum : int { MODE_RHS = 0, MODE_STAGE = 1, MODE_FSAL = 2 };

struct Smem {
  double h[TE][NPP];          // full depth (FP64)
  double H[TE][NPP];          // nodal still depth (its gradient is formed from it)
  double d[2][TE][NPP];       // hu, hv (FP64: their linear fluxes are formed in FP64)
  float q[2][TE][NPP];        // hw, hp (FP32 deviations)
  float G[NV + 1][TE][NPP];   // column-pass results (dG incl. the y hydrostatic part, By)
  double hhalo[3 * NHALO * NP];  // halo h, hu, hv; slot layout of sgnb_kernels.cuh
  float qhalo[2 * NHALO * NP];   // halo hw, hp
  double Hf[(2 * TE + TY + TX) * NP];
  double red[NWARP][3];
};

__device__ __forceinline__ double& hf_x(Smem& S, int i, int t) { return S.Hf[i * NP + t]; }
__device__ __forceinline__ double& hf_y(Smem& S, int i, int t) { return S.Hf[(TE + i) * NP + t]; }
__device__ __forceinline__ double& hf_xr(Smem& S, int iy, int t) { return S.Hf[(2 * TE + iy) * NP + t]; }
__device__ __forceinline__ double& hf_yt(Smem& S, int ix, int t) { return S.Hf[(2 * TE + TY + ix) * NP + t]; }

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

struct StageInM {
  const double* __restrict__ in;
  const double* __restrict__ u;
  const float* __restrict__ k;
  const float* __restrict__ k1;
  const float* __restrict__ k2;
  const float* __restrict__ k3;
  double acoef, dt;
};

// FP64 stage combinations (src/solver/rk.cpp:100-108 with FP32 derivatives promoted),
// every product and sum rounded on its own: a tile forms its own nodes and its
// neighbours' halo nodes in different code, and the two must agree bit for bit.
__device__ __forceinline__ double stage_m(double u, double acoef, float k) {
  return __dadd_rn(u, __dmul_rn(acoef, (double)k));
}
__device__ __forceinline__ double fsal_m(double u, float k1, float k2, float k3, double dt) {
  const double s = __dadd_rn(__dadd_rn(__dmul_rn(2.0 / 9.0, (double)k1), __dmul_rn(1.0 / 3.0, (double)k2)),
                             __dmul_rn(4.0 / 9.0, (double)k3));
  return __dadd_rn(u, __dmul_rn(dt, s));
}

template <int MODE>
__device__ __forceinline__ double stage_value(const StageInM& I, long long idx) {
  if constexpr (MODE == MODE_RHS) {
    return I.in[idx];
  } else if constexpr (MODE == MODE_STAGE) {
    return stage_m(I.u[idx], I.acoef, I.k[idx]);
  } else {
    return fsal_m(I.u[idx], I.k1[idx], I.k2[idx], I.k3[idx], I.dt);
  }
}

// Nodal still-depth gradient at node (a, b) of an element from its nodal depths He (FP64):
// the element-local GLL derivative over the Jacobian (src/solver/sgn2d.cpp:54-71), formed
// from the depth tile instead of read from the precomputed arrays.
template <int DIR, class TC, class TB>
__device__ __forceinline__ double depth_grad(const TC& C, const TB& Tb, const double* He, int a,
                                             int b) {
  const int m = DIR == 0 ? a : b;
  double s = Tb.D[m * NP] * He[DIR == 0 ? NP * b : a];
#pragma unroll
  for (int k = 1; k < NP; ++k) s = fma(Tb.D[m * NP + k], He[DIR == 0 ? k + NP * b : a + NP * k], s);
  return s * (DIR == 0 ? C.iJx : C.iJy);
}

// One point as seen by the FP32 part.
struct PtF {
  float h, hn, hu, hv, hw, hp;  // full depth (rounded), normal discharge, discharges
  float u, v, w, p;             // primitives
};

template <int DIR>
__device__ __forceinline__ PtF make_pt(double h64, float hu, float hv, float hw, float hp) {
  PtF s;
  s.h = (float)h64;
  s.hu = hu; s.hv = hv; s.hw = hw; s.hp = hp;
  s.hn = DIR == 0 ? hu : hv;
  const float r = __fdividef(1.0f, s.h);
  s.u = hu * r; s.v = hv * r; s.w = hw * r; s.p = hp * r;
  return s;
}

// FP32 (deviation) part of flux field v. The hydrostatic term of the normal momentum, the
// mass flux hn and the c^2 hn part of the hp flux are formed in FP64 elsewhere.
template <int DIR, class TC>
__device__ __forceinline__ float flux_dev(const TC& C, int v, const PtF& s) {
  switch (v) {
    case 0: return 0.0f;
    case 1: return DIR == 0 ? s.hu * s.u + s.hp : s.hv * s.u;
    case 2: return DIR == 0 ? s.hu * s.v : s.hv * s.v + s.hp;
    case 3: return s.hn * s.w;
    default: return s.hn * s.p;
  }
}

template <int DIR, class TC>
__device__ __forceinline__ float wave_speed_f(const TC& C, const PtF& s) {
  const float arg = (float)C.g * s.h + s.p + (float)C.c2;
  return fabsf(DIR == 0 ? s.u : s.v) + sqrtf(fmaxf(arg, 0.0f));
}

// Hydrostatic part of the normal momentum flux, FP64: 0.5 g (h^2 - H^2) as
// 0.5 g (h - H)(h + H), which is exact at rest and cancels no digits.
template <class TC>
__device__ __forceinline__ double hydro64(const TC& C, double h, double Hl) {
  return C.halfg * ((h - Hl) * (h + Hl));
}

// One GLL line: dyn[5] (FR derivatives of the fluxes: the FP64 linear parts plus the FP32
// deviation parts, rounded once), hyd (FP64 FR derivative of the hydrostatic flux of the
// normal momentum) and deta (FP64 FR derivative of eta = h - H with the central face depth:
// a 5-point derivative of FP32-rounded eta would put grid-scale noise into the
// non-conservative products, as a derivative of FP32 discharges would into dh/dt).
// Emitted per node through the callbacks.
//   h[k]      full depth at the nodes (FP64), Hn[k] nodal still depth
//   hn[k]     FP64 normal discharge at the nodes; tLo64 / tHi64 the FP64 tangential
//             discharge at the two face nodes
//   qf[k][4]  FP32 hu, hv, hw, hp at the nodes
//   nd, nq    the neighbour node across each face: FP64 h, hu, hv and FP32 hw, hp
template <int DIR, class TC, class TB, class EmitN, class Emit>
__device__ __forceinline__ void line_mixed(const TC& C, const TB& Tb, const double (&h)[NP],
                                           const double (&Hn)[NP], const double (&hn)[NP],
                                           double tLo64, double tHi64, const float (&qf)[NP][4],
                                           const double* ndLo, const float* nqLo,
                                           const double* ndHi, const float* nqHi, double HfLo,
                                           double HfHi, EmitN&& emit_node, Emit&& emit) {
  PtF s[NP];
  double hyd[NP];
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    s[k] = make_pt<DIR>(h[k], qf[k][0], qf[k][1], qf[k][2], qf[k][3]);
    hyd[k] = hydro64(C, h[k], Hn[k]);
  }
  const PtF sLo = make_pt<DIR>(ndLo[0], (float)ndLo[1], (float)ndLo[2], nqLo[0], nqLo[1]);
  const PtF sHi = make_pt<DIR>(ndHi[0], (float)ndHi[1], (float)ndHi[2], nqHi[0], nqHi[1]);
  const PtF& tLo = s[0];
  const PtF& tHi = s[NP - 1];
  // Rusanov, FP32 deviation part (sgn_flux2d.h:169-179)
  const float lamLo = fmaxf(wave_speed_f<DIR>(C, sLo), wave_speed_f<DIR>(C, tLo));
  const float lamHi = fmaxf(wave_speed_f<DIR>(C, tHi), wave_speed_f<DIR>(C, sHi));
  // jumps of the conserved variables: h, hu, hv in FP64, rounded after the difference
  const float dhLo = (float)(h[0] - ndLo[0]), dhHi = (float)(ndHi[0] - h[NP - 1]);
  float jLo[NV], jHi[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const float FdLo = flux_dev<DIR>(C, v, tLo), FdHi = flux_dev<DIR>(C, v, tHi);
    const float FnLo = flux_dev<DIR>(C, v, sLo), FnHi = flux_dev<DIR>(C, v, sHi);
    float duLo, duHi;  // own minus neighbour (low face), neighbour minus own (high face)
    switch (v) {
      case 0: duLo = dhLo; duHi = dhHi; break;
      case 1:
        duLo = (float)((DIR == 0 ? hn[0] : tLo64) - ndLo[1]);
        duHi = (float)(ndHi[1] - (DIR == 0 ? hn[NP - 1] : tHi64));
        break;
      case 2:
        duLo = (float)((DIR == 1 ? hn[0] : tLo64) - ndLo[2]);
        duHi = (float)(ndHi[2] - (DIR == 1 ? hn[NP - 1] : tHi64));
        break;
      case 3: duLo = tLo.hw - sLo.hw; duHi = sHi.hw - tHi.hw; break;
      default: duLo = tLo.hp - sLo.hp; duHi = sHi.hp - tHi.hp; break;
    }
    jLo[v] = 0.5f * (FnLo - FdLo) - 0.5f * lamLo * duLo;
    jHi[v] = 0.5f * (FnHi - FdHi) - 0.5f * lamHi * duHi;
  }
  // hydrostatic jumps at the faces (FP64): central average minus own face value
  const double jHydLo = 0.5 * (hydro64(C, ndLo[0], HfLo) - hydro64(C, h[0], HfLo));
  const double jHydHi = 0.5 * (hydro64(C, ndHi[0], HfHi) - hydro64(C, h[NP - 1], HfHi));
  // central jumps of the normal discharge (FP64): the mass flux hn and the c^2 hn part of
  // the hp flux share its FR-corrected derivative dlin (their Rusanov dissipation, on h
  // and on hp, is in the FP32 part)
  const double jcLo = 0.5 * (ndLo[1 + DIR] - hn[0]);
  const double jcHi = 0.5 * (ndHi[1 + DIR] - hn[NP - 1]);
  // depth jumps with the central common depth h* = (h- + h+)/2 (sgn2d.cpp:213-214)
  const double jeLo = -0.5 * (h[0] - ndLo[0]), jeHi = 0.5 * (ndHi[0] - h[NP - 1]);
  const float iJ = (float)(DIR == 0 ? C.iJx : C.iJy);
  const double iJ64 = DIR == 0 ? C.iJx : C.iJy;
  double dlin[NP];
#pragma unroll
  for (int m = 0; m < NP; ++m) {
    double se = jeLo * Tb.gLp[m] + jeHi * Tb.gRp[m];
    double sh = jHydLo * Tb.gLp[m] + jHydHi * Tb.gRp[m];
    double sl = jcLo * Tb.gLp[m] + jcHi * Tb.gRp[m];
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      se = fma(Tb.D[m * NP + k], h[k] - Hn[k], se);
      sh = fma(Tb.D[m * NP + k], hyd[k], sh);
      sl = fma(Tb.D[m * NP + k], hn[k], sl);
    }
    dlin[m] = sl * iJ64;
    emit_node(m, se * iJ64, sh * iJ64, s[m]);
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    float F[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) F[k] = flux_dev<DIR>(C, v, s[k]);
#pragma unroll
    for (int m = 0; m < NP; ++m) {
      float d;
      if (v == 1 || v == 2) {
        // the momentum fluxes carry hp linearly (|hp| grows to ~10 |hu| on configuration
        // 1): their FP32 values are contracted in FP64, rounded once
        double a = (double)jLo[v] * Tb.gLp[m];
        a = fma((double)jHi[v], Tb.gRp[m], a);
#pragma unroll
        for (int k = 0; k < NP; ++k) a = fma(Tb.D[m * NP + k], (double)F[k], a);
        d = (float)(a * iJ64);
      } else {
        float a = jLo[v] * Tb.gLpf[m];
        a = fmaf(jHi[v], Tb.gRpf[m], a);
        if (v != 0) {
#pragma unroll
          for (int k = 0; k < NP; ++k) a = fmaf(Tb.Df[m * NP + k], F[k], a);
        }
        d = a * iJ;
      }
      if (v == 0) d = (float)(dlin[m] + (double)d);
      else if (v == NV - 1) d = (float)(C.c2 * dlin[m] + (double)d);
      emit(m, v, d, s[m]);
    }
  }
}

// One tile (bx, by) of the mixed-precision right-hand side / stage kernel, error partial
// slot blk. Shared by the single-instance kernel and the batched kernel. FULL: the mesh is
// a whole number of tiles (the per-item range checks are compiled out).
// TMA: the intermediate stage's nodal depths and FP32 stage derivatives arrive by
// tensor-memory-accelerator copies described by M (full tiles of the single-instance
// kernel only).
template <int MODE, class TC, class TB, class TA, bool FRIC = false, bool FULL = false,
          bool TMA = false>
__device__ __forceinline__ void mixed_tile(const TC& C, const TB& Tb, const TA& A, int bx, int by,
                                           long long blk, Smem& S,
                                           const TileMapsM* M = nullptr) {
  static_assert(!TMA || (FULL && MODE == MODE_STAGE), "tile copies: full tiles, intermediate stage");

  int cur = 0;
  double atol = 0.0, rtol = 0.0;
  StageInM I;
  I.in = A.in;
  I.dt = 0.0;
  I.acoef = 0.0;
  if constexpr (MODE != MODE_RHS) {
    if (A.ctrl->done) return;
    cur = A.ctrl->cur;
    I.dt = A.ctrl->dt;
    I.acoef = A.coef * I.dt;
    atol = A.ctrl->atol;
    rtol = A.ctrl->rtol;
  }
  I.u = A.U[cur];
  I.k = A.kin_k2 ? A.K2 : A.K1[cur];
  I.k1 = A.K1[cur];
  I.k2 = A.K2;
  I.k3 = A.K3;

  int tid;  // opaque: keeps per-thread descriptors out of the batched kernel's tile loop
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
  const bool wallL = C.bcx && ex0 == 0, wallR = C.bcx && ex0 + TXv == Nx;
  const bool wallB = C.bcy && ey0 == 0, wallT = C.bcy && ey0 + TYv == Ny;

  int gof[NIT];  // node offset within one field (Nd <= 2^31 by the mesh-size limit)
  int sof[NIT];
  bool okk[NIT];
  auto item_map = [&]() {
#pragma unroll
    for (int u = 0; u < NIT; ++u) {
      // the end-point stage on full tiles keeps a thread's items in one tile row, NTHR /
      // TY doubles apart (one base address and immediate offsets: 1.1 % faster); the other
      // modes and partial tiles (the batched kernel, 0.9 % faster so) take q = tid + NTHR*u
      // in tile-row order
      constexpr int PER_ROW = NTHR / TY;
      static_assert(NTHR % TY == 0 && RUN == NIT * PER_ROW, "items split evenly over the rows");
      int iy, k;
      if constexpr (MODE == MODE_FSAL && FULL) {
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

  // ---- load phase ----------------------------------------------------------------
  const unsigned mbar = smem_addr(&S.red[0][0]);  // TMA: the tile copies' barrier
  {
    // statics by asynchronous copies straight into shared memory (TMA: one thread copies
    // the nodal depths and the stage derivative, one field of the tile per copy, on an
    // mbarrier that aliases the not yet used reduction slots)
    if constexpr (TMA) {
      if (tid == 0) mbar_init(mbar);
      __syncthreads();
      if (tid == 0) {
        const int x = ex0 * NPP;  // 16-byte aligned: 800 bytes of FP32 per tile column
        mbar_expect_tx(mbar, (unsigned)(TE * NPP * (sizeof(double) + NV * sizeof(float))));
        tma_load_2d(smem_addr(&S.H[0][0]), &M->H, x, ey0, mbar);
        const CUtensorMap* mk = A.kin_k2 ? &M->K2 : &M->K1[cur];
#pragma unroll 1
        for (int v = 0; v < NV; ++v) tma_load_3d(smem_addr(&S.G[v][0][0]), mk, x, ey0, v, mbar);
      }
    } else {
#pragma unroll
      for (int u = 0; u < NIT; ++u)
        if (okk[u]) {
          if (SGNB_INB(gof[u], Nd)) cp_async8(&(&S.H[0][0])[sof[u]], C.Hnod + gof[u]);
        }
    }
    // halos: the neighbour tiles' trace nodes, stage inputs formed in registers
    double hv[NHIT];
    int hq[NHIT];
    auto halo_load = [&]() {
      long long hg[NHIT];
#pragma unroll
      for (int u = 0; u < NHIT; ++u) {
        const int q = tid + NTHR * u;
        const int t = q % NP, r = q / NP;
        const int slot = r % NHALO, v = r / NHALO;
        bool ok = q < NV * NHALO * NP;
        long long e = 0;
        int node = 0;
        if (slot < TY) {
          ok = ok && slot < TYv && !wallL;
          e = (long long)(exL) + (long long)Nx * (ey0 + slot);
          node = (NP - 1) + NP * t;
        } else if (slot < 2 * TY) {
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
        hg[u] = (long long)v * Nd + e * NPP + node;
      }
#pragma unroll
      for (int u = 0; u < NHIT; ++u)
        if (hq[u] >= 0 && SGNB_INB(hg[u], NV * Nd)) hv[u] = stage_value<MODE>(I, hg[u]);
    };
    // face depths through registers (right-hand-side mode)
    auto face_load = [&](double (&fv)[NFIT], int (&fq)[NFIT]) {
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
              fv[u] = SGNB_INB(wallR ? (long long)ey * NP + t
                                     : ((long long)(exR) + (long long)Nx * ey) * NP + t,
                               wallR ? (long long)Ny * NP : Nd / NP)
                          ? (wallR ? C.HfXEnd[(long long)ey * NP + t]
                            : C.HfX[((long long)(exR) + (long long)Nx * ey) * NP + t])
                          : 0.0;
              fq[u] = q;
            }
          } else if (slot - TY < TXv) {
            const int ex = ex0 + slot - TY;
            fv[u] = SGNB_INB(wallT ? (long long)ex * NP + t
                                   : ((long long)ex + (long long)Nx * (eyT)) * NP + t,
                             wallT ? (long long)Nx * NP : Nd / NP)
                        ? (wallT ? C.HfYEnd[(long long)ex * NP + t]
                          : C.HfY[((long long)ex + (long long)Nx * (eyT)) * NP + t])
                        : 0.0;
            fq[u] = q;
          }
        }
      }
    };
    // stage modes: face depths by asynchronous copies straight into shared memory, issued
    // with the statics (the right-hand-side mode is faster loading them after its state)
    if constexpr (MODE != MODE_RHS) {
#pragma unroll
      for (int u = 0; u < NFIT; ++u) {
        const int q = tid + NTHR * u;
        const double* fp = nullptr;  // source of face-depth item q (none: not in this tile)
        bool fok = false;
        if (q < 2 * TE * NP) {
          const int t = q % NP, i = (q / NP) % TE, s = q / (NP * TE);
          const int ix = i % TX, iy = i / TX;
          if (ix < TXv && iy < TYv) {
            const long long e = (long long)(ex0 + ix) + (long long)Nx * (ey0 + iy);
            fok = true;
            if (SGNB_INB(e * NP + t, Nd / NP)) fp = (s == 0 ? C.HfX : C.HfY) + e * NP + t;
          }
        } else if (q < NFACE) {
          const int r = q - 2 * TE * NP;
          const int t = r % NP, slot = r / NP;
          if (slot < TY) {
            if (slot < TYv) {
              const int ey = ey0 + slot;
              const long long fe = (long long)ey * NP + t;
              const long long fx = ((long long)(exR) + (long long)Nx * ey) * NP + t;
              fok = true;
              if (wallR) { if (SGNB_INB(fe, (long long)Ny * NP)) fp = C.HfXEnd + fe; }
              else if (SGNB_INB(fx, Nd / NP)) fp = C.HfX + fx;
            }
          } else if (slot - TY < TXv) {
            const int ex = ex0 + slot - TY;
            const long long fe = (long long)ex * NP + t;
            const long long fy = ((long long)ex + (long long)Nx * (eyT)) * NP + t;
            fok = true;
            if (wallT) { if (SGNB_INB(fe, (long long)Nx * NP)) fp = C.HfYEnd + fe; }
            else if (SGNB_INB(fy, Nd / NP)) fp = C.HfY + fy;
          }
        }
        if (fok && SGNB_INB(q, NFACE)) {
          if (fp) cp_async8(&S.Hf[q], fp);
          else S.Hf[q] = 0.0;
        }
      }
    }
    double* __restrict__ unew = A.U[cur ^ 1];
    if constexpr (MODE == MODE_STAGE && !TMA) {
      // k (FP32) by asynchronous copies into the still unused G area
#pragma unroll
      for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int u = 0; u < NIT; ++u)
          if (okk[u] && SGNB_INB(gof[u], Nd)) {
            const unsigned sa = (unsigned)__cvta_generic_to_shared(&(&S.G[v][0][0])[sof[u]]);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa),
                         "l"((I.k + (long long)v * Nd) + gof[u]) : "memory");
          }
    }
    // end-point stage: k1 and k2 by asynchronous copies into the (still unused) G, q and d
    // areas, ten FP32 fields: those of fields 0, 1, 2 in G (never written while the
    // candidate is formed), of field 3 in q (hw and hp, written by the same thread at the
    // same index after their read), of field 4 in d viewed as floats (written, as doubles
    // at other indices, only after a barrier that follows every read)
    auto k12_slot = [&](int w, int v) -> float* {  // w: 0 = k1, 1 = k2
      if (v < 3) return &S.G[2 * v + w][0][0];
      if (v == 3) return &S.q[w][0][0];
      return reinterpret_cast<float*>(&S.d[0][0][0]) + w * TE * NPP;
    };
    if constexpr (MODE == MODE_FSAL) {
#pragma unroll
      for (int w = 0; w < 2; ++w)
#pragma unroll
        for (int v = 0; v < NV; ++v)
#pragma unroll
          for (int u = 0; u < NIT; ++u)
            if (okk[u] && SGNB_INB(gof[u], Nd)) {
              const unsigned sa = (unsigned)__cvta_generic_to_shared(k12_slot(w, v) + sof[u]);
              asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa),
                           "l"(((w == 0 ? I.k1 : I.k2) + (long long)v * Nd) + gof[u]) : "memory");
            }
    }
    // end-point stage: the halo loads go first, in flight together with the tile's own
    // (the other modes are faster issuing them after the combination)
    if constexpr (MODE == MODE_FSAL) halo_load();
    // every u load (and, at the end point, every k3 load) of the tile in flight before the
    // first combination
    double ux[NV][NIT];
    float k3x[NV][NIT];
    if constexpr (MODE != MODE_RHS) {
#pragma unroll
      for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int u = 0; u < NIT; ++u)
          if (okk[u] && SGNB_INB(gof[u], Nd)) {
            ux[v][u] = (I.u + (long long)v * Nd)[gof[u]];
            if constexpr (MODE == MODE_FSAL) k3x[v][u] = (I.k3 + (long long)v * Nd)[gof[u]];
          }
      cp_async_wait_all();  // k (k1, k2) and the statics have landed
      if constexpr (TMA) {
        bool landed = false;
        for (int it = 0; it < kTmaTries && !landed; ++it) landed = mbar_try_wait(mbar, 0);
        if (!landed) {
          // the copies did not complete: this thread's state items become NaN, so the
          // launch's results are non-finite and the controller ends the run with that error
          const double nan = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
          for (int v = 0; v < NV; ++v)
#pragma unroll
            for (int u = 0; u < NIT; ++u) ux[v][u] = nan;
        }
      }
    }
    // fields in the order 3, 4, 0, 1, 2: the end-point stage's field-4 derivatives sit in
    // the d area, which fields 1 and 2 overwrite after the barrier
#pragma unroll
    for (int o = 0; o < NV; ++o) {
      const int v = (o + 3) % NV;
      if (MODE == MODE_FSAL && v == 1) __syncthreads();
      double x[NIT];
#pragma unroll
      for (int u = 0; u < NIT; ++u)
        if (okk[u]) {
          if constexpr (MODE == MODE_STAGE)
            x[u] = stage_m(ux[v][u], I.acoef, (&S.G[v][0][0])[sof[u]]);
          else if constexpr (MODE == MODE_FSAL)
            x[u] = fsal_m(ux[v][u], k12_slot(0, v)[sof[u]], k12_slot(1, v)[sof[u]], k3x[v][u],
                          I.dt);
          else
            x[u] = SGNB_INB(gof[u], Nd) ? stage_value<MODE>(I, (long long)v * Nd + gof[u]) : 0.0;
        }
#pragma unroll
      for (int u = 0; u < NIT; ++u)
        if (okk[u]) {
          if (v == 0) (&S.h[0][0])[sof[u]] = x[u];
          else if (v < 3) (&S.d[v - 1][0][0])[sof[u]] = x[u];
          else (&S.q[v - 3][0][0])[sof[u]] = (float)x[u];
          if constexpr (MODE == MODE_FSAL)
            if (SGNB_INB(gof[u], Nd)) __stcs(&(unew + (long long)v * Nd)[gof[u]], x[u]);
        }
    }
    if constexpr (MODE != MODE_FSAL) halo_load();
    double fv[NFIT];
    int fq[NFIT];
    if constexpr (MODE == MODE_RHS) face_load(fv, fq);
#pragma unroll
    for (int u = 0; u < NHIT; ++u)
      if (hq[u] >= 0 && SGNB_INB(hq[u], NV * NHALO * NP)) {
        const int q = hq[u];
        const int v = q / (NHALO * NP), rest = q - v * NHALO * NP;
        if (v < 3) S.hhalo[v * NHALO * NP + rest] = hv[u];
        else S.qhalo[(v - 3) * NHALO * NP + rest] = (float)hv[u];
      }
    if constexpr (MODE == MODE_RHS) {
#pragma unroll
      for (int u = 0; u < NFIT; ++u)
        if (fq[u] >= 0 && SGNB_INB(fq[u], NFACE)) S.Hf[fq[u]] = fv[u];
    }
    cp_async_wait_all();
  }
  __syncthreads();
  if constexpr (TMA) {
    if (tid == 0) mbar_inval(mbar);  // its slots serve the error reduction later
  }

  const int i = lane;
  const int ix = i % TX, iy = i / TX;
  const bool valid = FULL || (ix < TXv && iy < TYv);
  const int j = warp;
  const float c2f = (float)C.c2, mc2f = (float)C.mc2, gammaf = (float)C.gamma;

  // neighbour node across a face: in the tile, in the halo, or the wall mirror (normal
  // discharge negated, nd[1 + DIR])
  auto halo_node = [&](int slot, int t, double* nd, float* nq) {
    const int idx = t + NP * slot;
#pragma unroll
    for (int c = 0; c < 3; ++c) nd[c] = S.hhalo[c * NHALO * NP + idx];
#pragma unroll
    for (int c = 0; c < 2; ++c) nq[c] = S.qhalo[c * NHALO * NP + idx];
  };
  auto tile_node = [&](int e, int loc, double* nd, float* nq) {
    nd[0] = S.h[e][loc];
    nd[1] = S.d[0][e][loc];
    nd[2] = S.d[1][e][loc];
    nq[0] = S.q[0][e][loc];
    nq[1] = S.q[1][e][loc];
  };
  auto mirror_node = [&](int dir, double hh, double hu, double hv, const float* qq, double* nd,
                         float* nq) {
    nd[0] = hh;
    nd[1] = dir == 0 ? -hu : hu;
    nd[2] = dir == 1 ? -hv : hv;
    nq[0] = qq[2];
    nq[1] = qq[3];
  };

  // ---- column pass: y-line a = j ---------------------------------------------
  if (valid) {
    double h[NP], Hn[NP], hn[NP];
    float qf[NP][4];
#pragma unroll
    for (int b = 0; b < NP; ++b) {
      const int loc = j + NP * b;
      h[b] = S.h[i][loc];
      Hn[b] = S.H[i][loc];
      hn[b] = S.d[1][i][loc];
      qf[b][0] = (float)S.d[0][i][loc];
      qf[b][1] = (float)hn[b];
      qf[b][2] = S.q[0][i][loc];
      qf[b][3] = S.q[1][i][loc];
    }
    const double tLo64 = S.d[0][i][j], tHi64 = S.d[0][i][j + NP * (NP - 1)];
    double ndLo[3], ndHi[3];
    float nqLo[2], nqHi[2];
    if (iy > 0) tile_node(i - TX, j + NP * (NP - 1), ndLo, nqLo);
    else if (wallB) mirror_node(1, h[0], tLo64, hn[0], qf[0], ndLo, nqLo);
    else halo_node(2 * TY + ix, j, ndLo, nqLo);
    if (iy + 1 < TYv) tile_node(i + TX, j, ndHi, nqHi);
    else if (wallT) mirror_node(1, h[NP - 1], tHi64, hn[NP - 1], qf[NP - 1], ndHi, nqHi);
    else halo_node(2 * TY + TX + ix, j, ndHi, nqHi);
    const double HfLo = hf_y(S, i, j);
    const double HfHi = (iy + 1 < TYv) ? hf_y(S, i + TX, j) : hf_yt(S, ix, j);
    float hydv[NP];
    line_mixed<1>(
        C, Tb, h, Hn, hn, tLo64, tHi64, qf, ndLo, nqLo, ndHi, nqHi, HfLo, HfHi,
        [&](int b, double deta, double dhyd, const PtF& s) {
          const int loc = j + NP * b;
          const double Hyl = depth_grad<1>(C, Tb, S.H[i], j, b);
          // ncpY with h_y = D eta + H_y (sgn_flux2d.h:156-161), the sum in FP64
          S.G[NV][i][loc] = mc2f * s.v * (float)(deta + Hyl);
          // y hydrostatic part of dU[HV]: -d_y hyd + g (h - H) H_y, cancelled in FP64
          hydv[b] = (float)(C.g * (h[b] - Hn[b]) * Hyl - dhyd);
        },
        [&](int b, int v, float d, const PtF&) {
          S.G[v][i][j + NP * b] = (v == 2) ? d - hydv[b] : d;
        });
  }
  __syncthreads();

  // ---- row pass: x-line b = j, then assembly ---------------------------------
  if (valid) {
    double h[NP], Hn[NP], hn[NP];
    float qf[NP][4];
#pragma unroll
    for (int a = 0; a < NP; ++a) {
      const int loc = a + NP * j;
      h[a] = S.h[i][loc];
      Hn[a] = S.H[i][loc];
      hn[a] = S.d[0][i][loc];
      qf[a][0] = (float)hn[a];
      qf[a][1] = (float)S.d[1][i][loc];
      qf[a][2] = S.q[0][i][loc];
      qf[a][3] = S.q[1][i][loc];
    }
    const double tLo64 = S.d[1][i][NP * j], tHi64 = S.d[1][i][(NP - 1) + NP * j];
    double ndLo[3], ndHi[3];
    float nqLo[2], nqHi[2];
    if (ix > 0) tile_node(i - 1, (NP - 1) + NP * j, ndLo, nqLo);
    else if (wallL) mirror_node(0, h[0], hn[0], tLo64, qf[0], ndLo, nqLo);
    else halo_node(iy, j, ndLo, nqLo);
    if (ix + 1 < TXv) tile_node(i + 1, NP * j, ndHi, nqHi);
    else if (wallR) mirror_node(0, h[NP - 1], hn[NP - 1], tHi64, qf[NP - 1], ndHi, nqHi);
    else halo_node(TY + iy, j, ndHi, nqHi);
    const double HfLo = hf_x(S, i, j);
    const double HfHi = (ix + 1 < TXv) ? hf_x(S, i + 1, j) : hf_xr(S, iy, j);
    float hydu[NP], Bx[NP], Hxf[NP];
    line_mixed<0>(
        C, Tb, h, Hn, hn, tLo64, tHi64, qf, ndLo, nqLo, ndHi, nqHi, HfLo, HfHi,
        [&](int a, double deta, double dhyd, const PtF& s) {
          const double Hxl = depth_grad<0>(C, Tb, S.H[i], a, j);
          Bx[a] = mc2f * s.u * (float)(deta + Hxl);  // ncpX, h_x summed in FP64
          hydu[a] = (float)(C.g * (h[a] - Hn[a]) * Hxl - dhyd);
          Hxf[a] = (float)Hxl;
        },
        [&](int a, int v, float d, const PtF& s) {
          const int loc = a + NP * j;
          const float g = S.G[v][i][loc];
          float res;
          if (v == 0) {
            res = -(d + g);
          } else if (v == 1 || v == 2) {
            // Manning friction n^2 g |vel| vel / h^(1/3), a deviation term (FP32)
            float fr = 0.0f;
            if constexpr (FRIC)
              fr = (float)C.n2g * sqrtf(s.u * s.u + s.v * s.v) / cbrtf(s.h) *
                   (v == 1 ? s.u : s.v);
            res = v == 1 ? hydu[a] + gammaf * s.p * Hxf[a] - fr - (d + g)
                         : gammaf * s.p * (float)depth_grad<1>(C, Tb, S.H[i], a, j) - fr - (d + g);
          } else if (v == 3) {
            res = gammaf * s.p - (d + g);
          } else {
            const float Hxl = Hxf[a], Hyl = (float)depth_grad<1>(C, Tb, S.H[i], a, j);
            const float S4 = (float)C.m2c2 * (s.w + s.u * Hxl + s.v * Hyl);
            res = S4 - (d + g) - Bx[a] - S.G[NV][i][loc];
          }
          S.G[v][i][loc] = res;
        });
  }
  __syncthreads();

  // ---- copy-out and the FP64 embedded error of the end-point stage ---------------
  // Results are stored, and the end-point stage's last reads of u, k1, k2, k3 loaded,
  // with the streaming (evict-first) hint, as in the FP64 kernels.
  double esum = 0.0, emax = 0.0;
  int enan = 0;
  item_map();
  if constexpr (MODE == MODE_RHS) {
    // FP64 output for rhs callers, FP32 into the stage buffer for the FSAL head
#pragma unroll 1
    for (int v = 0; v < NV; ++v)
#pragma unroll
      for (int u = 0; u < NIT; ++u)
        if (okk[u] && SGNB_INB(gof[u], Nd)) {
          const float val = (&S.G[v][0][0])[sof[u]];
          if (A.outd) __stcs(&(A.outd + (long long)v * Nd)[gof[u]], (double)val);
          else __stcs(&(A.out + (long long)v * Nd)[gof[u]], val);
        }
  } else if constexpr (MODE == MODE_STAGE) {
#pragma unroll 1
    for (int v = 0; v < NV; ++v)
#pragma unroll
      for (int u = 0; u < NIT; ++u)
        if (okk[u] && SGNB_INB(gof[u], Nd)) __stcs(&(A.out + (long long)v * Nd)[gof[u]], (&S.G[v][0][0])[sof[u]]);
  } else {
    const CtrlReload rc = ctrl_reload(A.ctrl);
    cur = rc.cur;
    const double dt = rc.dt;
    atol = rc.atol;
    rtol = rc.rtol;
    const double* __restrict__ u0 = A.U[cur];
    const float* __restrict__ k1p = A.K1[cur];
    const float* __restrict__ k2p = A.K2;
    const float* __restrict__ k3p = A.K3;
    float* __restrict__ outp = A.K1[cur ^ 1];
    // next field's u, k1, k2, k3 prefetched while the current field's error is formed
    double uu[NIT], nu[NIT];
    float c1[NIT], c2[NIT], c3[NIT], n1[NIT], n2[NIT], n3[NIT];
#pragma unroll
    for (int u = 0; u < NIT; ++u)
      if (okk[u]) {
        const int g = gof[u];
        if (SGNB_INB(g, Nd)) { uu[u] = __ldcs(&u0[g]); c1[u] = __ldcs(&k1p[g]); c2[u] = __ldcs(&k2p[g]); c3[u] = __ldcs(&k3p[g]); }
      }
#pragma unroll 1
    for (int v = 0; v < NV; ++v) {
      if (v + 1 < NV) {
#pragma unroll
        for (int u = 0; u < NIT; ++u)
          if (okk[u]) {
            const long long o = (long long)(v + 1) * Nd;
            const int gi = gof[u];
            if (SGNB_INB(o + gi, NV * Nd)) { nu[u] = __ldcs(&(u0 + o)[gi]); n1[u] = __ldcs(&(k1p + o)[gi]); n2[u] = __ldcs(&(k2p + o)[gi]); n3[u] = __ldcs(&(k3p + o)[gi]); }
          }
      }
#pragma unroll
      for (int u = 0; u < NIT; ++u)
        if (okk[u]) {
          const float k4 = (&S.G[v][0][0])[sof[u]];
          if (SGNB_INB(gof[u], Nd)) __stcs(&(outp + (long long)v * Nd)[gof[u]], k4);
          const double b1 = c1[u], b2 = c2[u], b3 = c3[u], b4 = k4;
          const double un = uu[u] + dt * (2.0 / 9.0 * b1 + 1.0 / 3.0 * b2 + 4.0 / 9.0 * b3);
          const double uEmb = uu[u] + dt * (7.0 / 24.0 * b1 + 0.25 * b2 + 1.0 / 3.0 * b3 + 0.125 * b4);
          const double e = un - uEmb;
          const double au = fabs(uu[u]), an = fabs(un);
          const double sc = atol + rtol * (au < an ? an : au);
          // the fast reciprocal (a few ulp) where sc is a normal number
          const double rr = sc >= 2.2250738585072014e-308 ? e * dev::fast_rcp(sc) : e / sc;
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

// Resident CTAs per SM the single-instance mixed kernels are compiled for (3 -> at most
// 128 registers per thread, 2 -> 204).
#ifndef SGNB_MIXED_MIN_CTAS
#define SGNB_MIXED_MIN_CTAS 3
#endif

template <int MODE, bool FRIC = false, bool FULL = false>
__global__ void __launch_bounds__(NTHR, SGNB_MIXED_MIN_CTAS) k_mixed(const RhsConsts C, const StageArgsM A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem& S = *reinterpret_cast<Smem*>(smem_raw);
  mixed_tile<MODE, RhsConsts, RhsConsts, StageArgsM, FRIC, FULL>(
      C, C, A, blockIdx.x, blockIdx.y, (long long)blockIdx.y * gridDim.x + blockIdx.x, S);
}

// Intermediate stage on a mesh of whole tiles, with the nodal depths and the stage
// derivative loaded by the tensor-memory accelerator from the context's buffers that M
// describes.
template <int MODE>
__global__ void __launch_bounds__(NTHR, SGNB_MIXED_MIN_CTAS)
    k_mixed_tma(const RhsConsts C, const StageArgsM A, const __grid_constant__ TileMapsM M) {
  extern __shared__ __align__(128) unsigned char smem_tiles_m[];  // the copies' destinations
  Smem& S = *reinterpret_cast<Smem*>(smem_tiles_m);
  mixed_tile<MODE, RhsConsts, RhsConsts, StageArgsM, false, true, true>(
      C, C, A, blockIdx.x, blockIdx.y, (long long)blockIdx.y * gridDim.x + blockIdx.x, S, &M);
}

// Batched form (8x4 tiles): the work list of BatchArgsM, per tile the instance's constants
// and buffer pointers copied into shared memory and read through volatile views.
// PERSIST: a fixed grid loops over the list; otherwise one CTA per tile.
template <int MODE>
__device__ __forceinline__ void mixed_batch_tile(const BatchArgsM& B, long long t, Smem& S,
                                                 RhsConsts& Cs, StageArgsM& As) {
  const int inst = B.tile_inst[t];
  const long long lt = t - B.tile_start[inst];
  __syncthreads();  // the previous tile is done with Cs / As
  {
    // both blocks' loads in flight before the first store (one round trip per tile)
    block_copy2<(int)(sizeof(RhsConsts) / 4), (int)(sizeof(StageArgsM) / 4), NTHR>(
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
  const int ntx = (Cs.Nx + TX - 1) / TX;
  mixed_tile<MODE>(static_cast<const volatile RhsConsts&>(Cs), B.tables,
                   static_cast<const volatile StageArgsM&>(As), (int)(lt % ntx), (int)(lt / ntx),
                   lt, S);
}

template <int MODE, bool PERSIST>
__global__ void __launch_bounds__(NTHR, 3) k_mixed_batch(const BatchArgsM B) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem& S = *reinterpret_cast<Smem*>(smem_raw);
  __shared__ RhsConsts Cs;
  __shared__ StageArgsM As;
  if constexpr (PERSIST) {
    for (long long t = blockIdx.x; t < B.ntiles; t += gridDim.x) mixed_batch_tile<MODE>(B, t, S, Cs, As);
  } else {
    if ((long long)blockIdx.x < B.ntiles) mixed_batch_tile<MODE>(B, blockIdx.x, S, Cs, As);
  }
}

}  // namespace mix
}  // namespace sgnb
