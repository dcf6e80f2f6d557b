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

namespace sgnb {
namespace dev {

constexpr int NP = 5;          // GLL points per direction (P = 4)
constexpr int NPP = 25;        // nodes per element
constexpr int NV = 5;          // conserved fields h, hu, hv, hw, hp
constexpr int TX = 8;          // tile width in elements
constexpr int TY = 4;          // tile height in elements
constexpr int TE = TX * TY;    // elements per tile = lanes per warp
constexpr int NWARP = 5;       // one warp per GLL line index
constexpr int NTHR = 32 * NWARP;

static_assert(TE == 32, "one tile element per lane");

// Stage modes of the fused kernel.
enum : int {
  MODE_RHS = 0,    // dU = R(U)
  MODE_STAGE = 1,  // k_out = R(u + coef*dt*k_in)
  MODE_FSAL = 2    // uNew = u + dt(2/9 k1 + 1/3 k2 + 4/9 k3); k4 = R(uNew); error partials
};

struct Smem {
  double U[NV][TE][NPP];       // tile state (input of R)
  double H[TE][NPP];           // nodal still depth
  double Hx[TE][NPP];          // nodal dH/dx
  double Hy[TE][NPP];          // nodal dH/dy
  double G[NV + 1][TE][NPP];   // column-pass results dG (5 fields) and By; then dU
  double haloL[NV][TY][NP];    // node (4,b) of the element left of the tile, per row
  double haloR[NV][TY][NP];    // node (0,b) of the element right of the tile
  double haloB[NV][TX][NP];    // node (a,4) of the element below the tile, per column
  double haloT[NV][TX][NP];    // node (a,0) of the element above the tile
  double HfX[TE][NP];          // left-edge depth of each tile element
  double HfY[TE][NP];          // bottom-edge depth
  double HfXR[TY][NP];         // right-edge depth of the last tile column, per row
  double HfYT[TX][NP];         // top-edge depth of the last tile row, per column
  double red[NWARP][3];        // block reduction of the error partials
};

// Stage input of one value: plain, u + (coef dt) k, or the BS3 candidate.
// Expression trees follow src/solver/rk.cpp:100-108 exactly.
template <int MODE>
__device__ __forceinline__ double stage_value(const StageArgs& A, int cur, double dt,
                                              double acoef, long long idx) {
  if constexpr (MODE == MODE_RHS) {
    return A.in[idx];
  } else if constexpr (MODE == MODE_STAGE) {
    return A.U[cur][idx] + acoef * (A.kin_k2 ? A.K2 : A.K1[cur])[idx];
  } else {
    return A.U[cur][idx] + dt * (2.0 / 9.0 * A.K1[cur][idx] + 1.0 / 3.0 * A.K2[idx] +
                                 4.0 / 9.0 * A.K3[idx]);
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
  __device__ __forceinline__ Prim(const double* U) {
    if constexpr (EXACT) {
      u = U[1] / U[0]; v = U[2] / U[0]; w = U[3] / U[0]; p = U[4] / U[0];
    } else {
      const double ih = 1.0 / U[0];
      u = U[1] * ih; v = U[2] * ih; w = U[3] * ih; p = U[4] * ih;
    }
  }
};

// Directional flux: fluxX (DIR 0) or fluxY (DIR 1), src/physics/sgn_flux2d.h:89-116.
template <bool EXACT, int DIR>
__device__ __forceinline__ void flux(const RhsConsts& C, const double* U, const Prim<EXACT>& q,
                                     double Hloc, double* F) {
  const double h = U[0];
  const double hn = DIR == 0 ? U[1] : U[2];  // normal discharge
  const double hyd = C.halfg * (h * h - Hloc * Hloc);
  const double hp = EXACT ? h * q.p : U[4];
  F[0] = hn;
  if constexpr (DIR == 0) {
    F[1] = hn * q.u + hyd + hp;
    F[2] = hn * q.v;
  } else {
    F[1] = hn * q.u;
    F[2] = hn * q.v + hyd + hp;
  }
  F[3] = hn * q.w;
  F[4] = hn * (q.p + C.c2);
}

// |normal velocity| + sqrt(max(g h + p + c^2, 0)), src/physics/sgn_flux2d.h:73-86.
template <bool EXACT, int DIR>
__device__ __forceinline__ double wave_speed(const RhsConsts& C, const double* U,
                                             const Prim<EXACT>& q) {
  const double arg = C.g * U[0] + q.p + C.c2;
  const double ce = sqrt(arg > 0.0 ? arg : 0.0);
  return fabs(DIR == 0 ? q.u : q.v) + ce;
}

// Results of one GLL line (5 nodes) in one direction.
struct LineOut {
  double d[NP][NV];  // FR-corrected flux derivative of each node, /J
  double dh[NP];     // FR-corrected depth derivative of each node, /J
};

// The line computation shared by the row (DIR 0) and column (DIR 1) passes:
// nodal fluxes, both Rusanov face fluxes with central depths, the element's own
// face fluxes, the 5-point differentiation and the correction lift
// (src/solver/sgn2d.cpp:188-275 restricted to one line).
//   Un[k]   raw node states along the line, k = 0..4 (low face at k = 0)
//   Hn[k]   nodal still depth
//   nLo/nHi raw node state of the neighbour across the low/high face (or the mirror
//           ghost at a wall)
//   HfLo/HfHi still depth at the two faces
template <bool EXACT, int DIR>
__device__ __forceinline__ void line_pass(const RhsConsts& C, const double (&Un)[NP][NV],
                                          const double (&Hn)[NP], const double* nLo,
                                          const double* nHi, double HfLo, double HfHi,
                                          LineOut& out) {
  // nodal fluxes
  double F[NP][NV];
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    const Prim<EXACT> q(Un[k]);
    flux<EXACT, DIR>(C, Un[k], q, Hn[k], F[k]);
  }
  // face traces (own side and the neighbour side)
  double tLo[NV], tHi[NV], sLo[NV], sHi[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    tLo[v] = canon<EXACT>(Un[0][v]);
    tHi[v] = canon<EXACT>(Un[NP - 1][v]);
    sLo[v] = canon<EXACT>(nLo[v]);
    sHi[v] = canon<EXACT>(nHi[v]);
  }
  const Prim<EXACT> qtLo(tLo), qtHi(tHi), qsLo(sLo), qsHi(sHi);
  // own face fluxes Fd (sgn2d.cpp:229-239) and the neighbours' fluxes at the faces
  double FdLo[NV], FdHi[NV], FnLo[NV], FnHi[NV];
  flux<EXACT, DIR>(C, tLo, qtLo, HfLo, FdLo);
  flux<EXACT, DIR>(C, tHi, qtHi, HfHi, FdHi);
  flux<EXACT, DIR>(C, sLo, qsLo, HfLo, FnLo);
  flux<EXACT, DIR>(C, sHi, qsHi, HfHi, FnHi);
  // Rusanov (sgn_flux2d.h:169-179); the low face has the neighbour on its left
  const double lamLo = fmax(wave_speed<EXACT, DIR>(C, sLo, qsLo), wave_speed<EXACT, DIR>(C, tLo, qtLo));
  const double lamHi = fmax(wave_speed<EXACT, DIR>(C, tHi, qtHi), wave_speed<EXACT, DIR>(C, sHi, qsHi));
  double jLo[NV], jHi[NV];  // common flux minus own face flux
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double fsLo = 0.5 * (FnLo[v] + FdLo[v]) - 0.5 * lamLo * (tLo[v] - sLo[v]);
    const double fsHi = 0.5 * (FdHi[v] + FnHi[v]) - 0.5 * lamHi * (sHi[v] - tHi[v]);
    jLo[v] = fsLo - FdLo[v];
    jHi[v] = fsHi - FdHi[v];
  }
  // central common depth h* and its jump (sgn2d.cpp:213-214, 271-274)
  const double jhLo = 0.5 * (sLo[0] + tLo[0]) - tLo[0];
  const double jhHi = 0.5 * (tHi[0] + sHi[0]) - tHi[0];
#pragma unroll
  for (int m = 0; m < NP; ++m) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      if constexpr (EXACT) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) s += C.D[m * NP + k] * F[k][v];
        const double c = jLo[v] * C.gLp[m] + jHi[v] * C.gRp[m];
        out.d[m][v] = (s + c) / (DIR == 0 ? C.Jx : C.Jy);
      } else {
        // accumulate with the unscaled tables, one rounding for 1/J at the end
        double s = jLo[v] * C.gLp[m];
        s = fma(jHi[v], C.gRp[m], s);
#pragma unroll
        for (int k = 0; k < NP; ++k) s = fma(C.D[m * NP + k], F[k][v], s);
        out.d[m][v] = s * (DIR == 0 ? C.iJx : C.iJy);
      }
    }
    if constexpr (EXACT) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < NP; ++k) s += C.D[m * NP + k] * Un[k][0];
      s += jhLo * C.gLp[m] + jhHi * C.gRp[m];
      out.dh[m] = s / (DIR == 0 ? C.Jx : C.Jy);
    } else {
      double s = jhLo * C.gLp[m];
      s = fma(jhHi, C.gRp[m], s);
#pragma unroll
      for (int k = 0; k < NP; ++k) s = fma(C.D[m * NP + k], Un[k][0], s);
      out.dh[m] = s * (DIR == 0 ? C.iJx : C.iJy);
    }
  }
}

// Mirror ghost across a wall normal to DIR: the normal discharge changes sign.
template <int DIR>
__device__ __forceinline__ void mirror(const double* own, double* ghost) {
#pragma unroll
  for (int v = 0; v < NV; ++v) ghost[v] = own[v];
  ghost[DIR == 0 ? 1 : 2] = -own[DIR == 0 ? 1 : 2];
}

__device__ __forceinline__ bool spin_ok(long long& n) { return ++n < (1ll << 40); }

template <int MODE, bool EXACT>
__global__ void __launch_bounds__(NTHR, 2) k_fused(const RhsConsts C, const StageArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem& S = *reinterpret_cast<Smem*>(smem_raw);

  // ---- controller state (stage modes only) ---------------------------------
  int cur = 0;
  double dt = 0.0, acoef = 0.0, atol = 0.0, rtol = 0.0;
  if constexpr (MODE != MODE_RHS) {
    if (A.ctrl->done) return;  // uniform across the grid
    cur = A.ctrl->cur;
    dt = A.ctrl->dt;
    acoef = A.coef * dt;  // 0.5 * dt or 0.75 * dt as in rk.cpp:100-103
    atol = A.ctrl->atol;
    rtol = A.ctrl->rtol;
  }

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int Nx = C.Nx, Ny = C.Ny;
  const long long Nd = C.Nd;
  const int ex0 = blockIdx.x * TX, ey0 = blockIdx.y * TY;
  const int TXv = min(TX, Nx - ex0), TYv = min(TY, Ny - ey0);
  const bool wallL = C.bcx && ex0 == 0, wallR = C.bcx && ex0 + TXv == Nx;
  const bool wallB = C.bcy && ey0 == 0, wallT = C.bcy && ey0 + TYv == Ny;

  // ---- load phase: tile state, statics and halos into shared memory --------
  {
    double* dstU = &S.U[0][0][0];
    double* dstH = &S.H[0][0];
    // own nodes: per field and tile row, TXv*25 contiguous doubles
    for (int it = tid; it < NV * TY * TX * NPP; it += NTHR) {
      const int k = it % (TX * NPP);
      const int r = it / (TX * NPP);
      const int iy = r % TY, v = r / TY;
      if (iy >= TYv || k >= TXv * NPP) continue;
      const long long eg = (long long)ex0 + (long long)Nx * (ey0 + iy);
      const long long gi = (long long)v * Nd + eg * NPP + k;
      const double val = stage_value<MODE>(A, cur, dt, acoef, gi);
      dstU[(v * TE + iy * TX) * NPP + k] = val;
      if constexpr (MODE == MODE_FSAL) A.U[cur ^ 1][gi] = val;
    }
    for (int it = tid; it < 3 * TY * TX * NPP; it += NTHR) {
      const int k = it % (TX * NPP);
      const int r = it / (TX * NPP);
      const int iy = r % TY, s = r / TY;
      if (iy >= TYv || k >= TXv * NPP) continue;
      const long long eg = (long long)ex0 + (long long)Nx * (ey0 + iy);
      const double* src = s == 0 ? C.Hnod : (s == 1 ? C.Hx : C.Hy);
      dstH[(s * TE + iy * TX) * NPP + k] = src[eg * NPP + k];
    }
    // halos: left/right nodes per tile row, bottom/top nodes per tile column
    for (int it = tid; it < NV * (2 * TY + 2 * TX) * NP; it += NTHR) {
      const int t = it % NP;
      const int r = it / NP;
      const int slot = r % (2 * TY + 2 * TX), v = r / (2 * TY + 2 * TX);
      long long e;
      int node;
      double* dst;
      if (slot < TY) {  // left
        const int iy = slot;
        if (iy >= TYv || wallL) continue;
        e = (long long)((ex0 - 1 + Nx) % Nx) + (long long)Nx * (ey0 + iy);
        node = (NP - 1) + NP * t;
        dst = &S.haloL[v][iy][t];
      } else if (slot < 2 * TY) {  // right
        const int iy = slot - TY;
        if (iy >= TYv || wallR) continue;
        e = (long long)((ex0 + TXv) % Nx) + (long long)Nx * (ey0 + iy);
        node = NP * t;
        dst = &S.haloR[v][iy][t];
      } else if (slot < 2 * TY + TX) {  // bottom
        const int ix = slot - 2 * TY;
        if (ix >= TXv || wallB) continue;
        e = (long long)(ex0 + ix) + (long long)Nx * ((ey0 - 1 + Ny) % Ny);
        node = t + NP * (NP - 1);
        dst = &S.haloB[v][ix][t];
      } else {  // top
        const int ix = slot - 2 * TY - TX;
        if (ix >= TXv || wallT) continue;
        e = (long long)(ex0 + ix) + (long long)Nx * ((ey0 + TYv) % Ny);
        node = t;
        dst = &S.haloT[v][ix][t];
      }
      *dst = stage_value<MODE>(A, cur, dt, acoef, (long long)v * Nd + e * NPP + node);
    }
    // face depths
    for (int it = tid; it < 2 * TE * NP + (TY + TX) * NP; it += NTHR) {
      if (it < 2 * TE * NP) {
        const int t = it % NP, i = (it / NP) % TE, s = it / (NP * TE);
        const int ix = i % TX, iy = i / TX;
        if (ix >= TXv || iy >= TYv) continue;
        const long long e = (long long)(ex0 + ix) + (long long)Nx * (ey0 + iy);
        if (s == 0) S.HfX[i][t] = C.HfX[e * NP + t];
        else S.HfY[i][t] = C.HfY[e * NP + t];
      } else {
        const int r = it - 2 * TE * NP;
        const int t = r % NP, slot = r / NP;
        if (slot < TY) {
          const int iy = slot;
          if (iy >= TYv) continue;
          const int ey = ey0 + iy;
          S.HfXR[iy][t] = wallR ? C.HfXEnd[(long long)ey * NP + t]
                                : C.HfX[((long long)((ex0 + TXv) % Nx) + (long long)Nx * ey) * NP + t];
        } else {
          const int ix = slot - TY;
          if (ix >= TXv) continue;
          const int ex = ex0 + ix;
          S.HfYT[ix][t] = wallT ? C.HfYEnd[(long long)ex * NP + t]
                                : C.HfY[((long long)ex + (long long)Nx * ((ey0 + TYv) % Ny)) * NP + t];
        }
      }
    }
  }
  __syncthreads();

  const int i = lane;  // tile element of this lane
  const int ix = i % TX, iy = i / TX;
  const bool valid = ix < TXv && iy < TYv;
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
      for (int v = 0; v < NV; ++v) nLo[v] = S.U[v][i - TX][j + NP * (NP - 1)];
    } else if (wallB) {
      mirror<1>(Un[0], nLo);
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) nLo[v] = S.haloB[v][ix][j];
    }
    if (iy + 1 < TYv) {
#pragma unroll
      for (int v = 0; v < NV; ++v) nHi[v] = S.U[v][i + TX][j];
    } else if (wallT) {
      mirror<1>(Un[NP - 1], nHi);
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) nHi[v] = S.haloT[v][ix][j];
    }
    const double HfLo = S.HfY[i][j];
    const double HfHi = (iy + 1 < TYv) ? S.HfY[i + TX][j] : S.HfYT[ix][j];
    LineOut lo;
    line_pass<EXACT, 1>(C, Un, Hn, nLo, nHi, HfLo, HfHi, lo);
#pragma unroll
    for (int b = 0; b < NP; ++b) {
      const int loc = j + NP * b;
#pragma unroll
      for (int v = 0; v < NV; ++v) S.G[v][i][loc] = lo.d[b][v];
      // ncpY (sgn_flux2d.h:156-161): -c^2 v h_y
      double vv;
      if constexpr (EXACT) vv = Un[b][2] / Un[b][0]; else vv = Un[b][2] * (1.0 / Un[b][0]);
      const double hy = lo.dh[b];
      S.G[NV][i][loc] = EXACT ? C.mc2 * vv * hy : C.mc2 * vv * hy;
    }
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
      for (int v = 0; v < NV; ++v) nLo[v] = S.U[v][i - 1][(NP - 1) + NP * j];
    } else if (wallL) {
      mirror<0>(Un[0], nLo);
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) nLo[v] = S.haloL[v][iy][j];
    }
    if (ix + 1 < TXv) {
#pragma unroll
      for (int v = 0; v < NV; ++v) nHi[v] = S.U[v][i + 1][NP * j];
    } else if (wallR) {
      mirror<0>(Un[NP - 1], nHi);
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) nHi[v] = S.haloR[v][iy][j];
    }
    const double HfLo = S.HfX[i][j];
    const double HfHi = (ix + 1 < TXv) ? S.HfX[i + 1][j] : S.HfXR[iy][j];
    LineOut lo;
    line_pass<EXACT, 0>(C, Un, Hn, nLo, nHi, HfLo, HfHi, lo);
#pragma unroll
    for (int a = 0; a < NP; ++a) {
      const int loc = a + NP * j;
      const double* Uq = Un[a];
      const Prim<EXACT> q(Uq);
      const double Hl = Hn[a], Hxl = S.Hx[i][loc], Hyl = S.Hy[i][loc];
      // source (sgn_flux2d.h:122-134), Manning off
      const double bath = C.g * (Uq[0] - Hl) + C.gamma * q.p;
      const double S1 = bath * Hxl, S2 = bath * Hyl, S3 = C.gamma * q.p;
      const double S4 = C.m2c2 * (q.w + q.u * Hxl + q.v * Hyl);
      // ncpX (sgn_flux2d.h:150-155)
      const double Bx = C.mc2 * q.u * lo.dh[a];
      const double By = S.G[NV][i][loc];
      const double g0 = S.G[0][i][loc], g1 = S.G[1][i][loc], g2 = S.G[2][i][loc];
      const double g3 = S.G[3][i][loc], g4 = S.G[4][i][loc];
      // dU = -dF - dG - Bx - By + S (sgn2d.cpp:285-287); Bx, By vanish except in hp
      if constexpr (EXACT) {
        S.G[0][i][loc] = (-lo.d[a][0] - g0) + 0.0;
        S.G[1][i][loc] = (-lo.d[a][1] - g1) + S1;
        S.G[2][i][loc] = (-lo.d[a][2] - g2) + S2;
        S.G[3][i][loc] = (-lo.d[a][3] - g3) + S3;
        S.G[4][i][loc] = (((-lo.d[a][4] - g4) - Bx) - By) + S4;
      } else {
        S.G[0][i][loc] = -(lo.d[a][0] + g0);
        S.G[1][i][loc] = S1 - (lo.d[a][1] + g1);
        S.G[2][i][loc] = S2 - (lo.d[a][2] + g2);
        S.G[3][i][loc] = S3 - (lo.d[a][3] + g3);
        S.G[4][i][loc] = S4 - (lo.d[a][4] + g4) - Bx - By;
      }
    }
  }
  __syncthreads();

  // ---- copy-out (and the embedded error of the FSAL stage) ------------------
  double esum = 0.0, emax = 0.0;
  int enan = 0;
  {
    const double* srcU = &S.G[0][0][0];
    double* outp;
    if constexpr (MODE == MODE_RHS || MODE == MODE_STAGE) outp = A.out;
    else outp = A.K1[cur ^ 1];
    for (int it = tid; it < NV * TY * TX * NPP; it += NTHR) {
      const int k = it % (TX * NPP);
      const int r = it / (TX * NPP);
      const int iy2 = r % TY, v = r / TY;
      if (iy2 >= TYv || k >= TXv * NPP) continue;
      const long long eg = (long long)ex0 + (long long)Nx * (ey0 + iy2);
      const long long gi = (long long)v * Nd + eg * NPP + k;
      const double val = srcU[(v * TE + iy2 * TX) * NPP + k];
      outp[gi] = val;
      if constexpr (MODE == MODE_FSAL) {
        // scaled embedded error, src/solver/rk.cpp:118-128
        const double u = A.U[cur][gi], k1 = A.K1[cur][gi], k2 = A.K2[gi], k3 = A.K3[gi];
        const double un = u + dt * (2.0 / 9.0 * k1 + 1.0 / 3.0 * k2 + 4.0 / 9.0 * k3);
        const double uEmb = u + dt * (7.0 / 24.0 * k1 + 0.25 * k2 + 1.0 / 3.0 * k3 + 0.125 * val);
        const double e = un - uEmb;
        const double au = fabs(u), an = fabs(un);
        const double sc = atol + rtol * (au < an ? an : au);
        const double rr = e / sc;
        esum += rr * rr;
        const double ar = fabs(rr);
        emax = emax < ar ? ar : emax;
        enan |= (rr != rr);
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
      const long long blk = (long long)blockIdx.y * gridDim.x + blockIdx.x;
      A.partials[3 * blk + 0] = s;
      A.partials[3 * blk + 1] = m;
      A.partials[3 * blk + 2] = n;
    }
  }
}

}  // namespace dev
}  // namespace sgnb
