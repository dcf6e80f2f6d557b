// sgnb_adjoint.cu -- vector-Jacobian products of the right-hand side and of the BS3(2)
// update (no reference counterpart: the reference has no adjoint).
//
// R(U; H) is the FR discretisation of src/solver/sgn2d.cpp:125-290 as the fused kernels
// compute it (sgnb_kernels.cuh, line_pass and the assembly of the row pass): for every
// element and every GLL line in x and in y,
//   nodal fluxes F_k = flux(U_k, H_k)                       (sgn_flux2d.h:89-116)
//   face fluxes: Rusanov with lam = max(ws(s), ws(t))      (sgn_flux2d.h:169-179)
//   j = F* - F(own trace), dF_m = (sum_k D[m,k] F_k + jLo gL'[m] + jHi gR'[m]) / J
//   dh_m likewise with the central common depth            (sgn2d.cpp:265-275)
//   R -= dF; R[hp] -= -c^2 u_n dh  (non-conservative term, sgn_flux2d.h:150-161)
// plus the pointwise sources (sgn_flux2d.h:122-142, Manning friction included). Given a
// cotangent Rb of R, the line kernel reverses one line (one thread per element line and
// direction) and writes:
//   * the cotangent of the line's own nodes, per direction (each node lies on exactly one
//     x line and one y line of its element, so these are plain stores);
//   * the cotangent of the neighbour's trace node across each face (a per-face buffer the
//     gather kernel adds to the neighbour's node) or, at a wall, folded back through the
//     mirror ghost onto the own trace;
//   * the cotangents of the depth statics: nodal H (fluxes and sources), the nodal dH/dx,
//     dH/dy (sources, x pass) and the face depths, per face side.
// The gather kernel (one thread per node) sums the two directions and the neighbours'
// face contributions in a fixed order, so the result is deterministic without atomics,
// and folds in the RK-stage combination. Built with -fmad=true like the fast forward.
#include "sgnb_checked.cuh"
#include "sgnb_device.h"

namespace sgnb {
namespace dev {
namespace {

constexpr int NP = 5, NPP = 25, NV = 5;

struct LineIn {
  double U[NP][NV];  // stage input y at the line's nodes
  double H[NP];
};

__device__ __forceinline__ double stage_in(const VjpArgs& A, long long idx) {
  // y = u or u + (c dt) k, with the forward's rounding (stage_axpy of the fused kernels)
  return A.k ? __dadd_rn(A.u[idx], __dmul_rn(A.acoef, A.k[idx])) : A.u[idx];
}

__device__ __forceinline__ double sgn0(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0); }

// Cotangent of the primitive variables (u, v, w, p) = (hu, hv, hw, hp) / h at a point,
// added to the conserved cotangent Ub.
__device__ __forceinline__ void prim_back(const double* U, double ub, double vb, double wb,
                                          double pb, double* Ub) {
  const double ih = 1.0 / U[0];
  const double u = U[1] * ih, v = U[2] * ih, w = U[3] * ih, p = U[4] * ih;
  Ub[1] += ub * ih;
  Ub[2] += vb * ih;
  Ub[3] += wb * ih;
  Ub[4] += pb * ih;
  Ub[0] -= (ub * u + vb * v + wb * w + pb * p) * ih;
}

// Reverse of the directional flux F = flux_DIR(U, H): adds to Ub, returns dH.
template <int DIR>
__device__ __forceinline__ double flux_back(const RhsConsts& C, const double* U, double H,
                                            const double* Fb, double* Ub) {
  constexpr int nd = 1 + DIR, td = 2 - DIR;
  const double ih = 1.0 / U[0];
  const double hn = U[nd];
  const double n = hn * ih, t = U[td] * ih, w = U[3] * ih, p = U[4] * ih;
  // F0 = hn, F[nd] = hn n + g/2 (h^2 - H^2) + hp, F[td] = hn t, F3 = hn w, F4 = hn (p + c^2)
  const double hnb = Fb[0] + Fb[nd] * n + Fb[td] * t + Fb[3] * w + Fb[4] * (p + C.c2);
  const double nb = Fb[nd] * hn, tb = Fb[td] * hn, wb = Fb[3] * hn, pb = Fb[4] * hn;
  Ub[0] += Fb[nd] * C.g * U[0];
  Ub[4] += Fb[nd];
  Ub[nd] += hnb;
  double q[4] = {0.0, 0.0, wb, pb};
  q[nd - 1] = nb;
  q[td - 1] = tb;
  prim_back(U, q[0], q[1], q[2], q[3], Ub);
  return -Fb[nd] * C.g * H;
}

// Wave speed ws = |u_n| + sqrt(max(g h + p + c^2, 0)) (sgn_flux2d.h:73-86).
template <int DIR>
__device__ __forceinline__ double wave_speed(const RhsConsts& C, const double* U) {
  const double ih = 1.0 / U[0];
  const double arg = C.g * U[0] + U[4] * ih + C.c2;
  return fabs(U[1 + DIR] * ih) + sqrt(arg > 0.0 ? arg : 0.0);
}

template <int DIR>
__device__ __forceinline__ void wave_speed_back(const RhsConsts& C, const double* U,
                                                double lb, double* Ub) {
  const double ih = 1.0 / U[0];
  const double un = U[1 + DIR] * ih;
  const double arg = C.g * U[0] + U[4] * ih + C.c2;
  const double unb = sgn0(un) * lb;  // |x|' = sign(x), 0 at 0 (the central difference)
  double ab = 0.0;
  if (arg > 0.0) ab = 0.5 * lb / sqrt(arg);
  Ub[0] += C.g * ab;
  double q[4] = {0.0, 0.0, 0.0, ab};
  q[DIR] = unb;
  prim_back(U, q[0], q[1], q[2], q[3], Ub);
}

// One line: reverse of its contribution to R (see the file comment).
template <int DIR>
__global__ void __launch_bounds__(128) k_vjp_lines(const RhsConsts C, const FrTablesDev T,
                                                   const VjpArgs A) {
  const long long ne = (long long)C.Nx * C.Ny;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= ne * NP) return;
  const long long e = idx / NP;
  const int j = (int)(idx - e * NP);
  const int ex = (int)(e % C.Nx), ey = (int)(e / C.Nx);
  const long long Nd = C.Nd;
  constexpr int nd = 1 + DIR;
  auto node = [&](int m) -> long long {
    return e * NPP + (DIR == 0 ? m + NP * j : j + NP * m);
  };
  const double iJ = DIR == 0 ? C.iJx : C.iJy;

  // ---- forward quantities of the line ---------------------------------------------
  LineIn L;
  double Rb[NP][NV];
#pragma unroll
  for (int m = 0; m < NP; ++m) {
    const long long g = node(m);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const bool ok = SGNB_INB(v * Nd + g, NV * Nd);
      L.U[m][v] = ok ? stage_in(A, v * Nd + g) : 0.0;
      double r = ok ? A.alpha * A.ra[v * Nd + g] : 0.0;
      if (A.rb && ok) r += A.beta * A.rb[v * Nd + g];
      Rb[m][v] = r;
    }
    L.H[m] = SGNB_INB(g, Nd) ? C.Hnod[g] : 0.0;
  }
  bool wallLo, wallHi;
  long long nLo, nHi;  // neighbour trace nodes
  double HfLo, HfHi;
  if (DIR == 0) {
    wallLo = C.bcx && ex == 0;
    wallHi = C.bcx && ex == C.Nx - 1;
    const long long eL = (long long)((ex - 1 + C.Nx) % C.Nx) + (long long)C.Nx * ey;
    const long long eR = (long long)((ex + 1) % C.Nx) + (long long)C.Nx * ey;
    nLo = eL * NPP + (NP - 1) + NP * j;
    nHi = eR * NPP + NP * j;
    HfLo = SGNB_INB(e * NP + j, ne * NP) ? C.HfX[e * NP + j] : 0.0;
    HfHi = SGNB_INB(wallHi ? (long long)ey * NP + j : eR * NP + j, wallHi ? (long long)C.Ny * NP : ne * NP)
               ? (wallHi ? C.HfXEnd[(long long)ey * NP + j] : C.HfX[eR * NP + j]) : 0.0;
  } else {
    wallLo = C.bcy && ey == 0;
    wallHi = C.bcy && ey == C.Ny - 1;
    const long long eB = (long long)ex + (long long)C.Nx * ((ey - 1 + C.Ny) % C.Ny);
    const long long eT = (long long)ex + (long long)C.Nx * ((ey + 1) % C.Ny);
    nLo = eB * NPP + j + NP * (NP - 1);
    nHi = eT * NPP + j;
    HfLo = SGNB_INB(e * NP + j, ne * NP) ? C.HfY[e * NP + j] : 0.0;
    HfHi = SGNB_INB(wallHi ? (long long)ex * NP + j : eT * NP + j, wallHi ? (long long)C.Nx * NP : ne * NP)
               ? (wallHi ? C.HfYEnd[(long long)ex * NP + j] : C.HfY[eT * NP + j]) : 0.0;
  }
  double sLo[NV], sHi[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    sLo[v] = wallLo ? (v == nd ? -L.U[0][v] : L.U[0][v])
                    : (SGNB_INB(v * Nd + nLo, NV * Nd) ? stage_in(A, v * Nd + nLo) : 0.0);
    sHi[v] = wallHi ? (v == nd ? -L.U[NP - 1][v] : L.U[NP - 1][v])
                    : (SGNB_INB(v * Nd + nHi, NV * Nd) ? stage_in(A, v * Nd + nHi) : 0.0);
  }
  const double* tLo = L.U[0];
  const double* tHi = L.U[NP - 1];
  const double jhLo = 0.5 * (sLo[0] + tLo[0]) - tLo[0];
  const double jhHi = 0.5 * (tHi[0] + sHi[0]) - tHi[0];

  double Ub[NP][NV];
  double Hb[NP];
#pragma unroll
  for (int m = 0; m < NP; ++m) {
    Hb[m] = 0.0;
#pragma unroll
    for (int v = 0; v < NV; ++v) Ub[m][v] = 0.0;
  }
  double sLb[NV], sHb[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) { sLb[v] = 0.0; sHb[v] = 0.0; }
  double HfLb = 0.0, HfHb = 0.0;

  // ---- non-conservative term B_m = -c^2 u_n dh_m, R[hp] -= B_m -----------------------
  {
    double dhb[NP];
#pragma unroll
    for (int m = 0; m < NP; ++m) {
      double s = jhLo * T.gLp[m] + jhHi * T.gRp[m];
#pragma unroll
      for (int k = 0; k < NP; ++k) s += T.D[m * NP + k] * L.U[k][0];
      const double dh = s * iJ;
      const double Bb = -Rb[m][4];
      const double un = L.U[m][nd] / L.U[m][0];
      dhb[m] = C.mc2 * un * Bb;
      double q[4] = {0.0, 0.0, 0.0, 0.0};
      q[DIR] = C.mc2 * dh * Bb;
      prim_back(L.U[m], q[0], q[1], q[2], q[3], Ub[m]);
    }
    double jhLb = 0.0, jhHb = 0.0;
#pragma unroll
    for (int m = 0; m < NP; ++m) {
      jhLb += T.gLp[m] * dhb[m];
      jhHb += T.gRp[m] * dhb[m];
    }
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      double s = 0.0;
#pragma unroll
      for (int m = 0; m < NP; ++m) s += T.D[m * NP + k] * dhb[m];
      Ub[k][0] += s * iJ;
    }
    jhLb *= iJ;
    jhHb *= iJ;
    sLb[0] += 0.5 * jhLb;
    Ub[0][0] -= 0.5 * jhLb;
    sHb[0] += 0.5 * jhHb;
    Ub[NP - 1][0] -= 0.5 * jhHb;
  }

  // ---- flux divergence: dF_m = (D F + jLo gL' + jHi gR') / J, R -= dF ----------------
  double jLb[NV], jHb[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double a = 0.0, b = 0.0;
#pragma unroll
    for (int m = 0; m < NP; ++m) {
      a -= T.gLp[m] * Rb[m][v];
      b -= T.gRp[m] * Rb[m][v];
    }
    jLb[v] = a * iJ;
    jHb[v] = b * iJ;
  }
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    double Fb[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double s = 0.0;
#pragma unroll
      for (int m = 0; m < NP; ++m) s -= T.D[m * NP + k] * Rb[m][v];
      Fb[v] = s * iJ;
    }
    Hb[k] += flux_back<DIR>(C, L.U[k], L.H[k], Fb, Ub[k]);
  }

  // ---- faces: j = F* - F(t), Rusanov F* (low face: neighbour on the left) ------------
  {
    // low face: j = 1/2 Fn - 1/2 Fd - 1/2 lam (t - s)
    const double wsS = wave_speed<DIR>(C, sLo), wsT = wave_speed<DIR>(C, tLo);
    const double lam = fmax(wsS, wsT);
    double Fnb[NV], Fdb[NV], lb = 0.0;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      Fnb[v] = 0.5 * jLb[v];
      Fdb[v] = -0.5 * jLb[v];
      lb -= 0.5 * jLb[v] * (tLo[v] - sLo[v]);
      Ub[0][v] -= 0.5 * lam * jLb[v];
      sLb[v] += 0.5 * lam * jLb[v];
    }
    HfLb += flux_back<DIR>(C, tLo, HfLo, Fdb, Ub[0]);
    HfLb += flux_back<DIR>(C, sLo, HfLo, Fnb, sLb);
    if (wsS >= wsT) wave_speed_back<DIR>(C, sLo, lb, sLb);
    else wave_speed_back<DIR>(C, tLo, lb, Ub[0]);
  }
  {
    // high face: j = 1/2 Fn - 1/2 Fd - 1/2 lam (s - t)
    const double wsT = wave_speed<DIR>(C, tHi), wsS = wave_speed<DIR>(C, sHi);
    const double lam = fmax(wsT, wsS);
    double Fnb[NV], Fdb[NV], lb = 0.0;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      Fnb[v] = 0.5 * jHb[v];
      Fdb[v] = -0.5 * jHb[v];
      lb -= 0.5 * jHb[v] * (sHi[v] - tHi[v]);
      sHb[v] -= 0.5 * lam * jHb[v];
      Ub[NP - 1][v] += 0.5 * lam * jHb[v];
    }
    HfHb += flux_back<DIR>(C, tHi, HfHi, Fdb, Ub[NP - 1]);
    HfHb += flux_back<DIR>(C, sHi, HfHi, Fnb, sHb);
    if (wsT >= wsS) wave_speed_back<DIR>(C, tHi, lb, Ub[NP - 1]);
    else wave_speed_back<DIR>(C, sHi, lb, sHb);
  }

  // ---- sources (x pass only; pointwise, sgn_flux2d.h:122-134) --------------------------
  if (DIR == 0) {
#pragma unroll
    for (int m = 0; m < NP; ++m) {
      const long long g = node(m);
      const double* U = L.U[m];
      if (!SGNB_INB(g, Nd)) continue;
      const double Hx = C.Hx[g], Hy = C.Hy[g];
      const double ih = 1.0 / U[0];
      const double u = U[1] * ih, v = U[2] * ih, p = U[4] * ih;
      const double r1 = Rb[m][1], r2 = Rb[m][2], r3 = Rb[m][3], r4 = Rb[m][4];
      const double bath = C.g * (U[0] - L.H[m]) + C.gamma * p;
      const double sHr = Hx * r1 + Hy * r2;
      Ub[m][0] += C.g * sHr;
      Hb[m] -= C.g * sHr;
      A.Hxb[g] = bath * r1 + C.m2c2 * u * r4;
      A.Hyb[g] = bath * r2 + C.m2c2 * v * r4;
      double ub = C.m2c2 * Hx * r4, vb = C.m2c2 * Hy * r4;
      if (C.manning) {
        // friction (-cf u, -cf v), cf = n^2 g |vel| h^(-1/3)
        const double vm = sqrt(u * u + v * v);
        const double kc = C.n2g / cbrt(U[0]);
        const double cf = kc * vm;
        const double ruv = r1 * u + r2 * v;
        ub -= r1 * cf;
        vb -= r2 * cf;
        if (vm > 0.0) {
          ub -= kc * ruv * u / vm;
          vb -= kc * ruv * v / vm;
        }
        Ub[m][0] += ruv * cf / (3.0 * U[0]);  // d/dh of h^(-1/3)
      }
      prim_back(U, ub, vb, C.m2c2 * r4, C.gamma * sHr + C.gamma * r3, Ub[m]);
    }
  }

  // ---- mirror ghosts fold back onto the own trace ------------------------------------
  if (wallLo) {
#pragma unroll
    for (int v = 0; v < NV; ++v) Ub[0][v] += v == nd ? -sLb[v] : sLb[v];
  } else {
    double* o = A.Sn[DIR][0] + idx * NV;
#pragma unroll
    for (int v = 0; v < NV; ++v)
      if (SGNB_INB(idx * NV + v, ne * NP * NV)) o[v] = sLb[v];
  }
  if (wallHi) {
#pragma unroll
    for (int v = 0; v < NV; ++v) Ub[NP - 1][v] += v == nd ? -sHb[v] : sHb[v];
  } else {
    double* o = A.Sn[DIR][1] + idx * NV;
#pragma unroll
    for (int v = 0; v < NV; ++v)
      if (SGNB_INB(idx * NV + v, ne * NP * NV)) o[v] = sHb[v];
  }
  if (SGNB_INB(idx, ne * NP)) {
    A.Hf[DIR][0][idx] = HfLb;
    A.Hf[DIR][1][idx] = HfHb;
  }
#pragma unroll
  for (int m = 0; m < NP; ++m) {
    const long long g = node(m);
    if (!SGNB_INB(g, Nd)) continue;
#pragma unroll
    for (int v = 0; v < NV; ++v) A.Ub[DIR][v * Nd + g] = Ub[m][v];
    A.Hb[DIR][g] = Hb[m];
  }
}

// One thread per node: the node's cotangent from both directions and from the
// neighbours' faces, the RK-stage combination, and the statics accumulators.
__global__ void __launch_bounds__(256) k_vjp_gather(const RhsConsts C, const VjpArgs A,
                                                    const GatherArgs G) {
  const long long Nd = C.Nd;
  const long long gnode = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gnode >= Nd) return;
  const long long e = gnode / NPP;
  const int loc = (int)(gnode - e * NPP);
  const int a = loc % NP, b = loc / NP;
  const int ex = (int)(e % C.Nx), ey = (int)(e / C.Nx);
  const long long eL = (long long)((ex - 1 + C.Nx) % C.Nx) + (long long)C.Nx * ey;
  const long long eR = (long long)((ex + 1) % C.Nx) + (long long)C.Nx * ey;
  const long long eB = (long long)ex + (long long)C.Nx * ((ey - 1 + C.Ny) % C.Ny);
  const long long eT = (long long)ex + (long long)C.Nx * ((ey + 1) % C.Ny);
  const bool wL = C.bcx && ex == 0, wR = C.bcx && ex == C.Nx - 1;
  const bool wB = C.bcy && ey == 0, wT = C.bcy && ey == C.Ny - 1;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const long long g = v * Nd + gnode;
    double y = A.Ub[0][g] + A.Ub[1][g];
    // line index of a face entry: (element * 5 + line) * 5 + v
    [[maybe_unused]] const long long nl = (long long)C.Nx * C.Ny * NP * NV;
    if (a == 0 && !wL && SGNB_INB((eL * NP + b) * NV + v, nl)) y += A.Sn[0][1][(eL * NP + b) * NV + v];
    if (a == NP - 1 && !wR && SGNB_INB((eR * NP + b) * NV + v, nl)) y += A.Sn[0][0][(eR * NP + b) * NV + v];
    if (b == 0 && !wB && SGNB_INB((eB * NP + a) * NV + v, nl)) y += A.Sn[1][1][(eB * NP + a) * NV + v];
    if (b == NP - 1 && !wT && SGNB_INB((eT * NP + a) * NV + v, nl)) y += A.Sn[1][0][(eT * NP + a) * NV + v];
    if (G.ybar) G.ybar[g] = y;
    if (G.init) G.uacc[g] = (G.lam ? G.lam[g] : 0.0) + y;
    else G.uacc[g] += y;
  }
  G.Hacc[gnode] += A.Hb[0][gnode] + A.Hb[1][gnode];
  G.Hxacc[gnode] += A.Hxb[gnode];
  G.Hyacc[gnode] += A.Hyb[gnode];
  [[maybe_unused]] const long long nf = (long long)C.Nx * C.Ny * NP;
  if (a == 0 && SGNB_INB(e * NP + b, nf) && SGNB_INB(eL * NP + b, nf)) {
    double s = A.Hf[0][0][e * NP + b];
    if (!wL) s += A.Hf[0][1][eL * NP + b];
    G.HfXacc[e * NP + b] += s;
  }
  if (a == NP - 1 && wR && SGNB_INB((long long)ey * NP + b, (long long)C.Ny * NP) &&
      SGNB_INB(e * NP + b, nf))
    G.HfXEndacc[(long long)ey * NP + b] += A.Hf[0][1][e * NP + b];
  if (b == 0 && SGNB_INB(e * NP + a, nf) && SGNB_INB(eB * NP + a, nf)) {
    double s = A.Hf[1][0][e * NP + a];
    if (!wB) s += A.Hf[1][1][eB * NP + a];
    G.HfYacc[e * NP + a] += s;
  }
  if (b == NP - 1 && wT && SGNB_INB((long long)ex * NP + a, (long long)C.Nx * NP) &&
      SGNB_INB(e * NP + a, nf))
    G.HfYEndacc[(long long)ex * NP + a] += A.Hf[1][1][e * NP + a];
}

// u_new = u + dt ((2/9 k1 + 1/3 k2) + 4/9 k3) with the end-point stage's rounding
// (src/solver/rk.cpp:106-108).
__global__ void k_rk_update(const double* __restrict__ u, const double* __restrict__ k1,
                            const double* __restrict__ k2, const double* __restrict__ k3,
                            const double* __restrict__ dts, long long step,
                            double* __restrict__ out, long long n) {
  const double dt = dts[step];
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double part = __dadd_rn(__dmul_rn(2.0 / 9.0, k1[i]), __dmul_rn(1.0 / 3.0, k2[i]));
    out[i] = __dadd_rn(u[i], __dmul_rn(dt, __dadd_rn(part, __dmul_rn(4.0 / 9.0, k3[i]))));
  }
}

// eta at the gauges: eta[g] = h(node_g) - H(node_g)
__global__ void k_gauges(const double* __restrict__ U, const double* __restrict__ Hnod,
                         const long long* __restrict__ nodes, int ng, double* __restrict__ eta) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < ng) eta[g] = U[nodes[g]] - Hnod[nodes[g]];  // nodes checked on the host
}

// lam[h](node_g) += etab[g]
__global__ void k_gauges_back(double* __restrict__ lam, const long long* __restrict__ nodes,
                              int ng, const double* __restrict__ etab) {
  // gauges may share a node: one thread adds all of them, in order
  if (blockIdx.x == 0 && threadIdx.x == 0)
    for (int g = 0; g < ng; ++g) lam[nodes[g]] += etab[g];
}

}  // namespace

// The checked build's out-of-range count of the adjoint kernels (reset: then zero it);
// cudaErrorNotSupported in the normal build.
cudaError_t read_oob_adjoint(unsigned long long* out, bool reset) {
#ifdef SGNB_CHECKED
  cudaError_t e = cudaMemcpyFromSymbol(out, g_sgnb_oob, sizeof(*out));
  if (e == cudaSuccess && reset) {
    const unsigned long long z = 0;
    e = cudaMemcpyToSymbol(g_sgnb_oob, &z, sizeof(z));
  }
  return e;
#else
  *out = 0;
  (void)reset;
  return cudaErrorNotSupported;
#endif
}

cudaError_t launch_vjp_rhs(const RhsConsts& C, const FrTablesDev& T, const VjpArgs& A,
                           const GatherArgs& G, cudaStream_t s) {
  const long long lines = (long long)C.Nx * C.Ny * NP;
  const unsigned nb = (unsigned)((lines + 127) / 128);
  k_vjp_lines<0><<<nb, 128, 0, s>>>(C, T, A);
  k_vjp_lines<1><<<nb, 128, 0, s>>>(C, T, A);
  const unsigned ng = (unsigned)((C.Nd + 255) / 256);
  k_vjp_gather<<<ng, 256, 0, s>>>(C, A, G);
  return cudaGetLastError();
}

cudaError_t launch_rk_update(const double* u, const double* k1, const double* k2,
                             const double* k3, const double* dts, long long step, double* out,
                             long long n, cudaStream_t s) {
  k_rk_update<<<4 * 148, 256, 0, s>>>(u, k1, k2, k3, dts, step, out, n);
  return cudaGetLastError();
}

cudaError_t launch_gauges(const double* U, const double* Hnod, const long long* nodes, int ng,
                          double* eta, cudaStream_t s) {
  k_gauges<<<(ng + 127) / 128, 128, 0, s>>>(U, Hnod, nodes, ng, eta);
  return cudaGetLastError();
}

cudaError_t launch_gauges_back(double* lam, const long long* nodes, int ng, const double* etab,
                               cudaStream_t s) {
  k_gauges_back<<<1, 32, 0, s>>>(lam, nodes, ng, etab);
  return cudaGetLastError();
}

}  // namespace dev
}  // namespace sgnb
