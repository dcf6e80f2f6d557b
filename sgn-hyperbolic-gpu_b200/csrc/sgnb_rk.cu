// sgnb_rk.cu -- device-side controller of the adaptive Bogacki-Shampine 3(2) loop and
// the diagnostic reductions. Built with -fmad=false: the controller arithmetic follows
// src/solver/rk.cpp:112-161 operation for operation.
#include "sgnb_device.h"

#include <cmath>

namespace sgnb {
namespace dev {

namespace {

constexpr int kCtrlThreads = 256;

__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }  // std::max
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }  // std::min

// One adaptive attempt has just written its per-CTA error partials. Reduce them in a
// fixed order (so reruns are bit-reproducible), then apply the reference controller:
// accept if the RMS scaled error <= 1 (rk.cpp:129-142), PI update clamped to
// [facMin, facMax] (:148-152), dtMin abort (:155-160), and the loop test and the
// end-time clip of the next attempt (:95-97).
// row(b): the three partials (sum r^2, max |r|, NaN count) of error block b.
template <class Row>
__device__ __forceinline__ void controller_core(CtrlState* c, const Row& row, long long nblk,
                                                long long n) {
  __shared__ double ss[kCtrlThreads], sm[kCtrlThreads], sn[kCtrlThreads];
  if (c->done) return;
  const int t = threadIdx.x;
  double s = 0.0, m = 0.0, nn = 0.0;
  // rows b = t, t + T, t + 2T, ... in this order; eight rows' loads are issued before
  // they are summed, so the walk takes one memory latency per eight rows
  constexpr int kAhead = 8;
  long long b = t;
  for (; b + (kAhead - 1) * kCtrlThreads < nblk; b += kAhead * kCtrlThreads) {
    double r0[kAhead], r1[kAhead], r2[kAhead];
#pragma unroll
    for (int k = 0; k < kAhead; ++k) {
      const double* r = row(b + k * kCtrlThreads);
      r0[k] = r[0];
      r1[k] = r[1];
      r2[k] = r[2];
    }
#pragma unroll
    for (int k = 0; k < kAhead; ++k) {
      s += r0[k];
      m = dmax(m, r1[k]);
      nn += r2[k];
    }
  }
  for (; b < nblk; b += kCtrlThreads) {
    const double* r = row(b);
    s += r[0];
    m = dmax(m, r[1]);
    nn += r[2];
  }
  ss[t] = s;
  sm[t] = m;
  sn[t] = nn;
  __syncthreads();
  for (int off = kCtrlThreads / 2; off > 0; off >>= 1) {
    if (t < off) {
      ss[t] += ss[t + off];
      sm[t] = dmax(sm[t], sm[t + off]);
      sn[t] += sn[t + off];
    }
    __syncthreads();
  }
  if (t != 0) return;
  const double errL2 = sqrt(ss[0] / (double)n);
  const double errMax = sm[0];
  const double errNorm = dmax(errL2, 1e-300);
  const bool bad = (sn[0] > 0.0) || (errNorm != errNorm);
  if (c->log && c->attempts < c->logCap) {
    double* row = c->log + 4 * c->attempts;
    row[0] = c->t;
    row[1] = c->dt;
    row[2] = errNorm;
    row[3] = (c->frozen || errNorm <= 1.0) ? 1.0 : 0.0;
  }
  c->attempts += 1;
  c->rhsEvals += 3;
  c->errLast = errNorm;
  if (c->frozen) {  // replay of a given dt sequence: every step is taken
    c->t += c->dt;
    c->cur ^= 1;
    c->accepted += 1;
    c->tReached = c->t;
    c->dtLast = c->dt;
    c->maxNormLast = errMax;
    if (bad) { c->done = 3; return; }
    if (c->accepted >= c->nList) { c->done = 1; return; }
    c->dt = c->dtList[c->accepted];
    return;
  }
  bool stop = false;
  if (errNorm <= 1.0) {
    c->t += c->dt;
    c->cur ^= 1;  // uNew becomes u and k4 becomes k1 (FSAL)
    c->accepted += 1;
    c->tReached = c->t;
    c->dtLast = c->dt;
    c->maxNormLast = errMax;
    c->errPrev = errNorm;
    stop = c->maxAccepted > 0 && c->accepted >= c->maxAccepted;
  } else {
    c->rejected += 1;
  }
  if (bad) { c->done = 3; return; }  // the reference would loop forever here
  double fac = c->safety * pow(errNorm, -c->alpha) * pow(c->errPrev, c->beta);
  fac = (fac < c->facMin) ? c->facMin : ((c->facMax < fac) ? c->facMax : fac);
  double dtNext = c->dt * fac;
  dtNext = dmin(dtNext, c->dtMax);
  if (dtNext < c->dtMin) {
    c->done = 2;
    c->dtLast = dtNext;
    return;
  }
  c->dt = dtNext;
  if (stop) { c->done = 1; return; }  // fixed number of accepted steps reached
  const double tEnd = c->tEnd;
  if (!(c->t < tEnd - 1e-15 * dmax(1.0, fabs(tEnd)))) { c->done = 1; return; }
  if (c->t + c->dt > tEnd) c->dt = tEnd - c->t;
}

__device__ __forceinline__ void controller_block(CtrlState* c, const double* partials, int nblk,
                                                 long long n) {
  controller_core(c, [&](long long b) { return partials + 3 * b; }, nblk, n);
}

__global__ void __launch_bounds__(kCtrlThreads) k_controller(CtrlState* c, const double* partials,
                                                             int nblk, long long n) {
  controller_block(c, partials, nblk, n);
}

// The controller of the device-side loop: one attempt's decision, then the WHILE node's
// condition for the next pass of the body (one block; thread 0 wrote the state).
__global__ void __launch_bounds__(kCtrlThreads) k_controller_loop(CtrlState* c, const double* partials,
                                                                  int nblk, long long n,
                                                                  cudaGraphConditionalHandle loop) {
  controller_block(c, partials, nblk, n);
  if (threadIdx.x == 0)
    cudaGraphSetConditional(loop, (c->done == 0 && c->attempts < c->attemptCap) ? 1u : 0u);
}

__global__ void __launch_bounds__(kCtrlThreads) k_controller_batch_loop(
    CtrlState* ctrls, const double* const* partials, const int* nblk, const long long* n,
    int* counters, cudaGraphConditionalHandle loop) {
  const int i = blockIdx.x;
  CtrlState* c = ctrls + i;
  controller_block(c, partials[i], nblk[i], n[i]);
  if (threadIdx.x != 0) return;
  if (c->done == 0 && c->attempts < c->attemptCap) atomicAdd(&counters[0], 1);
  __threadfence();
  if (atomicAdd(&counters[1], 1) == (int)gridDim.x - 1) {  // the last block of this attempt
    __threadfence();
    const int running = atomicExch(&counters[0], 0);
    counters[1] = 0;
    cudaGraphSetConditional(loop, running > 0 ? 1u : 0u);
  }
}

// Slab controller: the error blocks of every slab of a decomposed mesh, read in place (on
// other devices: peer loads) in slab order, as one list.
__global__ void __launch_bounds__(kCtrlThreads) k_controller_slabs(CtrlState* c, const SlabPartials L,
                                                                   long long n) {
  controller_core(
      c,
      [&](long long b) {
        int s = 0;
        while (s + 1 < L.ns && b >= L.start[s + 1]) ++s;
        return L.p[s] + 3 * (b - L.start[s]);
      },
      L.start[L.ns], n);
}

// Batched controller: block i runs instance i's controller on its own partials.
__global__ void __launch_bounds__(kCtrlThreads) k_controller_batch(CtrlState* ctrls,
                                                                   const double* const* partials,
                                                                   const int* nblk, const long long* n) {
  const int i = blockIdx.x;
  controller_block(ctrls + i, partials[i], nblk[i], n[i]);
}

struct QW {
  double w[5];
};

// Per-block reductions over the nodes of a state: what = 0 largest characteristic
// speed (SGN2D::maxWaveSpeed, src/solver/sgn2d.cpp:295-305), 1 mass (:319-329),
// 2 energy (:334-348). Each block writes one partial; the host combines them.
__global__ void __launch_bounds__(256) k_diag(int what, const RhsConsts C, const double* U,
                                              const QW q, double* out) {
  __shared__ double sh[256];
  const long long Nd = C.Nd;
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < Nd;
       i += (long long)gridDim.x * blockDim.x) {
    const double h = U[i];  // the mass reads h alone
    const int loc = (int)(i % 25);
    const double wq = q.w[loc % 5] * q.w[loc / 5];
    if (what == 0) {
      const double hu = U[Nd + i], hv = U[2 * Nd + i];
      const double p = U[4 * Nd + i] / h;
      const double arg = C.g * h + p + C.c2;
      const double ce = sqrt(arg > 0.0 ? arg : 0.0);
      const double lx = fabs(hu / h) + ce, ly = fabs(hv / h) + ce;
      acc = fmax(acc, fmax(lx, ly));
    } else if (what == 1) {
      acc += wq * h;
    } else {
      const double u = U[Nd + i] / h, v = U[2 * Nd + i] / h, w = U[3 * Nd + i] / h;
      const double e = 0.5 * h * (u * u + v * v + (1.0 / C.gamma) * w * w +
                                  C.g * (h - 2.0 * C.Hnod[i]));
      acc += wq * e;
    }
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int off = 128; off > 0; off >>= 1) {
    if (threadIdx.x < off)
      sh[threadIdx.x] = (what == 0) ? fmax(sh[threadIdx.x], sh[threadIdx.x + off])
                                    : sh[threadIdx.x] + sh[threadIdx.x + off];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

}  // namespace

cudaError_t launch_controller(CtrlState* c, const double* partials, int nblk, long long n,
                              cudaStream_t s) {
  k_controller<<<1, kCtrlThreads, 0, s>>>(c, partials, nblk, n);
  return cudaGetLastError();
}

cudaError_t launch_controller_loop(CtrlState* c, const double* partials, int nblk, long long n,
                                   cudaGraphConditionalHandle loop, cudaStream_t s) {
  k_controller_loop<<<1, kCtrlThreads, 0, s>>>(c, partials, nblk, n, loop);
  return cudaGetLastError();
}

cudaError_t launch_controller_batch_loop(CtrlState* ctrls, const double* const* partials,
                                         const int* nblk, const long long* n, int ninst,
                                         int* counters, cudaGraphConditionalHandle loop,
                                         cudaStream_t s) {
  k_controller_batch_loop<<<ninst, kCtrlThreads, 0, s>>>(ctrls, partials, nblk, n, counters, loop);
  return cudaGetLastError();
}

cudaError_t launch_controller_slabs(CtrlState* c, const SlabPartials& L, long long n,
                                    cudaStream_t s) {
  k_controller_slabs<<<1, kCtrlThreads, 0, s>>>(c, L, n);
  return cudaGetLastError();
}

cudaError_t launch_controller_batch(CtrlState* ctrls, const double* const* partials,
                                    const int* nblk, const long long* n, int ninst,
                                    cudaStream_t s) {
  k_controller_batch<<<ninst, kCtrlThreads, 0, s>>>(ctrls, partials, nblk, n);
  return cudaGetLastError();
}

// ---- rk4Step (src/solver/rk.cpp:23-38) -------------------------------------------------
// The three intermediate stages run the fused stage kernel, which reads the step size from
// the controller state; this sets it for step i of a given list.
__global__ void k_rk4_set_dt(CtrlState* c, const double* dts, long long i) { c->dt = dts[i]; }

// u += (dt / 6) * (k1 + 2 k2 + 2 k3 + k4), summed left to right and every operation rounded
// on its own, as the CPU evaluates rk.cpp:36-37 (this file is built with -fmad=false).
__global__ void __launch_bounds__(256) k_rk4_update(double* __restrict__ u,
                                                    const double* __restrict__ k1,
                                                    const double* __restrict__ k2,
                                                    const double* __restrict__ k3,
                                                    const double* __restrict__ k4,
                                                    const CtrlState* c, long long n) {
  const double w = c->dt / 6.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double s = ((k1[i] + 2.0 * k2[i]) + 2.0 * k3[i]) + k4[i];
    u[i] = u[i] + w * s;
  }
}

cudaError_t launch_rk4_set_dt(CtrlState* c, const double* dts, long long i, cudaStream_t s) {
  k_rk4_set_dt<<<1, 1, 0, s>>>(c, dts, i);
  return cudaGetLastError();
}

cudaError_t launch_rk4_update(double* u, const double* k1, const double* k2, const double* k3,
                              const double* k4, const CtrlState* c, long long n, int sms,
                              cudaStream_t s) {
  const long long want = (n + 255) / 256, cap = 8LL * sms;  // 8 blocks of 256 per SM
  k_rk4_update<<<(unsigned)(want < cap ? want : cap), 256, 0, s>>>(u, k1, k2, k3, k4, c, n);
  return cudaGetLastError();
}

cudaError_t launch_reduce_diag(int what, const RhsConsts& C, const double* U, const double* qw,
                               double* out_partials, int nblk, cudaStream_t s) {
  QW q;
  for (int k = 0; k < 5; ++k) q.w[k] = qw[k];
  k_diag<<<nblk, 256, 0, s>>>(what, C, U, q, out_partials);
  return cudaGetLastError();
}

// Largest eta = h - H over the nodes inside the window [x0, x1] x [y0, y1] and the node that
// holds it (smallest index on ties), per block; the node coordinates are formed as the
// set-up forms them (node_coords, sgnb_setup.cpp), so the window test agrees with the host.
struct EtaWin {
  double x0, x1, y0, y1, hx, hy;
  double xi[5];
  int ex0;  // global index of the first element column (slabs)
};

__global__ void __launch_bounds__(256) k_eta_max(const RhsConsts C, const double* U,
                                                 const EtaWin W, double* out) {
  __shared__ double sv[256];
  __shared__ long long si[256];
  const long long Nd = C.Nd;
  double best = -HUGE_VAL;
  long long bi = -1;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < Nd;
       i += (long long)gridDim.x * blockDim.x) {
    const long long e = i / 25;
    const int loc = (int)(i - e * 25);
    const int ex = (int)(e % C.Nx), ey = (int)(e / C.Nx);
    const double x = (W.ex0 + ex) * W.hx + 0.5 * W.hx * (W.xi[loc % 5] + 1.0);
    const double y = ey * W.hy + 0.5 * W.hy * (W.xi[loc / 5] + 1.0);
    if (x < W.x0 || x > W.x1 || y < W.y0 || y > W.y1) continue;
    const double eta = U[i] - C.Hnod[i];
    if (eta > best) { best = eta; bi = i; }  // grid-stride order: first index wins ties
  }
  sv[threadIdx.x] = best;
  si[threadIdx.x] = bi;
  __syncthreads();
  for (int off = 128; off > 0; off >>= 1) {
    if (threadIdx.x < off) {
      const double ov = sv[threadIdx.x + off];
      const long long oi = si[threadIdx.x + off];
      if (oi >= 0 && (si[threadIdx.x] < 0 || ov > sv[threadIdx.x] ||
                      (ov == sv[threadIdx.x] && oi < si[threadIdx.x]))) {
        sv[threadIdx.x] = ov;
        si[threadIdx.x] = oi;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[2 * blockIdx.x] = sv[0];
    out[2 * blockIdx.x + 1] = (double)si[0];  // exact below 2^53
  }
}

cudaError_t launch_eta_max(const RhsConsts& C, const double* U, double x0, double x1, double y0,
                           double y1, double hx, double hy, int ex0, const double* xi,
                           double* out, int nblk, cudaStream_t s) {
  EtaWin W;
  W.x0 = x0; W.x1 = x1; W.y0 = y0; W.y1 = y1; W.hx = hx; W.hy = hy; W.ex0 = ex0;
  for (int k = 0; k < 5; ++k) W.xi[k] = xi[k];
  k_eta_max<<<nblk, 256, 0, s>>>(C, U, W, out);
  return cudaGetLastError();
}

// Element means (GLL quadrature average: weights sum to 2 per direction, hence 0.25) of
// eta = h - H, u, v, p and H, out[f * ne + e], in the order and rounding of the
// reference's VTK writer (src/io/vtk2d.h:38-44, 69-81): s += qw[a] qw[b] f, then 0.25 s.
__global__ void k_elem_means(const RhsConsts C, const double* U, const QW q, double* out) {
  const long long ne = (long long)C.Nx * C.Ny;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const long long Nd = C.Nd;
  for (int f = 0; f < 5; ++f) {
    double s = 0.0;
    for (int b = 0; b < 5; ++b)
      for (int a = 0; a < 5; ++a) {
        const long long i = e * 25 + a + 5 * b;
        double val;
        switch (f) {
          case 0: val = U[i] - C.Hnod[i]; break;
          case 1: val = U[Nd + i] / U[i]; break;
          case 2: val = U[2 * Nd + i] / U[i]; break;
          case 3: val = U[4 * Nd + i] / U[i]; break;
          default: val = C.Hnod[i]; break;
        }
        s += q.w[a] * q.w[b] * val;
      }
    out[f * ne + e] = 0.25 * s;
  }
}

cudaError_t launch_elem_means(const RhsConsts& C, const double* U, const double* qw, double* out,
                              cudaStream_t s) {
  QW q;
  for (int k = 0; k < 5; ++k) q.w[k] = qw[k];
  const long long ne = (long long)C.Nx * C.Ny;
  k_elem_means<<<(unsigned)((ne + 127) / 128), 128, 0, s>>>(C, U, q, out);
  return cudaGetLastError();
}

// eta at the given nodes
__global__ void k_sample_eta(const double* U, const double* Hnod, const long long* nodes, int n,
                             double* out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[k] = U[nodes[k]] - Hnod[nodes[k]];
}

cudaError_t launch_sample_eta(const double* U, const double* Hnod, const long long* nodes, int n,
                              double* out, cudaStream_t s) {
  k_sample_eta<<<(n + 127) / 128, 128, 0, s>>>(U, Hnod, nodes, n, out);
  return cudaGetLastError();
}

}  // namespace dev
}  // namespace sgnb
