// sgnb_noalloc.cu -- the diagnostics reduction (mass, energy, largest wave speed) for
// callers that cannot allocate device memory.
//
// sgnb_mass / sgnb_energy / sgnb_max_wave_speed reduce the state of a context into
// per-block partials held in a buffer the context allocated with cudaMalloc. Some
// callers cannot allocate: a framework that owns all device memory through its own
// pool or arena, or a fixed-budget time loop that must not touch the allocator (and its
// implicit synchronisation) between steps. sgnb_diag_noalloc does the same reduction for
// device arrays the caller passes in, with the per-block partials in a file-scope
// __device__ array instead: it calls no cudaMalloc, cudaFree or allocating library
// routine, and needs no context.
//
// The array holds kDiagMaxBlocks doubles (128 KB); every GPU that loads the library keeps
// it until exit. One block reduces kNodesPerBlock nodes, so a call covers at most
// kDiagMaxBlocks * kNodesPerBlock = 67,108,864 nodes per field (2,684,354 elements at
// P = 4); larger meshes are rejected with SGNB_ERR_INVALID.
//
// All calls on a device share the array. Each call writes every partial it reads before
// reading it, so nothing has to be cleared between calls, but calls whose kernels overlap
// on the GPU (different streams, no ordering between them) race on the partials.
//
// In host code the array's name is not a device address. Every call looks the address up
// on the current device (cudaGetSymbolAddress, a host-side lookup that allocates nothing),
// so no address outlives a device reset. The first call on a device also loads this
// library's device code there; make that first call before any stream capture.
#include "sgnb.h"
#include "sgnb_setup.h"

#include <cuda_runtime.h>

#include <cmath>

namespace {

constexpr int kDiagMaxBlocks = 16384;
constexpr int kNodesPerBlock = 4096;
constexpr int kThreads = 256;

static __device__ __align__(256) double g_diag_scratch[kDiagMaxBlocks];

struct DiagArgs {
  double g, c2, gamma;
  double qw[5];
};

// Per-block partial over kNodesPerBlock consecutive nodes: what = 0 largest
// characteristic speed (SGN2D::maxWaveSpeed, src/solver/sgn2d.cpp:295-305), 1 mass
// (:319-329), 2 energy (:334-348) of the reference.
__global__ void __launch_bounds__(kThreads) k_diag_partial(int what, DiagArgs a, const double* U,
                                                           const double* Hnod, long long Nd,
                                                           double* partial) {
  __shared__ double sh[kThreads];
  const long long base = (long long)blockIdx.x * kNodesPerBlock;
  double acc = 0.0;
  for (int k = threadIdx.x; k < kNodesPerBlock; k += kThreads) {
    const long long i = base + k;
    if (i >= Nd) break;
    const double h = U[i];
    const int loc = (int)(i % 25);
    const double wq = a.qw[loc % 5] * a.qw[loc / 5];
    if (what == 0) {
      const double hu = U[Nd + i], hv = U[2 * Nd + i];
      const double p = U[4 * Nd + i] / h;
      const double arg = a.g * h + p + a.c2;
      const double ce = sqrt(arg > 0.0 ? arg : 0.0);
      acc = fmax(acc, fmax(fabs(hu / h) + ce, fabs(hv / h) + ce));
    } else if (what == 1) {
      acc += wq * h;
    } else {
      const double u = U[Nd + i] / h, v = U[2 * Nd + i] / h, w = U[3 * Nd + i] / h;
      acc += wq * (0.5 * h * (u * u + v * v + (1.0 / a.gamma) * w * w + a.g * (h - 2.0 * Hnod[i])));
    }
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int off = kThreads / 2; off > 0; off >>= 1) {
    if (threadIdx.x < off)
      sh[threadIdx.x] = (what == 0) ? fmax(sh[threadIdx.x], sh[threadIdx.x + off])
                                    : sh[threadIdx.x] + sh[threadIdx.x + off];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// Combines the partials in a fixed order and writes the scaled result.
__global__ void __launch_bounds__(kThreads) k_diag_final(int what, const double* partial, int nblk,
                                                         double scale, double* out) {
  __shared__ double sh[kThreads];
  double acc = 0.0;
  for (int b = threadIdx.x; b < nblk; b += kThreads)
    acc = (what == 0) ? fmax(acc, partial[b]) : acc + partial[b];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int off = kThreads / 2; off > 0; off >>= 1) {
    if (threadIdx.x < off)
      sh[threadIdx.x] = (what == 0) ? fmax(sh[threadIdx.x], sh[threadIdx.x + off])
                                    : sh[threadIdx.x] + sh[threadIdx.x + off];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = sh[0] * scale;
}

// Device address of the scratch array on the current device, looked up on every call.
cudaError_t scratch_for_current_device(double** out) {
  double* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_diag_scratch);
  if (e != cudaSuccess) return e;
  *out = p;
  return cudaSuccess;
}

}  // namespace

extern "C" int sgnb_diag_noalloc(int what, int Nx, int Ny, double Lx, double Ly, double g,
                                 double c, double gamma, const double* U_dev,
                                 const double* Hnod_dev, double* out_dev, void* stream) {
  if (what < 0 || what > 2 || !U_dev || !out_dev || (what == 2 && !Hnod_dev))
    return SGNB_ERR_INVALID;
  if (Nx < 2 || Ny < 2 || !(Lx > 0) || !(Ly > 0)) return SGNB_ERR_INVALID;
  const long long Nd = 25LL * Nx * Ny;
  const long long nblk = (Nd + kNodesPerBlock - 1) / kNodesPerBlock;
  if (nblk > kDiagMaxBlocks) return SGNB_ERR_INVALID;  // beyond the scratch array
  double* scratch = nullptr;
  if (scratch_for_current_device(&scratch) != cudaSuccess) return SGNB_ERR_CUDA;
  sgnb::FrTables t;
  sgnb::fr_tables(4, t);
  DiagArgs a;
  a.g = g;
  a.c2 = c * c;
  a.gamma = gamma;
  for (int k = 0; k < 5; ++k) a.qw[k] = t.qw[k];
  const double hx = Lx / Nx, hy = Ly / Ny;
  const double scale = (what == 0) ? 1.0 : (0.5 * hx) * (0.5 * hy);
  cudaStream_t s = (cudaStream_t)stream;
  k_diag_partial<<<(int)nblk, kThreads, 0, s>>>(what, a, U_dev, Hnod_dev, Nd, scratch);
  if (cudaGetLastError() != cudaSuccess) return SGNB_ERR_CUDA;
  k_diag_final<<<1, kThreads, 0, s>>>(what, scratch, (int)nblk, scale, out_dev);
  if (cudaGetLastError() != cudaSuccess) return SGNB_ERR_CUDA;
  return SGNB_OK;
}
