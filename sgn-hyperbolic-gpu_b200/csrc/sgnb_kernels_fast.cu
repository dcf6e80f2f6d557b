// sgnb_kernels_fast.cu -- fused kernels in the fast arithmetic mode.
// Built with -fmad=true: FMA contraction, reciprocals of h and of the Jacobians.
// Agrees with the reference to round-off (relative 1e-13 per field is the test bound).
#define SGNB_EXACT false
#include "sgnb_kernels_inst.cuh"

namespace sgnb {
namespace dev {
cudaError_t launch_fused_fast(int mode, const RhsConsts& C, const StageArgs& A, cudaStream_t s,
                              const TileMaps* M) {
  return launch_any(mode, C, A, s, M);
}
cudaError_t prepare_fused_fast() { return prepare_all(); }

// The checked build's out-of-range count of this translation unit's kernels (reset: then
// zero it); cudaErrorNotSupported in the normal build.
cudaError_t read_oob_fast(unsigned long long* out, bool reset) {
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

// The fast mode's reciprocal (fn 0) and square root (fn 1) on a device array, for tests.
__global__ void k_fast_math(int fn, const double* __restrict__ x, double* __restrict__ y,
                            long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = fn == 0 ? fast_rcp(x[i]) : fast_sqrt(x[i]);
}

cudaError_t launch_fast_math(int fn, const double* x, double* y, long long n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_fast_math<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(fn, x, y, n);
  return cudaGetLastError();
}

// Slab edges: one thread per (side, field, row, transverse node). Side 0 reads the first
// element column's left nodes (a = 0) into sendL, side 1 the last column's right nodes
// (a = P) into sendR; both [field][row][node]. The stage inputs are formed with the same
// explicitly rounded combinations as the fused kernels' own and halo nodes, so a
// neighbour's ghost holds the bits its own tile would have formed.
__global__ void k_pack_ghosts(int mode, const RhsConsts C, const StageArgs A, double* sendL,
                              double* sendR) {
  const long long per = (long long)NV * C.Ny * NP;
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 2 * per) return;
  if (mode != 0 && A.ctrl->done) return;
  const int side = (int)(q / per);
  const long long r = q - side * per;
  const int t = (int)(r % NP), ey = (int)((r / NP) % C.Ny), v = (int)(r / ((long long)NP * C.Ny));
  const int ex = side == 0 ? 0 : C.Nx - 1, a = side == 0 ? 0 : NP - 1;
  const long long g = (long long)v * C.Nd + ((long long)ex + (long long)C.Nx * ey) * NPP + a + NP * t;
  double val;
  if (mode == 0) {
    val = A.in[g];
  } else {
    const int cur = A.ctrl->cur;
    const double dt = A.ctrl->dt;
    if (mode == 1) {
      const double* k = A.kin_k2 ? A.K2 : A.K1[cur];
      val = stage_axpy(A.U[cur][g], A.coef * dt, k[g]);
    } else {
      val = fsal_finish(A.U[cur][g], fsal_part(A.K1[cur][g], A.K2[g]), A.K3[g], dt);
    }
  }
  (side == 0 ? sendL : sendR)[r] = val;
}

cudaError_t launch_pack_ghosts(int mode, const RhsConsts& C, const StageArgs& A, double* sendL,
                               double* sendR, cudaStream_t s) {
  const long long n = 2LL * NV * C.Ny * NP;
  const int threads = 256;
  k_pack_ghosts<<<(unsigned)((n + threads - 1) / threads), threads, 0, s>>>(mode, C, A, sendL,
                                                                            sendR);
  return cudaGetLastError();
}

template <int MODE, int TXs, int TYs>
static cudaError_t launch_b(int blocks, const BatchArgs& B, cudaStream_t s) {
  const size_t smem = sizeof(typename Tile<TXs, TYs, false>::Smem);
  if (blocks > 0) {
    k_fused_batch<MODE, false, TXs, TYs, true><<<blocks, NTHR, smem, s>>>(B);
  } else {
    if (B.ntiles < 1 || B.ntiles > 0x7fffffffLL) return cudaErrorInvalidValue;
    k_fused_batch<MODE, false, TXs, TYs, false><<<(unsigned)B.ntiles, NTHR, smem, s>>>(B);
  }
  return cudaGetLastError();
}

template <int TXs, int TYs>
static cudaError_t launch_shape(int mode, int blocks, const BatchArgs& B, cudaStream_t s) {
  switch (mode) {
    case MODE_RHS: return launch_b<MODE_RHS, TXs, TYs>(blocks, B, s);
    case MODE_STAGE: return launch_b<MODE_STAGE, TXs, TYs>(blocks, B, s);
    case MODE_FSAL: return launch_b<MODE_FSAL, TXs, TYs>(blocks, B, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_fused_batch(int mode, int shape_id, int blocks, const BatchArgs& B,
                               cudaStream_t s) {
  switch (shape_id) {
    case 0: return launch_shape<8, 4>(mode, blocks, B, s);
    case 1: return launch_shape<16, 2>(mode, blocks, B, s);
    case 2: return launch_shape<4, 8>(mode, blocks, B, s);
    default: return cudaErrorInvalidValue;
  }
}

int batch_tile_tx(int shape_id) { return shape_id == 1 ? 16 : (shape_id == 2 ? 4 : 8); }

template <int MODE, int TXs, int TYs>
static cudaError_t prepare_mode() {
  const int bytes = (int)sizeof(typename Tile<TXs, TYs, false>::Smem);
  cudaError_t e = cudaFuncSetAttribute(k_fused_batch<MODE, false, TXs, TYs, true>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_fused_batch<MODE, false, TXs, TYs, false>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

template <int TXs, int TYs>
static cudaError_t prepare_shape() {
  cudaError_t e = prepare_mode<MODE_RHS, TXs, TYs>();
  if (e == cudaSuccess) e = prepare_mode<MODE_STAGE, TXs, TYs>();
  if (e == cudaSuccess) e = prepare_mode<MODE_FSAL, TXs, TYs>();
  return e;
}

cudaError_t prepare_fused_batch() {
  cudaError_t e = prepare_shape<8, 4>();
  if (e == cudaSuccess) e = prepare_shape<16, 2>();
  if (e == cudaSuccess) e = prepare_shape<4, 8>();
  return e;
}
}  // namespace dev
}  // namespace sgnb
