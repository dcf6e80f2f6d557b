// sgnb_kernels_fast.cu -- fused kernels in the fast arithmetic mode.
// Built with -fmad=true: FMA contraction, reciprocals of h and of the Jacobians.
// Agrees with the reference to round-off (relative 1e-13 per field is the test bound).
#define SGNB_EXACT false
#include "sgnb_kernels_inst.cuh"

namespace sgnb {
namespace dev {
cudaError_t launch_fused_fast(int mode, const RhsConsts& C, const StageArgs& A, cudaStream_t s) {
  return launch_any(mode, C, A, s);
}
cudaError_t prepare_fused_fast() { return prepare_all(); }

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
