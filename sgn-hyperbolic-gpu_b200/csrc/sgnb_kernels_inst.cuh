// sgnb_kernels_inst.cuh -- instantiates the fused kernels for one arithmetic mode.
// Included by sgnb_kernels_exact.cu (SGNB_EXACT = true, built with -fmad=false) and
// sgnb_kernels_fast.cu (SGNB_EXACT = false, built with -fmad=true).
#pragma once

#include "sgnb_kernels.cuh"

namespace sgnb {
namespace dev {

template <int MODE>
static cudaError_t launch_mode(const RhsConsts& C, const StageArgs& A, cudaStream_t s,
                               const TileMaps* M) {
  const dim3 grid((C.Nx + 7) / 8, (C.Ny + 3) / 4);
  const size_t smem = sizeof(Tile<8, 4, SGNB_EXACT>::Smem);
  if (C.gauss) {
    const long long n = 2LL * C.Nx * C.Ny * NP;
    k_traces<MODE, SGNB_EXACT><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(C, A);
    if (C.manning) k_fused<MODE, SGNB_EXACT, true, false, true><<<grid, NTHR, smem, s>>>(C, A);
    else k_fused<MODE, SGNB_EXACT, false, false, true><<<grid, NTHR, smem, s>>>(C, A);
    return cudaGetLastError();
  }
  const bool ghost = C.ghostL != nullptr || C.ghostR != nullptr;
  if (C.manning) {
    if (ghost) k_fused<MODE, SGNB_EXACT, true, true><<<grid, NTHR, smem, s>>>(C, A);
    else k_fused<MODE, SGNB_EXACT, true, false><<<grid, NTHR, smem, s>>>(C, A);
  } else {
    const bool full = C.Nx % 8 == 0 && C.Ny % 4 == 0;  // every tile full
    // the own-node tiles by the tensor-memory accelerator where the context's tensor maps
    // describe the buffers (and, for the rhs mode, a map of its input)
    const bool tma = full && M != nullptr && M->ok && (MODE != MODE_RHS || M->inOk);
    if (ghost) {
      if (tma) k_fused_tma<MODE, SGNB_EXACT, true><<<grid, NTHR, smem, s>>>(C, A, *M);
      else if (full) k_fused<MODE, SGNB_EXACT, false, true, false, true><<<grid, NTHR, smem, s>>>(C, A);
      else k_fused<MODE, SGNB_EXACT, false, true><<<grid, NTHR, smem, s>>>(C, A);
    } else if (full) {
      if (tma)
        k_fused_tma<MODE, SGNB_EXACT><<<grid, NTHR, smem, s>>>(C, A, *M);
      else
        k_fused<MODE, SGNB_EXACT, false, false, false, true><<<grid, NTHR, smem, s>>>(C, A);
    } else {
      k_fused<MODE, SGNB_EXACT, false, false><<<grid, NTHR, smem, s>>>(C, A);
    }
  }
  return cudaGetLastError();
}

template <bool FRIC, bool GHOST, bool GAUSS = false, bool FULL = false>
static cudaError_t prepare_variant() {
  const int bytes = (int)sizeof(Tile<8, 4, SGNB_EXACT>::Smem);
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(k_fused<MODE_RHS, SGNB_EXACT, FRIC, GHOST, GAUSS, FULL>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(k_fused<MODE_STAGE, SGNB_EXACT, FRIC, GHOST, GAUSS, FULL>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)) != cudaSuccess)
    return e;
  return cudaFuncSetAttribute(k_fused<MODE_FSAL, SGNB_EXACT, FRIC, GHOST, GAUSS, FULL>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

static cudaError_t prepare_all() {
  cudaError_t e = prepare_variant<false, false>();
  if (e == cudaSuccess) e = prepare_variant<true, false>();
  if (e == cudaSuccess) e = prepare_variant<false, true>();
  if (e == cudaSuccess) e = prepare_variant<true, true>();
  if (e == cudaSuccess) e = prepare_variant<false, false, true>();
  if (e == cudaSuccess) e = prepare_variant<true, false, true>();
  if (e == cudaSuccess) e = prepare_variant<false, false, false, true>();
  if (e == cudaSuccess) e = prepare_variant<false, true, false, true>();
  {
    const int bytes = (int)sizeof(Tile<8, 4, SGNB_EXACT>::Smem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_fused_tma<MODE_RHS, SGNB_EXACT>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_fused_tma<MODE_STAGE, SGNB_EXACT>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_fused_tma<MODE_FSAL, SGNB_EXACT>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_fused_tma<MODE_RHS, SGNB_EXACT, true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_fused_tma<MODE_STAGE, SGNB_EXACT, true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_fused_tma<MODE_FSAL, SGNB_EXACT, true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  }
  return e;
}

static cudaError_t launch_any(int mode, const RhsConsts& C, const StageArgs& A, cudaStream_t s,
                              const TileMaps* M = nullptr) {
  switch (mode) {
    case MODE_RHS: return launch_mode<MODE_RHS>(C, A, s, M);
    case MODE_STAGE: return launch_mode<MODE_STAGE>(C, A, s, M);
    case MODE_FSAL: return launch_mode<MODE_FSAL>(C, A, s, M);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace dev
}  // namespace sgnb
