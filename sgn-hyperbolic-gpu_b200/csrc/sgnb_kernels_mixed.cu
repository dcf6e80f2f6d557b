// sgnb_kernels_mixed.cu -- mixed-precision fused kernels (FP32 deviations, FP64
// hydrostatic balance, state and controller). Built with -fmad=true.
#include "sgnb_kernels_mixed.cuh"

namespace sgnb {
namespace dev {

template <int MODE>
static cudaError_t launch_m(const RhsConsts& C, const StageArgsM& A, cudaStream_t s,
                            const TileMapsM* M) {
  const dim3 grid((C.Nx + mix::TX - 1) / mix::TX, (C.Ny + mix::TY - 1) / mix::TY);
  if (C.manning) {
    mix::k_mixed<MODE, true><<<grid, mix::NTHR, sizeof(mix::Smem), s>>>(C, A);
  } else if (C.Nx % mix::TX == 0 && C.Ny % mix::TY == 0) {  // every tile full
    bool tma = false;
    // the intermediate stage's tiles by the tensor-memory accelerator (the end-point stage
    // was 1.4 % slower so: its per-thread copies land in five scattered areas)
    if constexpr (MODE == mix::MODE_STAGE) {
      if (M != nullptr && M->ok) {
        mix::k_mixed_tma<MODE><<<grid, mix::NTHR, sizeof(mix::Smem), s>>>(C, A, *M);
        tma = true;
      }
    }
    if (!tma) mix::k_mixed<MODE, false, true><<<grid, mix::NTHR, sizeof(mix::Smem), s>>>(C, A);
  } else {
    mix::k_mixed<MODE, false><<<grid, mix::NTHR, sizeof(mix::Smem), s>>>(C, A);
  }
  return cudaGetLastError();
}

// The checked build's out-of-range count of the mixed kernels (reset: then zero it);
// cudaErrorNotSupported in the normal build.
cudaError_t read_oob_mixed(unsigned long long* out, bool reset) {
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

cudaError_t launch_fused_mixed(int mode, const RhsConsts& C, const StageArgsM& A, cudaStream_t s,
                               const TileMapsM* M) {
  switch (mode) {
    case 0: return launch_m<mix::MODE_RHS>(C, A, s, M);
    case 1: return launch_m<mix::MODE_STAGE>(C, A, s, M);
    case 2: return launch_m<mix::MODE_FSAL>(C, A, s, M);
    default: return cudaErrorInvalidValue;
  }
}

template <bool FRIC, bool FULL = false>
static cudaError_t prepare_mixed_fric() {
  const int bytes = (int)sizeof(mix::Smem);
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(mix::k_mixed<mix::MODE_RHS, FRIC, FULL>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(mix::k_mixed<mix::MODE_STAGE, FRIC, FULL>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)) != cudaSuccess)
    return e;
  return cudaFuncSetAttribute(mix::k_mixed<mix::MODE_FSAL, FRIC, FULL>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

cudaError_t prepare_fused_mixed() {
  cudaError_t e = prepare_mixed_fric<false>();
  if (e == cudaSuccess) e = prepare_mixed_fric<false, true>();
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(mix::k_mixed_tma<mix::MODE_STAGE>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(mix::Smem));
  return e == cudaSuccess ? prepare_mixed_fric<true>() : e;
}

template <int MODE>
static cudaError_t launch_mb(int blocks, const BatchArgsM& B, cudaStream_t s) {
  if (blocks > 0) {
    mix::k_mixed_batch<MODE, true><<<blocks, mix::NTHR, sizeof(mix::Smem), s>>>(B);
  } else {
    if (B.ntiles < 1 || B.ntiles > 0x7fffffffLL) return cudaErrorInvalidValue;
    mix::k_mixed_batch<MODE, false><<<(unsigned)B.ntiles, mix::NTHR, sizeof(mix::Smem), s>>>(B);
  }
  return cudaGetLastError();
}

cudaError_t launch_mixed_batch(int mode, int blocks, const BatchArgsM& B, cudaStream_t s) {
  switch (mode) {
    case 0: return launch_mb<mix::MODE_RHS>(blocks, B, s);
    case 1: return launch_mb<mix::MODE_STAGE>(blocks, B, s);
    case 2: return launch_mb<mix::MODE_FSAL>(blocks, B, s);
    default: return cudaErrorInvalidValue;
  }
}

template <int MODE>
static cudaError_t prepare_mb() {
  const int bytes = (int)sizeof(mix::Smem);
  cudaError_t e = cudaFuncSetAttribute(mix::k_mixed_batch<MODE, true>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(mix::k_mixed_batch<MODE, false>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

cudaError_t prepare_mixed_batch() {
  cudaError_t e = prepare_mb<mix::MODE_RHS>();
  if (e == cudaSuccess) e = prepare_mb<mix::MODE_STAGE>();
  if (e == cudaSuccess) e = prepare_mb<mix::MODE_FSAL>();
  return e;
}

}  // namespace dev
}  // namespace sgnb
