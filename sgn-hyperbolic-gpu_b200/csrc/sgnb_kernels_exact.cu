// sgnb_kernels_exact.cu -- fused kernels in the exact arithmetic mode.
// Built with -fmad=false: every product and sum rounds separately, in the operation
// order of the reference CPU solver, so the results are bit-identical to it.
#define SGNB_EXACT true
#include "sgnb_kernels_inst.cuh"

namespace sgnb {
namespace dev {
cudaError_t launch_fused_exact(int mode, const RhsConsts& C, const StageArgs& A, cudaStream_t s,
                              const TileMaps* M) {
  return launch_any(mode, C, A, s, M);
}
cudaError_t prepare_fused_exact() { return prepare_all(); }
int fused_grid_blocks(int Nx, int Ny) { return ((Nx + 7) / 8) * ((Ny + 3) / 4); }
size_t fused_smem_bytes() { return sizeof(Tile<8, 4, true>::Smem); }
// The checked build's out-of-range count of this translation unit's kernels (reset: then
// zero it); cudaErrorNotSupported in the normal build.
cudaError_t read_oob_exact(unsigned long long* out, bool reset) {
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

}  // namespace dev
}  // namespace sgnb
