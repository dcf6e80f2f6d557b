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
}  // namespace dev
}  // namespace sgnb
