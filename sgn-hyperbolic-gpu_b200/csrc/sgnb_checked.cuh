// sgnb_checked.cuh -- index checks of the checked build of the library.
//
// libsgnb_checked.so is compiled with -DSGNB_CHECKED: SGNB_INB(i, n) is then false, and
// the out-of-range access is counted (g_sgnb_oob, one counter per translation unit, read by
// sgnb_checked_oob) and skipped, when i is outside [0, n). In the normal build SGNB_INB is
// the literal true, so the kernels compile exactly as without the checks.
#pragma once

#ifdef SGNB_CHECKED
static __device__ unsigned long long g_sgnb_oob;
__device__ __forceinline__ bool inb(long long i, long long n) {
  if (i >= 0 && i < n) return true;
  atomicAdd(&g_sgnb_oob, 1ULL);
  return false;
}
#define SGNB_INB(i, n) inb((i), (n))
#else
#define SGNB_INB(i, n) true
#endif
