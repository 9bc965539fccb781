// libcatn_b200: the persistent kernel without the routes of split precision
// and of the block Jacobi SVD.
//
// Launches whose instances all run in FP64 on the scalar Jacobi route,
// without the matrix-free randomized swaps (the batched spin-glass workload
// among them), take this instantiation.  It is the same engine compiled with
// CATN_LEAN and without tcgen05 instructions: code those launches never
// reach is left out, which frees registers and stack in the kernel that runs
// them (the arithmetic of every route it keeps is the same instruction for
// instruction as in capi.cu's instantiation).
#define CATN_LEAN 1
#define CATN_NO_TCGEN05 1
#include <cuda_runtime.h>
#include "persistent.cuh"

namespace catn_capi {

cudaError_t persistent_lean_attr() {
  return cudaFuncSetAttribute(catn_persistent_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytesLean);
}

cudaError_t persistent_lean_launch(const DeviceRun& R, int nhelp, const JobLink& jl, cudaStream_t st) {
  catn_persistent_kernel<1><<<R.ngrid, kThreads, kSmemBytesLean, st>>>(
      R.d_desc, R.d_order, R.ninst, R.d_i64, R.d_i32, R.d_dat, R.d_slots, R.L, R.d_res, R.d_trace, R.d_queue,
      R.d_board, nhelp, jl, 0);
  return cudaGetLastError();
}

}  // namespace catn_capi
