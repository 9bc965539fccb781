// libcatn_b200: the BraKet (<psi|psi>) kernel.  Networks made by
// catn_braket_create are contracted by catn_contract through this unit's
// persistent kernel, which runs run_instance_braket (braket.cuh); it is
// compiled on its own so that the forward kernel's register allocation
// (capi.cu) is unaffected.
#include <cuda_runtime.h>
#include "braket.cuh"
#include "capi_internal.h"

using namespace catn;
using namespace catn_capi;

namespace {

__global__ void __launch_bounds__(kThreads) catn_braket_kernel(
    const InstDesc* __restrict__ descs, const int* __restrict__ order, int ninst, const long long* i64,
    const int* i32, const double* dat, char* slots, SlotLayout L, catn_result* res, int* trace, int* queue) {
  extern __shared__ double smem[];
  Team T;
  T.red = smem;
  T.stage = (char*)(smem + 64);
  T.stage_bytes = GEMM_STAGE_BYTES;
  T.tcs = nullptr;
  T.tmem = 0;
  double* sws = (double*)(T.stage + GEMM_STAGE_BYTES);
  char* slot = slots + (long long)blockIdx.x * L.slot_bytes;
  for (;;) {
    long long inst = 0;
    if (threadIdx.x == 0) {
      const int q = atomicAdd(queue, 1);
      inst = q < ninst ? order[q] : ninst;
    }
    inst = T.bcast(inst);
    if (inst >= ninst) break;
    run_instance_braket(T, slot, L, descs[inst], i64, i32, dat, res + inst, trace, sws, kSwsDoubles);
  }
}

}  // namespace

namespace catn_capi {

catn_status braket_launch(DeviceRun& R, cudaStream_t st) {
  CUDA_TRY(cudaFuncSetAttribute(catn_braket_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes));
  CUDA_TRY(cudaMemsetAsync(R.d_queue, 0, sizeof(int), st));
  catn_braket_kernel<<<R.nslots, kThreads, kSmemBytes, st>>>(R.d_desc, R.d_order, R.ninst, R.d_i64, R.d_i32, R.d_dat,
                                                             R.d_slots, R.L, R.d_res, R.d_trace, R.d_queue);
  CUDA_TRY(cudaGetLastError());
  return CATN_OK;
}

}  // namespace catn_capi
