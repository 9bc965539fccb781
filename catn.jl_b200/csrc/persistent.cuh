// The persistent kernel of a forward launch, shared by the translation units
// that instantiate it: capi.cu (variant 0, every route) and capi_lean.cu
// (variant 1, compiled with CATN_LEAN: no block route, blocked QR,
// tensor-core merges or matrix-free swaps, for launches that use none).
#pragma once
#include "engine.cuh"
#include "capi_internal.h"

namespace catn_capi {

using namespace catn;

// `order` lists instance ids by descending work estimate, so the longest
// contractions start first (longest-processing-time scheduling).  With a job
// board, the last `nhelp` CTAs and every CTA that finds the queue drained
// help the large SVDs of the CTAs still contracting (help_jobs) until all are
// finished.  With split-precision instances every CTA holds TMEM columns and
// the tensor-core staging area for the block route's products.
template <int kVariant>
__global__ void __launch_bounds__(kThreads) catn_persistent_kernel(
    const InstDesc* __restrict__ descs, const int* __restrict__ order, int ninst, const long long* i64,
    const int* i32, const double* dat, char* slots, SlotLayout L, catn_result* res, int* trace, int* queue,
    JacobiJob* board, int nhelp, JobLink jl, int use_tc) {
  extern __shared__ double smem[];
  Team T;
  T.red = smem;
  T.stage = (char*)(smem + 64);
  T.stage_bytes = GEMM_STAGE_BYTES;
  T.tcs = nullptr;
  T.tmem = 0;
  if (use_tc) tc_setup(T, tc_region(smem));
  double* sws = (double*)(T.stage + GEMM_STAGE_BYTES);
  char* slot = slots + (long long)blockIdx.x * L.slot_bytes;
  jl.job = board ? board + blockIdx.x : nullptr;
  jl.qhead = queue;
  const bool helper = board && (int)blockIdx.x >= (int)gridDim.x - nhelp;
  for (;;) {
    if (helper) break;
    long long inst = 0;
    if (threadIdx.x == 0) {
      const int q = atomicAdd(queue, 1);
      inst = q < ninst ? order[q] : ninst;
    }
    inst = T.bcast(inst);
    if (inst >= ninst) break;
    run_instance(T, slot, L, descs[inst], i64, i32, dat, res + inst, trace, sws,
                 kVariant == 1 ? kSwsDoublesLean : kSwsDoubles,
                 board ? &jl : nullptr);
    if (board && threadIdx.x == 0) atomicAdd(queue + 1, 1);
    // A shared wait that ran out leaves a helper warp that may still write
    // into this slot's arena: the slot takes no further instance (the other
    // CTAs drain the queue).
    if (T.bcast(threadIdx.x == 0 ? res[inst].status : 0) == CATN_ETIMEOUT) break;
  }
  if (board) {
    if (jl.cta_jobs && !CATN_LEAN)
      help_jobs(T, board, (int)gridDim.x, queue + 1, ninst, sws);
    else
      help_jacobi(T, board, (int)gridDim.x, queue + 1, ninst);
  }
  tc_teardown(T);
}

}  // namespace catn_capi
