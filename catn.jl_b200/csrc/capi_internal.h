// Host-side helpers shared by the translation units of libcatn_b200
// (capi.cu: the persistent-kernel entry points; capi_static.cu: the
// allocation-free entry point).  Each unit compiles the device engine on its
// own, so the register allocation of one kernel's call tree never depends on
// another kernel that shares the engine's out-of-line routines.
#pragma once
#include <cuda_runtime.h>
#include <string>
#include "catn_b200.h"
#include "linalg.cuh"

namespace catn_capi {

constexpr int kThreads = 256;
// Dynamic shared memory per CTA: reduction area, GEMM tile staging, and the
// small-SVD workspace (two CTAs fit on one SM).
constexpr int kSmemBytes = 100 * 1024;
constexpr long long kSwsDoubles = (kSmemBytes - 64 * 8 - catn::GEMM_STAGE_BYTES) / 8;

// Records `msg` as the calling thread's last error and returns `s`.
catn_status fail(catn_status s, const std::string& msg);
catn_status cuda_fail(cudaError_t e, const char* what);
const char* status_text(int s);
// Argument checks shared by every create/contract entry point.
catn_status check_params(const catn_params* p);

}  // namespace catn_capi

#define CUDA_TRY(expr)                                                \
  do {                                                                \
    cudaError_t _e = (expr);                                          \
    if (_e != cudaSuccess) return catn_capi::cuda_fail(_e, #expr);    \
  } while (0)
