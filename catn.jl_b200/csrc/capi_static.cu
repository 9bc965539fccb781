// libcatn_b200: the allocation-free entry point, catn_ising_contract_static.
//
// One Ising network is contracted by one CTA entirely inside a fixed
// file-scope device array laid out as [result | packed input image | slot
// (control state + arena)].  It lives in its own translation unit so that the
// persistent kernel's register allocation (capi.cu) is unaffected by this
// kernel sharing the engine's out-of-line routines.
#include <cuda_runtime.h>
#include <string>
#include "engine.cuh"
#include "host_image.h"
#include "capi_internal.h"

using namespace catn;
using namespace catn_capi;

static __device__ __align__(256) char g_static_scratch[CATN_STATIC_SCRATCH_BYTES];

namespace {

__global__ void __launch_bounds__(kThreads) catn_static_kernel(char* base, long long off_res, long long off_desc,
                                                               long long off_i64, long long off_i32,
                                                               long long off_dat, long long off_slot,
                                                               SlotLayout L) {
  extern __shared__ double smem[];
  Team T;
  T.red = smem;
  T.stage = (char*)(smem + 64);
  T.stage_bytes = GEMM_STAGE_BYTES;
  T.tcs = nullptr;
  T.tmem = 0;
  double* sws = (double*)(T.stage + GEMM_STAGE_BYTES);
  const InstDesc D = *(const InstDesc*)(base + off_desc);
  run_instance(T, base + off_slot, L, D, (const long long*)(base + off_i64), (const int*)(base + off_i32),
               (const double*)(base + off_dat), (catn_result*)(base + off_res), nullptr, sws, kSwsDoubles);
}

// Device address of g_static_scratch on the current device.  It is looked up
// on every call, with that device current: the lookup allocates nothing, and
// an address kept from an earlier call would be stale after cudaDeviceReset
// (the module, and with it the array, is loaded again).
catn_status static_scratch_address(char** out) {
  void* ptr = nullptr;
  CUDA_TRY(cudaGetSymbolAddress(&ptr, g_static_scratch));
  CUDA_TRY(cudaFuncSetAttribute(catn_static_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes));
  *out = (char*)ptr;
  return CATN_OK;
}

}  // namespace

extern "C" catn_status catn_ising_contract_static(const catn_params* p, int32_t n, int32_t n_edges,
                                                  const int32_t* edges, const double* weights, const double* fields,
                                                  double beta, int32_t pos1, int32_t val1, int32_t pos2,
                                                  int32_t val2, void* stream, catn_result* res) {
  if (catn_status s = check_params(p)) return s;
  if (!res || (n_edges > 0 && (!edges || !weights)) || !fields) return fail(CATN_EINVAL, "NULL argument");
  catn_params q = *p;
  q.trace = 0;
  Image im;   // host-side packing only
  std::string e = im.add_ising(q, n, n_edges, edges, weights, fields, beta, pos1, val1, pos2, val2, 0);
  if (!e.empty()) return fail(CATN_EINVAL, e);
  // carve the fixed array: result, input image, slot
  const long long off_res = 0;
  const long long off_desc = align256((long long)sizeof(catn_result));
  const long long off_i64 = off_desc + align256((long long)sizeof(InstDesc));
  const long long off_i32 = off_i64 + align256((long long)(sizeof(long long) * im.i64.size()));
  const long long off_dat = off_i32 + align256((long long)(sizeof(int) * im.i32.size()));
  const long long off_slot = off_dat + align256((long long)(sizeof(double) * im.dat.size()));
  const SlotLayout L0 = make_layout(im.nmax, default_maxs(im), im.emax + 64, 0);
  const long long min_arena = 1LL << 20;
  const long long avail = CATN_STATIC_SCRATCH_BYTES - off_slot - L0.slot_bytes;
  if (avail < min_arena)
    return fail(CATN_ENOMEM, "network needs " + std::to_string(off_slot + L0.slot_bytes + min_arena) +
                                 " bytes of device scratch; the static maximum is " +
                                 std::to_string((long long)CATN_STATIC_SCRATCH_BYTES));
  const SlotLayout L = make_layout(im.nmax, default_maxs(im), im.emax + 64, avail & ~255LL);
  char* base = nullptr;
  if (catn_status s = static_scratch_address(&base)) return s;
  cudaStream_t st = (cudaStream_t)stream;
  // inputs in; the previous call's result is cleared so that a failed launch
  // cannot return stale values
  CUDA_TRY(cudaMemsetAsync(base + off_res, 0, sizeof(catn_result), st));
  CUDA_TRY(cudaMemcpyAsync(base + off_desc, im.desc.data(), sizeof(InstDesc), cudaMemcpyHostToDevice, st));
  if (!im.i64.empty())
    CUDA_TRY(cudaMemcpyAsync(base + off_i64, im.i64.data(), sizeof(long long) * im.i64.size(),
                             cudaMemcpyHostToDevice, st));
  if (!im.i32.empty())
    CUDA_TRY(cudaMemcpyAsync(base + off_i32, im.i32.data(), sizeof(int) * im.i32.size(), cudaMemcpyHostToDevice,
                             st));
  if (!im.dat.empty())
    CUDA_TRY(cudaMemcpyAsync(base + off_dat, im.dat.data(), sizeof(double) * im.dat.size(),
                             cudaMemcpyHostToDevice, st));
  catn_static_kernel<<<1, kThreads, kSmemBytes, st>>>(base, off_res, off_desc, off_i64, off_i32, off_dat, off_slot,
                                                       L);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(res, base + off_res, sizeof(catn_result), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  if (res->status != CATN_OK)
    return fail((catn_status)res->status, std::string("contraction failed: ") + status_text(res->status));
  return CATN_OK;
}
