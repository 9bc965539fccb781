// Host-side helpers shared by the translation units of libcatn_b200
// (capi.cu: the persistent-kernel entry points; capi_static.cu: the
// allocation-free entry point; capi_grad.cu: the adjoint; capi_braket.cu:
// the BraKet kernel).  Each unit
// compiles the device engine on its own, so the register allocation of one
// kernel's call tree never depends on another kernel that shares the
// engine's out-of-line routines.
#pragma once
#include <cuda_runtime.h>
#include <string>
#include "catn_b200.h"
#include "linalg.cuh"
#include "blockjac.cuh"
#include "host_image.h"

namespace catn {
struct JobLink;
}

namespace catn_capi {

constexpr int kThreads = 256;
// Dynamic shared memory per CTA: reduction area, GEMM tile staging, and the
// small-SVD workspace.  The persistent kernel's 255 registers per thread
// limit an SM to one 256-thread CTA.  Shared memory and the L1 cache share
// the SM's 256 KB, in configurations of 0 / 8 / 16 / 32 / 64 / 100 / 132 /
// 164 / 196 / 228 KB of shared memory, and the runtime reserves 1 KB per CTA.
// The engine's loads of slot data (L2-resident) go through L1, and its time
// follows L1's capacity (measured on the 512-instance spin-glass batch:
// 315 ms at 100 KB, i.e. the 132 KB configuration and 124 KB of L1; 305 ms
// at 98 KB, the 100 KB configuration; 300 ms at 62 KB, the 64 KB
// configuration; 378 ms at 200 KB).  98 KB keeps the block route's items and
// the blocked QR's panels in shared memory.
constexpr int kSmemBytes = 98 * 1024;
constexpr long long kSwsDoubles = (kSmemBytes - 64 * 8 - catn::GEMM_STAGE_BYTES) / 8;
static_assert(kSwsDoubles >= catn::kBlockWsDoubles, "block-route items need their workspace in shared memory");
static_assert(kSwsDoubles >= catn::kPanelWsDoubles + catn::kPanelW, "panel items need their workspace in shared memory");
// The lean instantiation (capi_lean.cu) has neither: 62 KB, the 64 KB
// configuration (192 KB of L1); its small-SVD workspace still holds the
// tiny one-warp SVDs (64 x 16) and every SVD up to 5792 doubles of workspace.
constexpr int kSmemBytesLean = 62 * 1024;
constexpr long long kSwsDoublesLean = (kSmemBytesLean - 64 * 8 - catn::GEMM_STAGE_BYTES) / 8;
static_assert(kSwsDoublesLean >= 2 * 64 * 16 + 3 * 16 * 16 + 8 * 16 + 64, "the tiny SVDs need their workspace");
// Launches with split-precision instances add the tensor-core staging area
// (blockjac_tc.cuh) after the small-SVD workspace.
constexpr int kSmemBytesTc = kSmemBytes + catn::kTcRegionBytes + 1024;
static_assert(kSmemBytesTc <= 227 * 1024, "shared memory per CTA");
// The staging area of a kernel's dynamic shared memory (1024-aligned).
__device__ inline unsigned char* tc_region(double* smem) {
  return (unsigned char*)((((uintptr_t)smem + kSmemBytes) + 1023) & ~(uintptr_t)1023);
}
// Smallest rows x columns whose Householder steps (pivoted QR, applying Q)
// are shared with helper warps: one publish/claim/wait per reflector must be
// outweighed.  On the 512-instance spin-glass batch 2^20 / 2^18 / 2^17 / 2^16
// elements measured 311 / 311 / 311 / 315 ms per launch (the helpers are
// then wanted by the shared Jacobi rounds).
constexpr long long kSharedHouseMinElems = 1LL << 20;

// Records `msg` as the calling thread's last error and returns `s`.
catn_status fail(catn_status s, const std::string& msg);
catn_status cuda_fail(cudaError_t e, const char* what);
const char* status_text(int s);
// Argument checks shared by every create/contract entry point.
catn_status check_params(const catn_params* p);

// Blocks of the process-wide cache (pool.cu): device memory, or pinned host
// memory with `host`.  pool_free keeps the block for a later request (or
// frees it); pointers that did not come from pool_alloc are ignored.
cudaError_t pool_alloc(void** p, size_t bytes, bool host = false);
void pool_free(void* p);
size_t pool_cached_bytes(bool host);
template <typename T>
inline cudaError_t pool_new(T** p, size_t bytes, bool host = false) {
  return pool_alloc((void**)p, bytes, host);
}

// Device copy of an Image plus slots and results.  The input image is packed
// into one pinned host buffer and one device buffer, so an upload is a single
// host-to-device copy.
struct DeviceRun {
  char* h_input = nullptr;   // pinned
  char* d_input = nullptr;
  catn::InstDesc* d_desc = nullptr;
  int* d_order = nullptr;
  long long* d_i64 = nullptr;
  int* d_i32 = nullptr;
  double* d_dat = nullptr;
  char* d_slots = nullptr;
  catn_result* d_res = nullptr;
  int* d_trace = nullptr;
  int* d_queue = nullptr;    // [0] work-queue head, [1] instances finished
  catn::JacobiJob* d_board = nullptr;   // shared Jacobi jobs, one per slot (batches only)
  catn::SlotLayout L;
  int nslots = 0;
  int ngrid = 0;   // CTAs per launch: nslots, or every resident CTA for one network (the rest help)
  int ninst = 0;
  int use_tc = 0;  // some instance runs in split precision: TMEM and the staging area per CTA
  int cta_jobs = 0;   // some instance takes the block SVD route (its jobs are CTA items)
  int lean = 0;       // forward launches run the lean instantiation (capi_lean.cu)
  long long input_bytes = 0;

  void release() {
    pool_free(h_input);
    pool_free(d_input); pool_free(d_slots); pool_free(d_res); pool_free(d_trace); pool_free(d_queue);
    pool_free(d_board);
    h_input = nullptr; d_input = nullptr; d_slots = nullptr; d_res = nullptr; d_trace = nullptr; d_queue = nullptr;
    d_board = nullptr;
    d_desc = nullptr; d_order = nullptr; d_i64 = nullptr; d_i32 = nullptr; d_dat = nullptr;
  }
};

// Device buffers of a gradient run: its own slots (heap + shadow + tape) and
// the gradients of the input sites, in the image's data layout.
struct GradRun {
  DeviceRun R;
  double* d_gimg = nullptr;
  double* h_gimg = nullptr;   // pinned
  long long arena = 0;
};

// Sizes slots and packs the image (capi.cu).
// `single_forward`: R is one network that catn_contract launches (its auto
// SVD route may then take the block route, see capi.cu).
catn_status prepare(const catn::Image& im, long long arena_bytes, int max_slots, DeviceRun& R,
                    bool single_forward = false);
catn_status upload(DeviceRun& R, cudaStream_t st);
// Helper pool and sharing thresholds of a launch of R from the tuning table
// in force (capi.cu); `grad` selects the gradient launches' pool.  One
// network always gets every other resident CTA as a helper.  The launch's
// CTAs fill in their own job and queue pointers.
void helper_config(const DeviceRun& R, bool grad, catn::JobLink* jl, int* nhelp);
// Helper pool of batch gradient launches: 0 / 8 / 16 / 24 CTAs measured 592-598
// / 547 / 578 / 610 ms on the 512-instance spin-glass batch (taped instances
// are long, so most CTAs are worth more as workers).
constexpr int kGradHelperCtas = 8;
// Arena of a single network when the caller passes 0 (capi.cu).
long long default_arena(long long a, const catn_params& p);
// Frees a gradient run (capi_grad.cu).
void grad_release(GradRun* g);
// The lean persistent kernel (capi_lean.cu): its shared-memory attribute,
// and a launch of R.
cudaError_t persistent_lean_attr();
cudaError_t persistent_lean_launch(const DeviceRun& R, int nhelp, const catn::JobLink& jl, cudaStream_t st);
// Runs the BraKet kernel over a prepared run (capi_braket.cu).
catn_status braket_launch(DeviceRun& R, cudaStream_t st);

}  // namespace catn_capi

struct catn_net {
  catn::Image im;
  catn_capi::DeviceRun R;
  long long arena = 0;      // arena bytes of the slot (after defaults)
  std::vector<int> cuts;    // cut_bondim! calls so far: i, idx_j_in_i, opt
  bool contracted = false;
  bool unusable = false;    // a failed cut left no device copy to contract
  catn_capi::GradRun* grad = nullptr;
};

namespace catn_capi {
// Device-side disorder of an Ising batch (catn_ising_batch_set_params /
// _randomize): the site recipes recorded at creation, the current couplings,
// fields and betas, and whether the device image holds values rebuilt from
// them instead of the ones given at creation.
struct IsingParams {
  catn::IsingSiteRecipe* d_rec = nullptr;
  double* d_w = nullptr;
  double* d_h = nullptr;
  double* d_beta = nullptr;
  long long nrec = 0, nw = 0, nh = 0, nb = 0;
  bool on_device = false;
  void release() {
    pool_free(d_rec); pool_free(d_w); pool_free(d_h); pool_free(d_beta);
    d_rec = nullptr; d_w = d_h = d_beta = nullptr;
  }
};
}  // namespace catn_capi

struct catn_batch {
  catn::Image im;
  catn_capi::DeviceRun R;
  long long arena = 0;
  catn_capi::GradRun* grad = nullptr;
  catn_capi::IsingParams ip;
};

#define CUDA_TRY(expr)                                                \
  do {                                                                \
    cudaError_t _e = (expr);                                          \
    if (_e != cudaSuccess) return catn_capi::cuda_fail(_e, #expr);    \
  } while (0)
