// libcatn_b200: the adjoint entry points (catn_ising_grad,
// catn_batch_grad_launch / catn_batch_grad_results).
//
// A gradient run is the persistent kernel with the tape on: every CTA
// contracts its instances with an append-only heap, walks the tape backwards
// (adjoint.cuh) and writes d lnZ / d(input site) into a gradient image laid
// out like the input data; the host maps those to d lnZ / d w and d lnZ / d h
// (ising_param_grad).  This unit compiles the engine on its own so that the
// forward kernel's register allocation (capi.cu) is unaffected.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>
#include <string>
#include "adjoint.cuh"
#include "capi_internal.h"

using namespace catn;
using namespace catn_capi;

namespace {

// Like the forward kernel, the last `nhelp` CTAs (every CTA but one for a
// single network) only help the Jacobi sweeps of the taped contractions'
// large SVDs, and CTAs that find the queue drained join them.
__global__ void __launch_bounds__(kThreads) catn_grad_kernel(
    const InstDesc* __restrict__ descs, const int* __restrict__ order, int ninst, const long long* i64,
    const int* i32, const double* dat, char* slots, SlotLayout L, catn_result* res, double* gimg, int* queue,
    JacobiJob* board, int nhelp, JobLink jl, int use_tc, long long sws_doubles) {
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
    run_instance_grad(T, slot, L, descs[inst], i64, i32, dat, res + inst, gimg, sws, sws_doubles,
                      board ? &jl : nullptr);
    if (board && threadIdx.x == 0) atomicAdd(queue + 1, 1);
    // A shared wait that ran out leaves a helper warp that may still write
    // into this slot's arena: the slot takes no further instance (the other
    // CTAs drain the queue).
    if (T.bcast(threadIdx.x == 0 ? res[inst].status : 0) == CATN_ETIMEOUT) break;
  }
  if (board) {
    if (jl.cta_jobs)
      help_jobs(T, board, (int)gridDim.x, queue + 1, ninst, sws);
    else
      help_jacobi(T, board, (int)gridDim.x, queue + 1, ninst);
  }
  tc_teardown(T);
}

// A gradient run holds the scratch stack, the tape, the append-only heap and
// its shadow: 2.5x the forward arena, at most half of the free device memory
// per slot.
long long grad_arena(long long forward_arena, int slots) {
  long long a = forward_arena / 2 * 5;
  size_t freeb = 0, totalb = 0;
  if (cudaMemGetInfo(&freeb, &totalb) == cudaSuccess && slots > 0) {
    freeb += pool_cached_bytes(false);   // cached blocks are given back when an allocation needs them
    a = std::min(a, (long long)(freeb / 2 / (size_t)slots) & ~255LL);
  }
  return a;
}

catn_status grad_prepare(const Image& im, long long arena, int max_slots, GradRun*& g) {
  if (g && g->arena == arena) return CATN_OK;
  grad_release(g);
  g = new GradRun();
  g->arena = arena;
  if (catn_status s = prepare(im, arena, max_slots, g->R)) {
    grad_release(g);
    g = nullptr;
    return s;
  }
  const size_t gbytes = sizeof(double) * (im.dat.size() + 1);
  CUDA_TRY(pool_new(&g->d_gimg, gbytes));
  CUDA_TRY(pool_new(&g->h_gimg, gbytes, true));
  CUDA_TRY(cudaFuncSetAttribute(catn_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytesTc));
  return CATN_OK;
}

catn_status grad_launch(GradRun* g, cudaStream_t st) {
  if (catn_status s = upload(g->R, st)) return s;
  CUDA_TRY(cudaMemsetAsync(g->R.d_queue, 0, 4 * sizeof(int), st));
  if (g->R.d_board) CUDA_TRY(cudaMemsetAsync(g->R.d_board, 0, sizeof(JacobiJob) * g->R.ngrid, st));
  int nhelp = 0;
  JobLink jl;
  helper_config(g->R, true, &jl, &nhelp);
  // Runs without the tensor-core area or block-route items take the smaller
  // shared-memory configuration, which leaves more of the SM to L1 (as the
  // lean forward kernel does).
  const bool small = !g->R.use_tc && !g->R.cta_jobs;
  catn_grad_kernel<<<g->R.ngrid, kThreads, g->R.use_tc ? kSmemBytesTc : (small ? kSmemBytesLean : kSmemBytes), st>>>(
      g->R.d_desc, g->R.d_order, g->R.ninst, g->R.d_i64, g->R.d_i32, g->R.d_dat, g->R.d_slots, g->R.L, g->R.d_res,
      g->d_gimg, g->R.d_queue, g->R.d_board, nhelp, jl, g->R.use_tc, small ? kSwsDoublesLean : kSwsDoubles);
  CUDA_TRY(cudaGetLastError());
  return CATN_OK;
}

// Results and the parameter gradients of every Ising instance, concatenated
// in the order the instances were added.
catn_status grad_results(const Image& im, GradRun* g, catn_result* res, double* dw, double* dh, cudaStream_t st) {
  CUDA_TRY(cudaMemcpyAsync(res, g->R.d_res, sizeof(catn_result) * g->R.ninst, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaMemcpyAsync(g->h_gimg, g->d_gimg, sizeof(double) * im.dat.size(), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  long long eoff = 0, noff = 0;
  for (const IsingSpec& sp : im.ising) {
    const int ne = (int)sp.w.size();
    const catn_result& r = res[sp.inst];
    if (r.status != CATN_OK)
      return fail((catn_status)r.status,
                  "instance " + std::to_string(sp.inst) + " failed: " + status_text(r.status));
    ising_param_grad(sp.n, ne, sp.edges.data(), sp.w.data(), sp.h.data(), sp.beta, sp.pos1, sp.val1, sp.pos2,
                     sp.val2, g->h_gimg + im.desc[sp.inst].data_off, dw + eoff, dh + noff);
    eoff += ne;
    noff += sp.n;
  }
  return CATN_OK;
}

catn_status check_ising_only(const Image& im) {
  if (im.ising.size() != im.desc.size())
    return fail(CATN_EINVAL, "gradients are defined for networks built by the Ising builder only");
  for (const InstDesc& d : im.desc)
    if (d.P.compress) return fail(CATN_EINVAL, "gradients of the compress sweeps are not implemented");
  return CATN_OK;
}

}  // namespace

namespace catn_capi {

void grad_release(GradRun* g) {
  if (!g) return;
  g->R.release();
  pool_free(g->d_gimg);
  pool_free(g->h_gimg);
  delete g;
}

}  // namespace catn_capi

extern "C" {

catn_status catn_ising_grad(catn_net* net, catn_result* res, double* dlnZ_dw, double* dlnZ_dh,
                            int32_t ckpt_interval) {
  if (!net || !res || !dlnZ_dh || (!dlnZ_dw && !net->im.ising.empty() && !net->im.ising[0].w.empty()))
    return fail(CATN_EINVAL, "NULL argument");
  if (ckpt_interval < 0) return fail(CATN_EINVAL, "ckpt_interval must be >= 0");
  if (catn_status s = check_ising_only(net->im)) return s;
  if (!net->cuts.empty()) return fail(CATN_EINVAL, "gradients of a network with cut_bondim! calls are not taped");
  if (catn_status s = grad_prepare(net->im, net->grad ? net->grad->arena : grad_arena(net->R.L.arena_bytes, 1), 1,
                                      net->grad)) return s;
  // this call's interval, in the uploaded instance descriptor
  ((InstDesc*)net->grad->R.h_input)[0].P.ckpt_interval = ckpt_interval;
  cudaStream_t st = 0;
  if (catn_status s = grad_launch(net->grad, st)) return s;
  return grad_results(net->im, net->grad, res, dlnZ_dw, dlnZ_dh, st);
}

catn_status catn_batch_grad_launch(catn_batch* b, void* stream) {
  if (!b) return fail(CATN_EINVAL, "NULL batch");
  if (catn_status s = check_ising_only(b->im)) return s;
  if (b->ip.on_device)
    return fail(CATN_ESTATE,
                "gradients use the parameters given at creation: catn_batch_upload restores them, or create a "
                "batch from the new parameters");
  if (catn_status s = grad_prepare(b->im, b->grad ? b->grad->arena : grad_arena(b->arena, b->R.nslots), b->R.nslots,
                                      b->grad)) return s;
  return grad_launch(b->grad, (cudaStream_t)stream);
}

catn_status catn_batch_grad_results(catn_batch* b, catn_result* results, double* dlnZ_dw, double* dlnZ_dh,
                                    void* stream) {
  if (!b || !results || !dlnZ_dh) return fail(CATN_EINVAL, "NULL argument");
  if (!b->grad) return fail(CATN_ESTATE, "catn_batch_grad_results before catn_batch_grad_launch");
  return grad_results(b->im, b->grad, results, dlnZ_dw, dlnZ_dh, (cudaStream_t)stream);
}

}  // extern "C"
