// libcatn_b200: C ABI over the device engine (engine.cuh).
//
// One persistent kernel runs every instance of a launch: each CTA owns one
// "slot" of HBM (control state + tensor arena), pulls instance ids from a
// device-side atomic work queue and contracts them start to finish.  A
// single network (catn_net) is the same kernel with one instance and one
// slot that stays resident afterwards for result_tensor.
#include <cuda_runtime.h>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>
#include "engine.cuh"
#include "host_image.h"
#include "capi_internal.h"
#include "persistent.cuh"

using namespace catn;
using namespace catn_capi;

namespace catn_capi {

thread_local std::string g_err;

catn_status fail(catn_status s, const std::string& msg) {
  g_err = msg;
  return s;
}
catn_status cuda_fail(cudaError_t e, const char* what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  return CATN_ECUDA;
}

const char* status_text(int s) {
  switch (s) {
    case CATN_OK: return "ok";
    case CATN_EINVAL: return "invalid argument";
    case CATN_ENOMEM: return "device arena or control capacity exhausted";
    case CATN_ENOCONV: return "Jacobi SVD did not converge";
    case CATN_ETIMEOUT: return "device wait timed out";
    case CATN_ECUDA: return "CUDA error";
    case CATN_ESTATE: return "reference error path (invalid network state)";
  }
  return "unknown";
}

catn_status check_params(const catn_params* p) {
  if (!p) return fail(CATN_EINVAL, "params is NULL");
  if (p->chi < 1) return fail(CATN_EINVAL, "chi must be >= 1");
  if (p->Dmax == 0) return fail(CATN_EINVAL, "Dmax must be nonzero (negative = exact mode)");
  if (p->norm_method < 0 || p->norm_method > 2) return fail(CATN_EINVAL, "norm_method must be 0, 1 or 2");
  if (p->select < 0 || p->select > 2) return fail(CATN_EINVAL, "select must be 0, 1 or 2");
  if (!(p->cutoff >= 0.0)) return fail(CATN_EINVAL, "cutoff must be >= 0");
  if (p->rsvd < 0 || p->rsvd > 2) return fail(CATN_EINVAL, "rsvd must be 0, 1 or 2");
  if (p->rsvd_min_dim < 0) return fail(CATN_EINVAL, "rsvd_min_dim must be >= 0");
  if (p->precision < 0 || p->precision > 1) return fail(CATN_EINVAL, "precision must be 0 (FP64) or 1 (split)");
  if (p->svd_route < 0 || p->svd_route > 2) return fail(CATN_EINVAL, "svd_route must be 0, 1 or 2");
  if (p->ckpt_interval < 0) return fail(CATN_EINVAL, "ckpt_interval must be >= 0");
  if (p->braket_loops < 0 || p->braket_loops > 1) return fail(CATN_EINVAL, "braket_loops must be 0 or 1");
  return CATN_OK;
}

}  // namespace catn_capi

namespace {

// Batch launches keep kHelperCtas CTAs that only help the large SVDs of the
// others, and open the Jacobi sweeps of SVDs with at least kSharedJacobiMinN
// columns to them: a launch lasts as long as its slowest instance (whose
// largest SVDs dominate it) or as the work left to the other CTAs, whichever
// is longer.  Measured on the
// 512-instance spin-glass batch (ms per launch, with shared Jacobi pairs held
// in registers): pool 8 / 12 / 16 / 20 / 24 at threshold 128: 309 / 306 / 307
// / 316 / 324; pool 16 at threshold 64 / 96: 312 / 312.  The pool's size
// trades the slowest instance (320 ms at 8, 290 ms at 24) against the work
// left to the other CTAs.
// The process-wide tuning table (catn_tuning_set) overrides both, and the
// element threshold for Householder work.
constexpr int kSharedJacobiMinN = 128;
constexpr int kHelperCtas = 16;

__global__ void __launch_bounds__(kThreads) catn_result_tensor_kernel(
    char* slot, SlotLayout L, catn_params P, int n, double* out, long long cap, long long* meta) {
  extern __shared__ double smem[];
  Team T;
  T.red = smem;
  T.stage = (char*)(smem + 64);
  T.stage_bytes = GEMM_STAGE_BYTES;
  T.tcs = nullptr;
  T.tmem = 0;
  Ctx C = make_ctx(T, slot, L, P, n, (double*)(T.stage + GEMM_STAGE_BYTES), kSwsDoubles);
  int nd = 0;
  long long dims[64];
  long long tot = result_tensor_dev(C, out, cap, dims, &nd);
  if (threadIdx.x == 0) {
    meta[0] = tot;
    meta[1] = nd;
    meta[2] = C.ctl[CTL_STATUS];
    for (int q = 0; q < nd && q < 64; ++q) meta[3 + q] = dims[q];
  }
}

}  // namespace

namespace catn_capi {

catn_status prepare(const Image& im, long long arena_bytes, int max_slots, DeviceRun& R, bool single_forward) {
  R.ninst = (int)im.desc.size();
  if (R.ninst == 0) return fail(CATN_EINVAL, "no instances");
  R.use_tc = 0;
  R.cta_jobs = 0;
  R.lean = 1;
  for (const InstDesc& d : im.desc) {
    if (d.P.precision == 1) R.use_tc = 1;
    if (d.P.svd_route == 2 || (d.P.svd_route == 0 && d.P.precision == 1)) R.cta_jobs = 1;
    if (d.P.precision != 0 || d.P.svd_route == 2 || d.P.rsvd == 2 || d.kind == 2) R.lean = 0;
  }
  if (R.lean) CUDA_TRY(persistent_lean_attr());
  R.L = make_layout(im.nmax, default_maxs(im), im.emax + 64, arena_bytes);
  int dev = 0, nsm = 0, per_sm = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  CUDA_TRY(cudaFuncSetAttribute(catn_persistent_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytesTc));
  CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, catn_persistent_kernel<0>, kThreads, kSmemBytes));
  if (per_sm < 1) per_sm = 1;
  long long resident = (long long)nsm * per_sm;
  long long ns = R.ninst < resident ? R.ninst : resident;
  if (max_slots > 0 && ns > max_slots) ns = max_slots;
  size_t freeb = 0, totalb = 0;
  CUDA_TRY(cudaMemGetInfo(&freeb, &totalb));
  freeb += pool_cached_bytes(false);   // cached blocks are given back when an allocation needs them
  long long budget = (long long)(freeb * 0.85);
  if (ns * R.L.slot_bytes > budget) ns = budget / R.L.slot_bytes;
  if (ns < 1) return fail(CATN_ENOMEM, "not enough device memory for one slot");
  R.nslots = (int)ns;
  // one network: the other resident CTAs only help its large SVDs (no slots)
  R.ngrid = (R.ninst == 1 && ns == 1 && resident > 1) ? (int)resident : (int)ns;
  const long long b_desc = align256((long long)(sizeof(InstDesc) * im.desc.size())) +
                           align256((long long)(sizeof(int) * im.desc.size()));
  std::vector<int> order(im.desc.size());
  for (size_t q = 0; q < order.size(); ++q) order[q] = (int)q;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return im.desc[a].cost > im.desc[b].cost; });
  const long long b_i64 = align256((long long)(sizeof(long long) * (im.i64.size() + 1)));
  const long long b_i32 = align256((long long)(sizeof(int) * (im.i32.size() + 1)));
  const long long b_dat = align256((long long)(sizeof(double) * (im.dat.size() + 1)));
  R.input_bytes = b_desc + b_i64 + b_i32 + b_dat;
  CUDA_TRY(pool_new(&R.h_input, (size_t)R.input_bytes, true));
  CUDA_TRY(pool_new(&R.d_input, (size_t)R.input_bytes));
  std::memset(R.h_input, 0, (size_t)R.input_bytes);
  std::memcpy(R.h_input, im.desc.data(), sizeof(InstDesc) * im.desc.size());
  const long long off_order = align256((long long)(sizeof(InstDesc) * im.desc.size()));
  std::memcpy(R.h_input + off_order, order.data(), sizeof(int) * order.size());
  if (!im.i64.empty()) std::memcpy(R.h_input + b_desc, im.i64.data(), sizeof(long long) * im.i64.size());
  if (!im.i32.empty()) std::memcpy(R.h_input + b_desc + b_i64, im.i32.data(), sizeof(int) * im.i32.size());
  if (!im.dat.empty()) std::memcpy(R.h_input + b_desc + b_i64 + b_i32, im.dat.data(), sizeof(double) * im.dat.size());
  // One network contracted on its own in FP64 on the auto route takes the
  // block Jacobi route for its large factors, since every other CTA of the
  // GPU is then free to help it (measured, FP64 block against scalar route:
  // 16.5 vs 41 s per beta on the n = 200 random-regular graph, 25.7 vs 31.1 s
  // on the 32 x 32 Gaussian lattice, 8.2 vs 21.2 s on a 6 x 6 PEPS double
  // layer, traces identical); batches and gradient runs keep the scalar route.
  if (single_forward && R.ninst == 1) {
    InstDesc* hd = (InstDesc*)R.h_input;
    if (hd[0].kind != 2 && hd[0].P.svd_route == 0 && hd[0].P.precision == 0) {
      hd[0].P.svd_route = 2;
      R.cta_jobs = 1;
      R.lean = 0;
    }
  }
  R.d_desc = (InstDesc*)R.d_input;
  R.d_order = (int*)(R.d_input + off_order);
  R.d_i64 = (long long*)(R.d_input + b_desc);
  R.d_i32 = (int*)(R.d_input + b_desc + b_i64);
  R.d_dat = (double*)(R.d_input + b_desc + b_i64 + b_i32);
  CUDA_TRY(pool_new(&R.d_slots, (size_t)(R.L.slot_bytes * ns)));
  CUDA_TRY(pool_new(&R.d_res, sizeof(catn_result) * im.desc.size()));
  CUDA_TRY(pool_new(&R.d_trace, sizeof(int) * (im.trace_total + 8)));
  CUDA_TRY(pool_new(&R.d_queue, 4 * sizeof(int)));
  if (R.ngrid > 1) CUDA_TRY(pool_new(&R.d_board, sizeof(JacobiJob) * R.ngrid));
  return CATN_OK;
}

// The tuning table in force (entries < 0: built-in defaults).
std::mutex g_tuning_mu;
catn_tuning g_tuning = {-1, -1, -1, -1, -1, -1, 0};

catn_tuning tuning_now() {
  std::lock_guard<std::mutex> lock(g_tuning_mu);
  catn_tuning t = g_tuning;
  if (t.helper_ctas < 0) t.helper_ctas = kHelperCtas;
  if (t.grad_helper_ctas < 0) t.grad_helper_ctas = kGradHelperCtas;
  if (t.shared_jacobi_min_n < 0) t.shared_jacobi_min_n = kSharedJacobiMinN;
  if (t.block_min_n < 0) t.block_min_n = (int32_t)catn::kBlockMinN;
  if (t.shared_house_min < 0) t.shared_house_min = kSharedHouseMinElems;
  if (t.blocked_qr_min_n < 0) t.blocked_qr_min_n = 1 << 30;
  return t;
}

void helper_config(const DeviceRun& R, bool grad, JobLink* jl, int* nhelp) {
  const catn_tuning t = tuning_now();
  int h = grad ? t.grad_helper_ctas : t.helper_ctas;
  if (!R.d_board || h < 0 || 4 * h > R.nslots || 4 * h > R.ninst) h = 0;
  if (R.d_board && R.ngrid > R.nslots) h = R.ngrid - R.nslots;
  *nhelp = h;
  jl->job = nullptr;
  jl->qhead = nullptr;
  jl->ninst = R.ninst;
  jl->min_n = std::max(2, (int)t.shared_jacobi_min_n);
  jl->pool = h > 0;
  jl->min_qr = std::max(1LL, (long long)t.shared_house_min);
  jl->block_min_n = std::max(4, (int)t.block_min_n);
  jl->blocked_qr_min_n = std::max(4, (int)t.blocked_qr_min_n);
  jl->cta_jobs = R.cta_jobs;
}

catn_status upload(DeviceRun& R, cudaStream_t st) {
  CUDA_TRY(cudaMemcpyAsync(R.d_input, R.h_input, (size_t)R.input_bytes, cudaMemcpyHostToDevice, st));
  return CATN_OK;
}

// Arena of a single network when the caller passes 0: the largest two-site
// matrix a swap can form is (chi*Dmax)^2 doubles, and a full-rank SVD of it
// holds five such buffers on the scratch stack (40 % of the arena) beside
// the scratch of the operations around it, so take 32x that matrix, at
// least 1 GiB and at most 48 GiB or a quarter of the free device memory.  Exact mode (Dmax < 0) keeps 1 GiB: its networks are
// small by construction.
long long default_arena(long long a, const catn_params& p) {
  if (a > 0) return a;
  long long arena = 1LL << 30;
  if (p.Dmax > 0) {
    const long long m = (long long)std::min(p.chi, 16384) * std::min(p.Dmax, 16384);
    arena = std::max(arena, 32 * 8 * m * m);
  }
  arena = std::min(arena, 48LL << 30);
  size_t freeb = 0, totalb = 0;
  if (cudaMemGetInfo(&freeb, &totalb) == cudaSuccess)
    arena = std::min(arena, (long long)((freeb + pool_cached_bytes(false)) / 4));
  return std::max(arena, 1LL << 30);
}

}  // namespace catn_capi

namespace {

catn_status launch(DeviceRun& R, cudaStream_t st) {
  CUDA_TRY(cudaMemsetAsync(R.d_queue, 0, 4 * sizeof(int), st));
  if (R.d_board) CUDA_TRY(cudaMemsetAsync(R.d_board, 0, sizeof(JacobiJob) * R.ngrid, st));
  int nhelp = 0;
  JobLink jl;
  helper_config(R, false, &jl, &nhelp);
  if (R.lean) {
    CUDA_TRY(persistent_lean_launch(R, nhelp, jl, st));
    return CATN_OK;
  }
  catn_persistent_kernel<0><<<R.ngrid, kThreads, R.use_tc ? kSmemBytesTc : kSmemBytes, st>>>(
      R.d_desc, R.d_order, R.ninst, R.d_i64, R.d_i32, R.d_dat, R.d_slots, R.L, R.d_res, R.d_trace, R.d_queue,
      R.d_board, nhelp, jl, R.use_tc);
  CUDA_TRY(cudaGetLastError());
  return CATN_OK;
}

// Site tensors of an Ising batch rebuilt from the batch's device copies of
// couplings, fields and betas (ising_build.cuh), one recipe per thread.
__global__ void catn_ising_fill_kernel(const IsingSiteRecipe* rec, long long nrec, const double* w,
                                       const double* h, const double* beta, double* dat) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nrec;
       q += (long long)gridDim.x * blockDim.x) {
    const IsingSiteRecipe r = rec[q];
    double v[8];
    const int c = ising_site_values(r, r.edge >= 0 ? w[r.edge] : 0.0, h[r.node], beta[r.inst], v);
    for (int k = 0; k < c; ++k) dat[r.dat + k] = v[k];
  }
}

// Couplings sigma_w N(0,1) (stream 0) and fields sigma_h N(0,1) (stream 1).
__global__ void catn_disorder_kernel(unsigned long long seed, double sigma_w, double sigma_h, double* w,
                                     long long nw, double* h, long long nh) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nw || q < nh;
       q += (long long)gridDim.x * blockDim.x) {
    if (q < nw) w[q] = sigma_w * disorder_normal(seed, 0, (unsigned long long)q);
    if (q < nh) h[q] = sigma_h * disorder_normal(seed, 1, (unsigned long long)q);
  }
}

catn_status params_restore(catn_batch* b, cudaStream_t st);

// Device copies of the creation parameters and the site recipes.
catn_status params_prepare(catn_batch* b, const double* weights, const double* fields, const double* betas,
                           long long nw, long long nh, long long nb) {
  IsingParams& P = b->ip;
  P.nrec = (long long)b->im.recipes.size();
  P.nw = nw;
  P.nh = nh;
  P.nb = nb;
  if (P.nrec == 0) return CATN_OK;
  CUDA_TRY(pool_new(&P.d_rec, sizeof(IsingSiteRecipe) * P.nrec));
  CUDA_TRY(pool_new(&P.d_w, sizeof(double) * std::max(nw, 1LL)));
  CUDA_TRY(pool_new(&P.d_h, sizeof(double) * std::max(nh, 1LL)));
  CUDA_TRY(pool_new(&P.d_beta, sizeof(double) * std::max(nb, 1LL)));
  CUDA_TRY(cudaMemcpy(P.d_rec, b->im.recipes.data(), sizeof(IsingSiteRecipe) * P.nrec, cudaMemcpyHostToDevice));
  return params_restore(b, nullptr);
}
// The device parameter copies back to the creation values (the host image
// holds the networks built from them).
catn_status params_restore(catn_batch* b, cudaStream_t st) {
  IsingParams& P = b->ip;
  std::vector<double> w, h, be;
  for (const IsingSpec& sp : b->im.ising) {
    w.insert(w.end(), sp.w.begin(), sp.w.end());
    h.insert(h.end(), sp.h.begin(), sp.h.end());
    be.push_back(sp.beta);
  }
  if ((long long)w.size() != P.nw || (long long)h.size() != P.nh || (long long)be.size() != P.nb)
    return fail(CATN_ESTATE, "batch parameter counts disagree with its instances");
  if (P.nw > 0) CUDA_TRY(cudaMemcpyAsync(P.d_w, w.data(), sizeof(double) * P.nw, cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(P.d_h, h.data(), sizeof(double) * P.nh, cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(P.d_beta, be.data(), sizeof(double) * P.nb, cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  P.on_device = false;
  return CATN_OK;
}
// Rebuild every site from the device parameters.
catn_status params_fill(catn_batch* b, cudaStream_t st) {
  IsingParams& P = b->ip;
  const int grid = (int)std::min<long long>((P.nrec + 255) / 256, 4096);
  catn_ising_fill_kernel<<<grid > 0 ? grid : 1, 256, 0, st>>>(P.d_rec, P.nrec, P.d_w, P.d_h, P.d_beta, b->R.d_dat);
  CUDA_TRY(cudaGetLastError());
  P.on_device = true;
  return CATN_OK;
}

}  // namespace


extern "C" {

void catn_params_default(catn_params* p) {
  if (!p) return;
  p->Dmax = 32;
  p->chi = 32;
  p->cutoff = 1e-15;
  p->norm_method = 1;
  p->select = 1;
  p->reverse = 1;
  p->svdopt = 1;
  p->swapopt = 1;
  p->compress = 0;
  p->cut_bond = 0;
  p->seed = 1;
  p->trace = 0;
  p->rsvd = 0;
  p->rsvd_min_dim = 0;
  p->precision = 0;
  p->svd_route = 0;
  p->ckpt_interval = 0;
  p->braket_loops = 0;
}

catn_status catn_tuning_get(catn_tuning* t) {
  if (!t) return fail(CATN_EINVAL, "NULL argument");
  *t = tuning_now();
  return CATN_OK;
}

catn_status catn_tuning_set(const catn_tuning* t) {
  if (!t) return fail(CATN_EINVAL, "NULL argument");
  if (t->helper_ctas > 4096 || t->grad_helper_ctas > 4096) return fail(CATN_EINVAL, "helper pool above 4096 CTAs");
  if (t->block_min_n >= 0 && t->block_min_n < 4) return fail(CATN_EINVAL, "block_min_n must be >= 4 (or < 0)");
  std::lock_guard<std::mutex> lock(g_tuning_mu);
  g_tuning = *t;
  return CATN_OK;
}

static catn_status net_finish(catn_net* net, long long arena_bytes, catn_net** out) {
  if (net->im.desc.empty()) {
    delete net;
    return fail(CATN_EINVAL, "no instances");
  }
  net->arena = default_arena(arena_bytes, net->im.desc[0].P);
  catn_status s = prepare(net->im, net->arena, 1, net->R, true);
  if (s != CATN_OK) {
    net->R.release();
    delete net;
    return s;
  }
  *out = net;
  return CATN_OK;
}

catn_status catn_net_create_mps(const catn_params* p, int32_t n_nodes, const int32_t* site_counts,
                                const int32_t* nbr_counts, const int32_t* canos, const int64_t* site_dims,
                                const double* site_data, const int32_t* neighbors, int64_t arena_bytes,
                                catn_net** out) {
  if (catn_status s = check_params(p)) return s;
  if (!out || !site_counts || !nbr_counts || !canos) return fail(CATN_EINVAL, "NULL argument");
  catn_net* net = new catn_net();
  int tc = p->trace ? 4 * 1024 * 64 : 0;
  long long nsite = 0;
  for (int k = 0; k < n_nodes; ++k) nsite += site_counts[k];
  if (p->trace) tc = (int)(nsite + 16);
  std::string e = net->im.add_mps(*p, n_nodes, site_counts, nbr_counts, canos, (const long long*)site_dims,
                                  site_data, neighbors, tc);
  if (!e.empty()) { delete net; return fail(CATN_EINVAL, e); }
  return net_finish(net, arena_bytes, out);
}

catn_status catn_net_create_dense(const catn_params* p, int32_t n_nodes, const int32_t* ndims, const int64_t* dims,
                                  const double* data, const int32_t* neighbors, int64_t arena_bytes,
                                  catn_net** out) {
  if (catn_status s = check_params(p)) return s;
  if (!out || !ndims) return fail(CATN_EINVAL, "NULL argument");
  catn_net* net = new catn_net();
  long long legs = 0;
  for (int k = 0; k < n_nodes; ++k) legs += ndims[k];
  int tc = p->trace ? (int)(legs + 16) : 0;
  std::string e = net->im.add_dense(*p, n_nodes, ndims, (const long long*)dims, data, neighbors, tc);
  if (!e.empty()) { delete net; return fail(CATN_EINVAL, e); }
  return net_finish(net, arena_bytes, out);
}

catn_status catn_ising_create(const catn_params* p, int32_t n, int32_t n_edges, const int32_t* edges,
                              const double* weights, const double* fields, double beta, int32_t pos1,
                              int32_t val1, int32_t pos2, int32_t val2, int64_t arena_bytes, catn_net** out) {
  if (catn_status s = check_params(p)) return s;
  if (!out || (n_edges > 0 && (!edges || !weights)) || !fields) return fail(CATN_EINVAL, "NULL argument");
  catn_net* net = new catn_net();
  int tc = p->trace ? 2 * n_edges + 16 : 0;
  std::string e = net->im.add_ising(*p, n, n_edges, edges, weights, fields, beta, pos1, val1, pos2, val2, tc);
  if (!e.empty()) { delete net; return fail(CATN_EINVAL, e); }
  return net_finish(net, arena_bytes, out);
}

catn_status catn_braket_create(const catn_params* p, int32_t n, const int32_t* ndims, const int64_t* dims,
                               const double* data, const int32_t* labels, int64_t arena_bytes, catn_net** out) {
  if (catn_status s = check_params(p)) return s;
  if (!out || !ndims || !dims || !data || !labels) return fail(CATN_EINVAL, "NULL argument");
  catn_net* net = new catn_net();
  long long legs = 0;
  for (int k = 0; k < n; ++k) legs += ndims[k];
  const int tc = p->trace ? (int)(legs + 16) : 0;
  std::string e = net->im.add_braket(*p, n, ndims, (const long long*)dims, data, labels, tc);
  if (!e.empty()) { delete net; return fail(CATN_EINVAL, e); }
  return net_finish(net, arena_bytes, out);
}

catn_status catn_contract(catn_net* net, catn_result* res, int32_t* trace, int32_t trace_cap) {
  if (!net || !res) return fail(CATN_EINVAL, "NULL argument");
  if (net->contracted) return fail(CATN_ESTATE, "network already contracted (contraction! consumes tn)");
  if (net->unusable) return fail(CATN_ESTATE, "network lost its device copy in a failed cut_bondim!");
  cudaStream_t st = 0;
  if (catn_status s = upload(net->R, st)) return s;
  if (net->im.desc[0].kind == 2) {
    if (catn_status s = braket_launch(net->R, st)) return s;
  } else if (catn_status s = launch(net->R, st)) {
    return s;
  }
  CUDA_TRY(cudaMemcpyAsync(res, net->R.d_res, sizeof(catn_result), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  net->contracted = true;
  if (trace && trace_cap > 0 && net->im.desc[0].trace_cap > 0) {
    int cnt = res->nsteps < trace_cap ? res->nsteps : trace_cap;
    if (cnt > net->im.desc[0].trace_cap) cnt = net->im.desc[0].trace_cap;
    if (cnt > 0) CUDA_TRY(cudaMemcpy(trace, net->R.d_trace, sizeof(int) * 8 * cnt, cudaMemcpyDeviceToHost));
  }
  if (res->status != CATN_OK) return fail((catn_status)res->status, std::string("contraction failed: ") + status_text(res->status));
  return CATN_OK;
}

catn_status catn_cut_bondim(catn_net* net, int32_t i, int32_t idx_j_in_i, int32_t opt, double* err) {
  if (!net || !err) return fail(CATN_EINVAL, "NULL argument");
  *err = 0.0;
  if (net->contracted) return fail(CATN_ESTATE, "network already contracted (contraction! consumes tn)");
  if (net->unusable) return fail(CATN_ESTATE, "network lost its device copy in a failed cut_bondim!");
  const InstDesc& D0 = net->im.desc[0];
  if (D0.kind == 2) return fail(CATN_EINVAL, "cut_bondim!: BraKet networks have no bond cuts");
  if (D0.P.Dmax < 0) return CATN_OK;   // tensor_network.jl:344 (and :401): a no-op returning 0.0
  const char* name = opt ? "cut_bondim_opt!" : "cut_bondim!";
  if (i < 1 || i > D0.n) return fail(CATN_EINVAL, std::string(name) + ": node id out of range");
  const std::vector<int> nbi = net->im.neighbors_of(i);
  if (idx_j_in_i < 1 || idx_j_in_i > (int)nbi.size()) return fail(CATN_EINVAL, std::string(name) + ": leg out of range");
  const int j = nbi[idx_j_in_i - 1];
  if (j <= 0)
    return fail(CATN_ESTATE, std::string(name) + ": leg " + std::to_string(idx_j_in_i) + " of node " +
                                 std::to_string(i) + " is an open leg (no neighbor)");
  const std::vector<int> nbj = net->im.neighbors_of(j);
  if (std::find(nbj.begin(), nbj.end(), i) == nbj.end())
    return fail(CATN_ESTATE, std::string(name) + ": node " + std::to_string(i) + " not found as neighbor of node " +
                                 std::to_string(j));
  // The network's state is its image plus the cuts so far: the launch loads
  // the image, replays every cut in order and stops after the new one.
  std::vector<int> cuts = net->cuts;
  cuts.push_back(i);
  cuts.push_back(idx_j_in_i);
  cuts.push_back(opt ? 1 : 0);
  net->im.set_cuts(cuts);
  net->im.desc[0].cut_only = 1;
  net->R.release();
  catn_status s = prepare(net->im, net->arena, 1, net->R, true);
  net->im.desc[0].cut_only = 0;
  if (s != CATN_OK) {
    net->im.set_cuts(net->cuts);
    net->R.release();
    if (prepare(net->im, net->arena, 1, net->R, true) != CATN_OK) net->unusable = true;
    return s;
  }
  cudaStream_t st = 0;
  catn_result res;
  std::memset(&res, 0, sizeof(res));
  if ((s = upload(net->R, st)) == CATN_OK && (s = launch(net->R, st)) == CATN_OK) {
    cudaError_t e = cudaMemcpyAsync(&res, net->R.d_res, sizeof(catn_result), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) s = cuda_fail(e, "cut_bondim! result");
  }
  if (s == CATN_OK && res.status != CATN_OK)
    s = fail((catn_status)res.status, std::string(name) + " failed: " + status_text(res.status));
  // the host copy of the image goes back to contraction launches, without
  // the new cut when it did not complete (the earlier cuts are replayed)
  InstDesc* hd = (InstDesc*)net->R.h_input;
  hd[0].cut_only = 0;
  if (s != CATN_OK) {
    net->im.set_cuts(net->cuts);
    hd[0].n_cuts = net->im.desc[0].n_cuts;
    return s;
  }
  net->cuts = cuts;
  *err = res.err;
  return CATN_OK;
}

catn_status catn_result_tensor(catn_net* net, double* out, int64_t cap, int64_t* numel, int32_t* ndim, int64_t* dims) {
  if (!net || !numel || !ndim) return fail(CATN_EINVAL, "NULL argument");
  if (!net->contracted) return fail(CATN_ESTATE, "result_tensor before contraction!");
  long long total_cap = cap > 0 ? cap : 0;
  double* d_out = nullptr;
  long long* d_meta = nullptr;
  CUDA_TRY(cudaMalloc(&d_meta, sizeof(long long) * 80));
  if (total_cap > 0) CUDA_TRY(cudaMalloc(&d_out, sizeof(double) * total_cap));
  cudaFuncSetAttribute(catn_result_tensor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
  catn_result_tensor_kernel<<<1, kThreads, kSmemBytes>>>(net->R.d_slots, net->R.L, net->im.desc[0].P,
                                                        net->im.desc[0].n, d_out, total_cap, d_meta);
  cudaError_t e = cudaGetLastError();
  long long meta[80];
  if (e == cudaSuccess) e = cudaMemcpy(meta, d_meta, sizeof(meta), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && out && meta[0] > 0 && meta[0] <= total_cap)
    e = cudaMemcpy(out, d_out, sizeof(double) * meta[0], cudaMemcpyDeviceToHost);
  cudaFree(d_out);
  cudaFree(d_meta);
  if (e != cudaSuccess) return cuda_fail(e, "result_tensor");
  if (meta[0] < 0 || meta[2] != 0)
    return fail(CATN_ESTATE, "result_tensor: expected one surviving open-leg node");
  *numel = meta[0] == 0 ? 1 : meta[0];
  *ndim = (int)meta[1];
  for (int q = 0; q < meta[1] && q < 64; ++q)
    if (dims) dims[q] = meta[3 + q];
  if (meta[0] == 0 && out && cap >= 1) out[0] = 1.0;   // closed network: 0-d one()
  return CATN_OK;
}

catn_status catn_net_destroy(catn_net* net) {
  if (!net) return CATN_OK;
  grad_release(net->grad);
  net->R.release();
  delete net;
  return CATN_OK;
}

catn_status catn_ising_batch_create(const catn_params* p, int32_t n_inst, const int32_t* n_nodes,
                                    const int64_t* node_off, const int64_t* edge_off, const int32_t* edges,
                                    const double* weights, const double* fields, const double* betas,
                                    const int32_t* pins, int64_t slot_arena_bytes, int32_t max_slots,
                                    catn_batch** out) {
  if (catn_status s = check_params(p)) return s;
  if (!out || n_inst < 1 || !n_nodes || !node_off || !edge_off || !fields || !betas)
    return fail(CATN_EINVAL, "bad batch arguments");
  catn_batch* b = new catn_batch();
  for (int q = 0; q < n_inst; ++q) {
    long long e0 = edge_off[q], e1 = edge_off[q + 1];
    int ne = (int)(e1 - e0);
    int pos1 = 0, val1 = 0, pos2 = 0, val2 = 0;
    if (pins) { pos1 = pins[4 * q]; val1 = pins[4 * q + 1]; pos2 = pins[4 * q + 2]; val2 = pins[4 * q + 3]; }
    int tc = p->trace ? 2 * ne + 16 : 0;
    std::string e = b->im.add_ising(*p, n_nodes[q], ne, edges + 2 * e0, weights + e0, fields + node_off[q],
                                    betas[q], pos1, val1, pos2, val2, tc, e0, node_off[q]);
    if (!e.empty()) { delete b; return fail(CATN_EINVAL, "instance " + std::to_string(q) + ": " + e); }
  }
  long long arena = slot_arena_bytes > 0 ? slot_arena_bytes : (128LL << 20);
  b->arena = arena;
  if (catn_status s = prepare(b->im, arena, max_slots, b->R)) {
    b->R.release();
    delete b;
    return s;
  }
  if (catn_status s = params_prepare(b, weights, fields, betas, edge_off[n_inst], node_off[n_inst], n_inst)) {
    b->ip.release();
    b->R.release();
    delete b;
    return s;
  }
  *out = b;
  return CATN_OK;
}

catn_status catn_batch_upload(catn_batch* b, void* stream) {
  if (!b) return fail(CATN_EINVAL, "NULL batch");
  if (catn_status s = upload(b->R, (cudaStream_t)stream)) return s;
  if (b->ip.on_device) {   // back to the networks given at creation
    if (catn_status s = params_restore(b, (cudaStream_t)stream)) return s;
  }
  return CATN_OK;
}

catn_status catn_ising_batch_set_params(catn_batch* b, const double* weights, const double* fields,
                                        const double* betas, void* stream) {
  if (!b || !fields || (!weights && b->ip.nw > 0)) return fail(CATN_EINVAL, "NULL argument");
  if (!b->ip.d_rec) return fail(CATN_EINVAL, "not an Ising batch");
  cudaStream_t st = (cudaStream_t)stream;
  if (b->ip.nw > 0)
    CUDA_TRY(cudaMemcpyAsync(b->ip.d_w, weights, sizeof(double) * b->ip.nw, cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(b->ip.d_h, fields, sizeof(double) * b->ip.nh, cudaMemcpyHostToDevice, st));
  if (betas) CUDA_TRY(cudaMemcpyAsync(b->ip.d_beta, betas, sizeof(double) * b->ip.nb, cudaMemcpyHostToDevice, st));
  return params_fill(b, st);
}

catn_status catn_ising_batch_randomize(catn_batch* b, uint64_t seed, double sigma_w, double sigma_h,
                                       void* stream) {
  if (!b) return fail(CATN_EINVAL, "NULL batch");
  if (!b->ip.d_rec) return fail(CATN_EINVAL, "not an Ising batch");
  if (!(sigma_w >= 0.0) || !(sigma_h >= 0.0)) return fail(CATN_EINVAL, "sigma_w and sigma_h must be >= 0");
  cudaStream_t st = (cudaStream_t)stream;
  const long long n = std::max(b->ip.nw, b->ip.nh);
  const int grid = (int)std::min<long long>((n + 255) / 256, 4096);
  catn_disorder_kernel<<<grid > 0 ? grid : 1, 256, 0, st>>>(seed, sigma_w, sigma_h, b->ip.d_w, b->ip.nw, b->ip.d_h,
                                                            b->ip.nh);
  CUDA_TRY(cudaGetLastError());
  return params_fill(b, st);
}

catn_status catn_ising_batch_get_params(const catn_batch* b, double* weights, double* fields, double* betas) {
  if (!b || !fields || !betas || (!weights && b->ip.nw > 0)) return fail(CATN_EINVAL, "NULL argument");
  if (!b->ip.d_rec) return fail(CATN_EINVAL, "not an Ising batch");
  if (b->ip.nw > 0) CUDA_TRY(cudaMemcpy(weights, b->ip.d_w, sizeof(double) * b->ip.nw, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(fields, b->ip.d_h, sizeof(double) * b->ip.nh, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(betas, b->ip.d_beta, sizeof(double) * b->ip.nb, cudaMemcpyDeviceToHost));
  return CATN_OK;
}

int64_t catn_ising_batch_param_bytes(const catn_batch* b) {
  return b ? (int64_t)(sizeof(double) * (b->ip.nw + b->ip.nh + b->ip.nb)) : 0;
}

catn_status catn_batch_launch(catn_batch* b, void* stream) {
  if (!b) return fail(CATN_EINVAL, "NULL batch");
  return launch(b->R, (cudaStream_t)stream);
}

catn_status catn_batch_results(catn_batch* b, catn_result* results, void* stream) {
  if (!b || !results) return fail(CATN_EINVAL, "NULL argument");
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(cudaMemcpyAsync(results, b->R.d_res, sizeof(catn_result) * b->R.ninst, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  for (int q = 0; q < b->R.ninst; ++q)
    if (results[q].status != CATN_OK)
      return fail((catn_status)results[q].status,
                  "instance " + std::to_string(q) + " failed: " + status_text(results[q].status));
  return CATN_OK;
}

catn_status catn_batch_run(catn_batch* b, catn_result* results) {
  if (catn_status s = catn_batch_upload(b, nullptr)) return s;
  if (catn_status s = catn_batch_launch(b, nullptr)) return s;
  return catn_batch_results(b, results, nullptr);
}

int32_t catn_batch_slots(const catn_batch* b) { return b ? b->R.nslots : 0; }
int64_t catn_batch_input_bytes(const catn_batch* b) { return b ? b->R.input_bytes : 0; }

catn_status catn_batch_destroy(catn_batch* b) {
  if (!b) return CATN_OK;
  b->ip.release();
  grad_release(b->grad);
  b->R.release();
  delete b;
  return CATN_OK;
}

size_t catn_last_error(char* buf, size_t cap) {
  if (!buf || cap == 0) return g_err.size();
  size_t n = g_err.size() < cap - 1 ? g_err.size() : cap - 1;
  std::memcpy(buf, g_err.data(), n);
  buf[n] = '\0';
  return n;
}

const char* catn_version(void) { return "catn_b200 0.2 (sm_100a: FP64 engine, 3xTF32 tcgen05 split precision)"; }

}  // extern "C"
