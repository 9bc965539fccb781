// Test-only host build of the device engine (team of one thread), used by the
// CPU test-suite to check the engine's integer bookkeeping and memory safety
// (under AddressSanitizer) against the oracle.  It is not part of
// libcatn_b200 and is never loaded by the product path.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "../../catn.jl_b200/csrc/engine.cuh"
#include "../../catn.jl_b200/csrc/adjoint.cuh"
#include "../../catn.jl_b200/csrc/braket.cuh"
#include "../../catn.jl_b200/csrc/host_image.h"

using namespace catn;

// Shared-memory workspace that the block route's items and the blocked QR's
// panel items use (the library's kernels always have at least this much).
static constexpr long long kItemWsDoubles =
    kBlockWsDoubles > kPanelWsDoubles + kPanelW ? kBlockWsDoubles : kPanelWsDoubles + kPanelW;

static int run_image(Image& im, long long arena_bytes, catn_result* res, int* trace) {
  if (im.desc.empty()) return CATN_EINVAL;
  SlotLayout L = make_layout(im.nmax, default_maxs(im), im.emax + 64, arena_bytes);
  std::vector<char> slot((size_t)L.slot_bytes + 256);
  char* sp = (char*)(((uintptr_t)slot.data() + 255) & ~(uintptr_t)255);
  std::vector<double> red(64);
  Team T;
  T.red = red.data();
  T.stage = nullptr;
  T.stage_bytes = 0;
  T.tcs = nullptr;
  T.tmem = 0;
  std::vector<int> tr((size_t)im.trace_total + 8);
  // stand-in for the GPU's shared-memory SVD workspace (same capacity)
  long long sws_doubles = (98 * 1024 - 64 * 8 - GEMM_STAGE_BYTES) / 8;
  // CATN_HOSTCHECK_SWS overrides the capacity (0 sends every SVD through the
  // large-matrix path, including its rank-revealing truncation)
  if (const char* e = std::getenv("CATN_HOSTCHECK_SWS")) sws_doubles = std::atoll(e);
  // at least the block route's and the blocked QR's item workspaces (as the
  // library's shared memory always holds), whatever capacity is reported
  std::vector<double> sws((size_t)std::max<long long>(sws_doubles, kItemWsDoubles));
  // CATN_HOSTCHECK_JOB=1 sends the Jacobi sweeps of every SVD on the global
  // path through the shared-job protocol (no helpers: the team claims all);
  // CATN_HOSTCHECK_BLOCK_MIN sets the smallest factor on the block route
  JacobiJob job;
  std::memset(&job, 0, sizeof(job));
  const int qhead = 1;
  const char* je = std::getenv("CATN_HOSTCHECK_JOB");
  const bool shared = je && je[0] == '1';
  JobLink jl;
  jl.job = shared ? &job : nullptr;
  jl.qhead = &qhead;
  jl.ninst = 1;
  jl.min_n = shared ? 2 : (1 << 30);
  jl.pool = 0;
  jl.min_qr = shared ? 1 : (1LL << 62);
  jl.block_min_n = kBlockMinN;
  if (const char* eb = std::getenv("CATN_HOSTCHECK_BLOCK_MIN")) jl.block_min_n = std::atoi(eb);
  // CATN_HOSTCHECK_BLOCKED_QR_MIN: the same for the blocked, norm-sorted QR
  jl.blocked_qr_min_n = 1 << 30;
  if (const char* eq = std::getenv("CATN_HOSTCHECK_BLOCKED_QR_MIN")) jl.blocked_qr_min_n = std::atoi(eq);
  jl.cta_jobs = 1;
  run_instance(T, sp, L, im.desc[0], im.i64.data(), im.i32.data(), im.dat.data(), res, tr.data(), sws.data(),
               sws_doubles, &jl);
  if (trace && im.desc[0].trace_cap > 0)
    std::memcpy(trace, tr.data(), sizeof(int) * 8 * (size_t)im.desc[0].trace_cap);
  return res->status;
}

extern "C" {

int catn_hostcheck_ising(const catn_params* p, int n, int n_edges, const int* edges, const double* w,
                         const double* h, double beta, int pos1, int val1, int pos2, int val2,
                         long long arena_bytes, catn_result* res, int* trace, int trace_cap) {
  Image im;
  std::string e = im.add_ising(*p, n, n_edges, edges, w, h, beta, pos1, val1, pos2, val2, trace_cap);
  if (!e.empty()) return CATN_EINVAL;
  return run_image(im, arena_bytes, res, trace);
}

// Gradient run (tape + adjoint) of one Ising network: lnZ in res, d lnZ/d w
// and d lnZ/d h through the host chain rule.
int catn_hostcheck_ising_grad(const catn_params* p, int n, int n_edges, const int* edges, const double* w,
                              const double* h, double beta, int pos1, int val1, int pos2, int val2,
                              long long arena_bytes, catn_result* res, double* dw, double* dh) {
  Image im;
  std::string e = im.add_ising(*p, n, n_edges, edges, w, h, beta, pos1, val1, pos2, val2, 0);
  if (!e.empty()) return CATN_EINVAL;
  SlotLayout L = make_layout(im.nmax, default_maxs(im), im.emax + 64, arena_bytes);
  std::vector<char> slot((size_t)L.slot_bytes + 256);
  char* sp = (char*)(((uintptr_t)slot.data() + 255) & ~(uintptr_t)255);
  std::vector<double> red(64);
  Team T;
  T.red = red.data();
  T.stage = nullptr;
  T.stage_bytes = 0;
  T.tcs = nullptr;
  T.tmem = 0;
  long long sws_doubles = (98 * 1024 - 64 * 8 - GEMM_STAGE_BYTES) / 8;
  if (const char* ev = std::getenv("CATN_HOSTCHECK_SWS")) sws_doubles = std::atoll(ev);
  // at least the block route's and the blocked QR's item workspaces (as the
  // library's shared memory always holds), whatever capacity is reported
  std::vector<double> sws((size_t)std::max<long long>(sws_doubles, kItemWsDoubles));
  std::vector<double> gimg(im.dat.size() + 1, 0.0);
  run_instance_grad(T, sp, L, im.desc[0], im.i64.data(), im.i32.data(), im.dat.data(), res, gimg.data(),
                    sws.data(), sws_doubles);
  if (res->status == CATN_OK)
    ising_param_grad(n, n_edges, edges, w, h, beta, pos1, val1, pos2, val2, gimg.data() + im.desc[0].data_off, dw,
                     dh);
  return res->status;
}

// BraKet network <psi|psi> (catn_braket_create's inputs).
int catn_hostcheck_braket(const catn_params* p, int n, const int* ndims, const long long* dims, const double* data,
                          const int* labels, long long arena_bytes, catn_result* res, int* trace, int trace_cap) {
  Image im;
  std::string e = im.add_braket(*p, n, ndims, dims, data, labels, trace_cap);
  if (!e.empty()) return CATN_EINVAL;
  SlotLayout L = make_layout(im.nmax, default_maxs(im), im.emax + 64, arena_bytes);
  std::vector<char> slot((size_t)L.slot_bytes + 256);
  char* sp = (char*)(((uintptr_t)slot.data() + 255) & ~(uintptr_t)255);
  std::vector<double> red(64);
  Team T;
  T.red = red.data();
  T.stage = nullptr;
  T.stage_bytes = 0;
  T.tcs = nullptr;
  T.tmem = 0;
  long long sws_doubles = (98 * 1024 - 64 * 8 - GEMM_STAGE_BYTES) / 8;
  std::vector<double> sws((size_t)std::max<long long>(sws_doubles, kItemWsDoubles));
  std::vector<int> tr((size_t)im.trace_total + 8);
  run_instance_braket(T, sp, L, im.desc[0], im.i64.data(), im.i32.data(), im.dat.data(), res, tr.data(), sws.data(),
                      sws_doubles);
  if (trace && im.desc[0].trace_cap > 0)
    std::memcpy(trace, tr.data(), sizeof(int) * 8 * (size_t)std::min(trace_cap, im.desc[0].trace_cap));
  return res->status;
}

int catn_hostcheck_dense(const catn_params* p, int n, const int* ndims, const long long* dims,
                         const double* data, const int* neighbors, long long arena_bytes,
                         catn_result* res, int* trace, int trace_cap) {
  Image im;
  std::string e = im.add_dense(*p, n, ndims, dims, data, neighbors, trace_cap);
  if (!e.empty()) return CATN_EINVAL;
  return run_image(im, arena_bytes, res, trace);
}

// A dense network with cut_bondim! calls (3 ints each: i, idx_j_in_i, opt)
// replayed before the contraction; cut_only stops after the cuts (res->err:
// the discarded sum of the last cut).
int catn_hostcheck_dense_cuts(const catn_params* p, int n, const int* ndims, const long long* dims,
                              const double* data, const int* neighbors, const int* cuts, int n_cuts, int cut_only,
                              long long arena_bytes, catn_result* res, int* trace, int trace_cap) {
  Image im;
  std::string e = im.add_dense(*p, n, ndims, dims, data, neighbors, trace_cap);
  if (!e.empty()) return CATN_EINVAL;
  im.set_cuts(std::vector<int>(cuts, cuts + 3 * n_cuts));
  im.desc[0].cut_only = cut_only;
  return run_image(im, arena_bytes, res, trace);
}

// Ising site recipes (ising_build.cuh) checked on the host: the batch is
// built from (w, h, betas) with recipes recorded, the recipes are evaluated
// with (w2, h2, betas2), and the values are compared with a batch built
// directly from (w2, h2, betas2).  Returns the recipe count (-1 on a build
// error); *maxdiff is the largest absolute difference, *covered the number
// of distinct image values the recipes wrote, *total the image size.
long long catn_hostcheck_ising_recipes(const catn_params* p, int n_inst, const int* n_nodes,
                                       const long long* node_off, const long long* edge_off, const int* edges,
                                       const double* w, const double* h, const double* betas, const double* w2,
                                       const double* h2, const double* betas2, const int* pins, double* maxdiff,
                                       long long* covered, long long* total) {
  Image A, B;
  for (int q = 0; q < n_inst; ++q) {
    const long long e0 = edge_off[q], ne = edge_off[q + 1] - e0;
    const int* pq = pins + 4 * q;
    if (!A.add_ising(*p, n_nodes[q], (int)ne, edges + 2 * e0, w + e0, h + node_off[q], betas[q], pq[0], pq[1],
                     pq[2], pq[3], 0, e0, node_off[q]).empty())
      return -1;
    if (!B.add_ising(*p, n_nodes[q], (int)ne, edges + 2 * e0, w2 + e0, h2 + node_off[q], betas2[q], pq[0], pq[1],
                     pq[2], pq[3], 0).empty())
      return -1;
  }
  if (A.dat.size() != B.dat.size()) return -1;
  std::vector<char> hit(A.dat.size(), 0);
  double md = 0.0;
  long long cov = 0;
  for (const IsingSiteRecipe& r : A.recipes) {
    double v[8];
    const int c = ising_site_values(r, r.edge >= 0 ? w2[r.edge] : 0.0, h2[r.node], betas2[r.inst], v);
    for (int k = 0; k < c; ++k) {
      const double d = std::fabs(v[k] - B.dat[r.dat + k]);
      if (!(d <= md)) md = d;
      if (!hit[r.dat + k]) {
        hit[r.dat + k] = 1;
        ++cov;
      }
    }
  }
  *maxdiff = md;
  *covered = cov;
  *total = (long long)A.dat.size();
  return (long long)A.recipes.size();
}

// The device disorder generator's formula evaluated on the host.
double catn_hostcheck_disorder_normal(unsigned long long seed, unsigned long long stream, unsigned long long index) {
  return disorder_normal(seed, stream, index);
}

}
