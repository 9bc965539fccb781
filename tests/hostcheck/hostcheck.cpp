// Test-only host build of the device engine (team of one thread), used by the
// CPU test-suite to check the engine's integer bookkeeping and memory safety
// (under AddressSanitizer) against the oracle.  It is not part of
// libcatn_b200 and is never loaded by the product path.
#include <cstdlib>
#include <cstring>
#include <vector>
#include "../../catn.jl_b200/csrc/engine.cuh"
#include "../../catn.jl_b200/csrc/adjoint.cuh"
#include "../../catn.jl_b200/csrc/braket.cuh"
#include "../../catn.jl_b200/csrc/host_image.h"

using namespace catn;

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
  std::vector<int> tr((size_t)im.trace_total + 8);
  // stand-in for the GPU's shared-memory SVD workspace (same capacity)
  long long sws_doubles = (100 * 1024 - 64 * 8 - GEMM_STAGE_BYTES) / 8;
  // CATN_HOSTCHECK_SWS overrides the capacity (0 sends every SVD through the
  // large-matrix path, including its rank-revealing truncation)
  if (const char* e = std::getenv("CATN_HOSTCHECK_SWS")) sws_doubles = std::atoll(e);
  std::vector<double> sws((size_t)(sws_doubles > 0 ? sws_doubles : 1));
  // CATN_HOSTCHECK_JOB=1 sends the Jacobi sweeps of every SVD on the global
  // path through the shared-job protocol (no helpers: the team claims all)
  JacobiJob job;
  std::memset(&job, 0, sizeof(job));
  const int qhead = 1;
  JobLink jl;
  jl.job = &job;
  jl.qhead = &qhead;
  jl.ninst = 1;
  jl.min_n = 2;
  jl.pool = 0;
  jl.min_qr = 1;
  const char* je = std::getenv("CATN_HOSTCHECK_JOB");
  run_instance(T, sp, L, im.desc[0], im.i64.data(), im.i32.data(), im.dat.data(), res, tr.data(), sws.data(),
               sws_doubles, (je && je[0] == '1') ? &jl : nullptr);
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
  long long sws_doubles = (100 * 1024 - 64 * 8 - GEMM_STAGE_BYTES) / 8;
  if (const char* ev = std::getenv("CATN_HOSTCHECK_SWS")) sws_doubles = std::atoll(ev);
  std::vector<double> sws((size_t)(sws_doubles > 0 ? sws_doubles : 1));
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
  long long sws_doubles = (100 * 1024 - 64 * 8 - GEMM_STAGE_BYTES) / 8;
  std::vector<double> sws((size_t)sws_doubles);
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

}
