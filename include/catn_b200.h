/* catn_b200.h -- C ABI of libcatn_b200.so, the B200 (sm_100a) implementation
 * of the CATN.jl `contraction!` hot path.
 *
 * The reference (xuanzhaogao/CATN.jl v0.1.0) has no FFI: its backend seam is
 * Julia dispatch on the array type `AT` of `TensorNetwork{T,AT}` /
 * `MPSNode{T,AT}` (src/tensor_network.jl:1, src/mps_node.jl:1) entered
 * through `Adapt.adapt_structure` (src/adapt.jl:6-24).  Each entry point
 * below replaces the reference function named beside it (a Julia `ccall`
 * binding for each is one line per function: the argument types below map
 * to Cint, Cdouble, Ptr{...} one to one).
 *
 * Conventions
 *   - Node ids are 1-based, neighbour ids of open legs are negative
 *     sentinels, exactly as in the reference.
 *   - Site tensors are (left, phys, right) in column-major order (Julia
 *     layout); dense tensors are column-major over their legs.
 *   - All buffers passed in are host memory owned by the caller for the
 *     duration of the call; the library copies what it needs to HBM.
 *   - Every function returns a catn_status; on failure a thread-local message
 *     is available from catn_last_error().
 */
#ifndef CATN_B200_H
#define CATN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  CATN_OK = 0,
  CATN_EINVAL = 1,    /* bad argument (reference: error()/@assert)          */
  CATN_ENOMEM = 2,    /* device arena or control capacity exhausted         */
  CATN_ENOCONV = 3,   /* Jacobi SVD hit its sweep cap                       */
  CATN_ETIMEOUT = 4,  /* a bounded device wait ran out                      */
  CATN_ECUDA = 5,     /* CUDA runtime error                                 */
  CATN_ESTATE = 6     /* reference error path (e.g. open-leg cut, merge!)   */
} catn_status;

/* Keyword arguments of TensorNetwork / ising_network
 * (src/tensor_network.jl:41-54, src/ising.jl:20-40). */
typedef struct {
  int32_t Dmax;        /* <0: exact mode                                   */
  int32_t chi;
  double cutoff;
  int32_t norm_method; /* 0 none, 1 Frobenius, 2 max-abs                     */
  int32_t select;      /* 0 min_dim, 1 min_dim_triangle, 2 sequential        */
  int32_t reverse;
  int32_t svdopt;
  int32_t swapopt;
  int32_t compress;
  int32_t cut_bond;
  int32_t seed;        /* key of the rsvd sketch generator (rsvd = 1)       */
  int32_t trace;       /* record the per-step integer trace                 */
  int32_t rsvd;        /* swap! matrices on the reference's randomized-SVD
                        * route (swapopt, both sides > 7000 or one > 20000,
                        * mps_node.jl:154-156): 0 = the exact top-chi
                        * subspace; 1 = the reference's randomized algorithm
                        * (linalg_utils.jl:44-58: sketch of min(n, 10 chi)
                        * columns, 10 power iterations), its Gaussian sketch
                        * drawn from the counter-based generator keyed by
                        * seed (forward runs; gradient runs use 0); 2 = the
                        * same with the products of the swap matrix applied
                        * from the two sites (matrix-free: the (d0 d1) x
                        * (d2 d3) matrix is never formed)                 */
  /* Fields below have no counterpart in the reference's keywords. */
  int32_t rsvd_min_dim; /* > 0: the randomized route above takes swap!
                        * matrices with both sides >= rsvd_min_dim or one
                        * side >= 3 rsvd_min_dim (tests reach it with small
                        * networks); 0 = the reference's 7000 / 20000      */
  int32_t precision;   /* 0 = FP64 throughout; 1 = split: the products of
                        * large swap merges and the pair Grams of the block
                        * Jacobi route's first phase in 3xTF32 on the
                        * tensor cores with FP32 accumulation, while the
                        * rotations, a second Jacobi phase on FP64 Grams,
                        * every singular-value cutoff test, the Dmax cut
                        * and lnZ stay FP64                              */
  int32_t svd_route;   /* large SVDs (not held in shared memory):
                        * 0 = auto (precision 0: block Jacobi from the tuning
                        *     table's size on for a network that
                        *     catn_contract contracts on its own, the whole
                        *     GPU helping it; scalar Jacobi in batches and
                        *     gradient runs; precision 1: block Jacobi from
                        *     the tuning table's size on),
                        * 1 = scalar one-sided Jacobi on the pivoted-QR
                        *     factor (the FP64 route of earlier releases,
                        *     bit for bit),
                        * 2 = block one-sided Jacobi on the pivoted-QR
                        *     factor from the tuning table's size on      */
  int32_t ckpt_interval; /* gradient runs: 0 = the tape of the whole
                        * contraction stays on the device; K > 0 = the
                        * forward pass keeps a checkpoint every K steps and
                        * the backward pass recomputes one K-step segment
                        * at a time (memory: one segment's tape plus the
                        * checkpoints; gradients bit-identical to K = 0)  */
  int32_t braket_loops; /* catn_braket_create: 0 = a cyclic virtual-bond
                        * graph is rejected, as the reference does
                        * (src/braket.jl:405-420); 1 = cycles are allowed
                        * and each pair of doubled bonds that an eat makes
                        * parallel is fused (ket with ket, bra with bra)
                        * before the next step                           */
} catn_params;

/* Launch-shape and route thresholds, one process-wide table (no reference
 * counterpart).  catn_tuning_get returns the table in force (the built-in
 * defaults until catn_tuning_set is called); the autotuner
 * (catn_b200.tune) measures candidates on the GPU and installs the winners
 * with catn_tuning_set.  A value < 0 selects the built-in default.  The
 * table is read when a launch starts; results never depend on the helper
 * and sharing entries, only the block-route entries change arithmetic. */
typedef struct {
  int32_t helper_ctas;         /* dedicated helper CTAs of a batch launch   */
  int32_t grad_helper_ctas;    /* the same for batch gradient launches      */
  int32_t shared_jacobi_min_n; /* smallest column count whose Jacobi rounds
                                * are opened to helper CTAs                 */
  int32_t block_min_n;         /* smallest column count of the Jacobi factor
                                * that takes the block route (svd_route 0
                                * with precision 1, and svd_route 2)        */
  int64_t shared_house_min;    /* smallest rows x columns whose Householder
                                * steps are opened to helper CTAs           */
  int32_t blocked_qr_min_n;    /* smallest column count whose QR on the
                                * block route is the blocked, norm-sorted
                                * one instead of the column-pivoted one
                                * (default: never; measured slower overall,
                                * the Jacobi after it needs more sweeps)    */
  int32_t reserved;
} catn_tuning;
catn_status catn_tuning_get(catn_tuning* t);
catn_status catn_tuning_set(const catn_tuning* t);

/* Default values of the reference's keyword arguments. */
void catn_params_default(catn_params* p);

/* Results of one contraction (`contraction!` return value plus state). */
typedef struct {
  double lnZ;          /* tn.lnZ                                            */
  double err;          /* accumulated discarded singular values             */
  double psi;          /* tn.psi (phase; +-1 for real networks)             */
  double sign;         /* tn.sign from network_lognorm                      */
  int32_t maxdim;      /* tn.maxdim_intermediate                            */
  int32_t status;      /* catn_status of this instance                      */
  int32_t nsteps;      /* contraction steps taken                           */
  int32_t jacobi_max;  /* largest Jacobi sweep count seen                   */
  int64_t arena_peak;  /* device bytes high-water mark                      */
  double flops;        /* algorithmic FLOPs of the contraction (see below)  */
  double bytes;        /* algorithmic bytes: site tensors read + written    */
  double prof[24];     /* SM cycles: [0] contraction total, [1] tiny SVDs
                          (one warp), [2] small SVDs (shared memory), [3]
                          large SVDs, [4] edge bookkeeping; counts: [5]
                          tiny, [6] small, [7] large SVDs; cycles: [8] swap
                          merge GEMM, [9] swap epilogue, [10] cano step
                          after its SVD, [11] eat folds, [12] merge fuse,
                          [13] Dmax cut (its SVD included), [14] reverse,
                          [15] loop control (re-pointing, checks); within
                          large SVDs: [16] pivoted QR, [17] Jacobi, [18]
                          application of Q; [19] block-route Jacobis, [20]
                          their summed sweeps, [21] summed columns of the
                          large Jacobi factors; cycles of [22] the
                          block-route Jacobis, [23] the Jacobis of >= 1024
                          columns                                         */
} catn_result;
/* Algorithmic work convention (per step, FP64 elements of 8 bytes):
 *   swap / compress pair: 2*m*n*k + 4*m*n*r  (m=d0*d1, n=d2*d3, k bond, r kept)
 *   cano step:            2*(dl*d)*dr^2 + 2*dr^2*(d'*dr')
 *   eat fold:             2*Dl*d*Dr + 2*dl2*d2*Dl*Dr
 *   Dmax cut:             2*(dl*dr)*d^2 * 2 + 2*di*dj*d + 4*di*dj*r
 *   merge fuse:           2*(dl*d1)*k*(d2*dr2)
 * bytes count the site tensors each step reads and writes; the merged
 * two-site matrix and SVD workspaces count as on-chip. */

typedef struct catn_net catn_net;       /* one network, device resident    */
typedef struct catn_batch catn_batch;   /* many networks, one launch       */

/* Network in MPS form (what ising_network and MPSNode carry).
 *   site_counts[k]        number of sites of node k+1
 *   nbr_counts[k]         number of neighbour entries of node k+1
 *   canos[k]              node.cano
 *   site_dims[3*s..]      (dl, d, dr) of every site, nodes in order
 *   site_data             all site tensors concatenated (float64)
 *   neighbors             all neighbour lists concatenated
 * Replaces TensorNetwork{T,AT}(nodes...) construction on the device side
 * (src/tensor_network.jl:118-139, src/ising.jl:205-226). */
catn_status catn_net_create_mps(const catn_params* p, int32_t n_nodes, const int32_t* site_counts,
                                const int32_t* nbr_counts, const int32_t* canos,
                                const int64_t* site_dims, const double* site_data,
                                const int32_t* neighbors, int64_t arena_bytes, catn_net** out);

/* Network from dense tensors (`TensorNetwork(tensors, ixs)`,
 * src/tensor_network.jl:41-140): node k has ndims[k] legs with the given
 * dims; the neighbour list gives, per leg, the node sharing it (negative
 * sentinel for open legs).  raw2mps (src/mps_node.jl:31-50) runs on the
 * device. */
catn_status catn_net_create_dense(const catn_params* p, int32_t n_nodes, const int32_t* ndims,
                                  const int64_t* dims, const double* data,
                                  const int32_t* neighbors, int64_t arena_bytes, catn_net** out);

/* contraction!(tn) -> (lnZ, error, psi)  (src/tensor_network.jl:556-717).
 * `trace` (optional, may be NULL) receives 8 int32 per step:
 *   i, j, rev_i | rev_j<<1, n_duplicates, fnv(duplicates), nsites_i,
 *   fnv(phys dims of i), maxdim_intermediate. */
catn_status catn_contract(catn_net* net, catn_result* res, int32_t* trace, int32_t trace_cap);

/* cut_bondim!(tn, i, idx_j_in_i) (src/tensor_network.jl:342-388) with
 * opt = 0, cut_bondim_opt!(tn, i, idx_j_in_i) (src/tensor_network.jl:399-477)
 * with opt != 0: truncates the bond between node i and its neighbour on leg
 * idx_j_in_i to at most Dmax singular values (after the cutoff) and writes
 * the discarded sum to *err.  Dmax < 0: a no-op with *err = 0, as in the
 * reference.  The cut changes the network that a later catn_contract
 * contracts; every cut runs on the device (the network's image is loaded
 * and the cuts so far are replayed in order).  CATN_ESTATE for an open leg
 * or a one-sided bond, as the reference's error() calls; CATN_EINVAL for a
 * BraKet network, for ids out of range, and later for catn_ising_grad on a
 * cut network. */
catn_status catn_cut_bondim(catn_net* net, int32_t i, int32_t idx_j_in_i, int32_t opt, double* err);

/* Shapes of the surviving nodes after contraction (result_tensor support,
 * src/tensor_network.jl:517-523): dense tensor of the single surviving
 * open-leg node, legs in its final MPS order.  `out` may be NULL to query
 * `numel`/`ndim`; `dims` receives up to 64 leg sizes. */
catn_status catn_result_tensor(catn_net* net, double* out, int64_t cap, int64_t* numel,
                               int32_t* ndim, int64_t* dims);

catn_status catn_net_destroy(catn_net* net);

/* Ising / spin-glass network in MPS form (src/ising.jl:20-227), built on the
 * host exactly as the reference's builder does, contracted on the device.
 * edges: 2*n_edges 1-based endpoints.  pos/val pin spins as in the
 * reference (0 = none). */
catn_status catn_ising_create(const catn_params* p, int32_t n, int32_t n_edges,
                              const int32_t* edges, const double* weights, const double* fields,
                              double beta, int32_t pos1, int32_t val1, int32_t pos2, int32_t val2,
                              int64_t arena_bytes, catn_net** out);

/* Device memory the allocation-free entry point below works in: one
 * file-scope array in the library, present on every GPU that loads it until
 * the process exits. */
#define CATN_STATIC_SCRATCH_BYTES (64LL << 20)

/* No counterpart in the reference.  Contracts one Ising / spin-glass network
 * exactly like catn_ising_create + catn_contract (same arguments, same
 * result), but allocates no device memory: the packed network, the
 * contraction's working memory and the result all live in the library's
 * fixed CATN_STATIC_SCRATCH_BYTES device array.  For callers that must not
 * call cudaMalloc -- code running under a caller-owned memory pool or a
 * strict device-memory budget, or inside a host loop where allocation
 * latency and fragmentation are not acceptable.
 *   - Networks whose working memory does not fit return CATN_ENOMEM with
 *     the required and available sizes in catn_last_error().
 *   - Every call looks up the array's device address on the current device
 *     (cudaGetSymbolAddress, which allocates nothing) and sets the kernel's
 *     shared-memory attribute; make the first call on a device before any
 *     stream capture.
 *   - Every call reuses the same array, so calls that overlap on the GPU
 *     (different streams, threads or processes sharing a context) race;
 *     serialise them.  The call synchronises `stream` before returning.
 *   - `stream` is a cudaStream_t (NULL = default stream); trace recording
 *     (p->trace) is not available here. */
catn_status catn_ising_contract_static(const catn_params* p, int32_t n, int32_t n_edges,
                                       const int32_t* edges, const double* weights,
                                       const double* fields, double beta, int32_t pos1,
                                       int32_t val1, int32_t pos2, int32_t val2, void* stream,
                                       catn_result* res);

/* No counterpart in the reference.  C (M x N) = A (M x K) * B (K x N), all
 * column-major FP64 host buffers, computed on the tensor cores in the
 * split-precision form of catn_params.precision = 1: the operands rounded
 * to FP32 and split into TF32 hi / lo parts, three tcgen05 TF32 products per
 * pair (hi hi + hi lo + lo hi) accumulated in FP32.  Relative error about
 * 1e-6 of |A| |B|.  It exposes the tensor-core primitive the split mode's
 * large products use, so that it can be checked on its own. */
catn_status catn_tc_matmul(int32_t M, int32_t N, int32_t K, const double* A, const double* B, double* C);

/* Batched Ising instances contracted in ONE persistent kernel launch with a
 * device work queue (no reference counterpart: the reference loops on the
 * host, e.g. magnetization/correlation at src/ising.jl:263-339).
 * Instance b uses edges[edge_off[b] .. edge_off[b+1]) (pairs), fields
 * [node_off[b] .. node_off[b+1]), betas[b], pins[4*b .. 4*b+3]
 * (pos1, val1, pos2, val2; NULL = none). */
catn_status catn_ising_batch_create(const catn_params* p, int32_t n_inst, const int32_t* n_nodes,
                                    const int64_t* node_off, const int64_t* edge_off,
                                    const int32_t* edges, const double* weights,
                                    const double* fields, const double* betas,
                                    const int32_t* pins, int64_t slot_arena_bytes,
                                    int32_t max_slots, catn_batch** out);

/* No counterpart in the reference, which rebuilds every network on the host
 * (ising_network, src/ising.jl:20-227).  New couplings, fields and inverse
 * temperatures for the instances of a batch made by catn_ising_batch_create,
 * with the same lattices and pins: weights in the order of the edges at
 * creation (all instances), fields likewise, betas one per instance (NULL =
 * keep).  Only these arrays cross to the device; a kernel rebuilds every site
 * tensor there (the builder's values, src/ising.jl:95-183), and the next
 * catn_batch_launch contracts the new networks.  catn_batch_upload restores
 * the networks given at creation; gradient launches need those
 * (CATN_ESTATE otherwise).  `stream` is a cudaStream_t (NULL = default). */
catn_status catn_ising_batch_set_params(catn_batch* b, const double* weights, const double* fields,
                                        const double* betas, void* stream);

/* No counterpart in the reference.  Disorder generated on the device:
 * weights sigma_w * N(0,1), fields sigma_h * N(0,1) (betas kept), from a
 * counter-based generator keyed by `seed` (SplitMix64 mixing, Box-Muller),
 * then the site tensors rebuilt as by catn_ising_batch_set_params. */
catn_status catn_ising_batch_randomize(catn_batch* b, uint64_t seed, double sigma_w, double sigma_h,
                                       void* stream);

/* The batch's current couplings, fields and betas (device copies; sizes as
 * in catn_ising_batch_set_params).  Synchronous. */
catn_status catn_ising_batch_get_params(const catn_batch* b, double* weights, double* fields, double* betas);

/* Bytes that catn_ising_batch_set_params copies host->device (all three
 * arrays). */
int64_t catn_ising_batch_param_bytes(const catn_batch* b);

/* Upload the inputs of the batch (host -> HBM), run the persistent kernel,
 * read back the per-instance results.  Timing-friendly split below. */
catn_status catn_batch_run(catn_batch* b, catn_result* results);

/* Device-only run: inputs already resident; `stream` is a cudaStream_t
 * (NULL = default stream).  Results stay on the device until
 * catn_batch_results(). */
catn_status catn_batch_launch(catn_batch* b, void* stream);
catn_status catn_batch_upload(catn_batch* b, void* stream);
catn_status catn_batch_results(catn_batch* b, catn_result* results, void* stream);
/* Number of CTA slots (resident blocks) the batch launches with. */
int32_t catn_batch_slots(const catn_batch* b);
/* Bytes of per-batch input copied host->device by catn_batch_upload. */
int64_t catn_batch_input_bytes(const catn_batch* b);
catn_status catn_batch_destroy(catn_batch* b);

/* braket_network(tensors, ixs; chi, cutoff, norm_method, svdopt, swapopt)
 * (src/braket.jl:369-508): the double-layer network <psi|psi> of a real ket
 * state.  Tensor k has ndims[k] axes with sizes dims[...] (concatenated) and
 * column-major data; labels[...] holds one positive label per axis.  A label
 * on one tensor is its physical index (exactly one per tensor), a label on
 * two tensors a virtual bond; a cyclic bond graph is rejected (CATN_EINVAL,
 * as the reference errors) unless p->braket_loops is 1, and two labels
 * shared by the same two tensors are always rejected.  Contract it with
 * catn_contract: lnZ = log of <psi|psi> up to psi, err = discarded weight,
 * maxdim = largest leg seen.  Only p->chi, cutoff, norm_method, svdopt and
 * braket_loops are used.  The edges are taken
 * in the order their labels first appear (the reference iterates a Julia
 * Dict there, src/braket.jl:489-497). */
catn_status catn_braket_create(const catn_params* p, int32_t n, const int32_t* ndims, const int64_t* dims,
                               const double* data, const int32_t* labels, int64_t arena_bytes, catn_net** out);

/* ---- adjoint (gradient of lnZ) ------------------------------------------
 * No reference counterpart: the reference obtains <s_k> and <s_i s_j> by
 * pinning, 1 + 2n and 1 + 4|E| full contractions (magnetization /
 * correlation, src/ising.jl:263-339).  Here one forward contraction records
 * a tape on the device and one backward pass gives
 *   dlnZ_dw[e] = d lnZ / d w_e  (= beta <s_i s_j> for edge e = (i, j)),
 *   dlnZ_dh[k] = d lnZ / d h_k  (= beta <s_k>),
 * exact up to the truncations of the contraction itself (the truncated part
 * of every SVD, and kept values below 1e-10 of the largest, count as zero in
 * the backward pass).  Networks from catn_ising_create only; compress = 1 is
 * rejected (CATN_EINVAL).  The gradient run allocates its own device slots
 * (2.5x the forward arena: tape, append-only heap and its shadow) on the
 * first call and keeps them until destroy.
 *
 * ckpt_interval (>= 0) sets the network's catn_params.ckpt_interval for
 * this call: 0 keeps the tape of the whole contraction on the device; K > 0
 * keeps a checkpoint every K steps and recomputes one segment at a time in
 * the backward pass (same gradients, bit for bit, in bounded memory).
 * Batch gradient runs take each instance's catn_params.ckpt_interval. */
catn_status catn_ising_grad(catn_net* net, catn_result* res, double* dlnZ_dw, double* dlnZ_dh,
                            int32_t ckpt_interval);
/* Every instance of a batch in one persistent launch (inputs uploaded by the
 * call); results and gradients are read back by catn_batch_grad_results,
 * dlnZ_dw / dlnZ_dh concatenated per instance in the edge_off / node_off
 * order of catn_ising_batch_create. */
catn_status catn_batch_grad_launch(catn_batch* b, void* stream);
catn_status catn_batch_grad_results(catn_batch* b, catn_result* results, double* dlnZ_dw, double* dlnZ_dh,
                                    void* stream);

/* Thread-local message of the last failure (always NUL-terminated). */
/* Device and pinned host blocks of destroyed networks and batches are kept
 * by the library for the next network or batch (no reference counterpart:
 * Julia's GC owns the reference's arrays).  A network created and destroyed
 * in a loop then pays no cudaMalloc / cudaFree per iteration.  Up to 8 blocks
 * per device and kind are kept; an allocation that finds the device full
 * frees them first.  catn_release_cached_memory frees every kept block (for
 * callers that hand the memory to other libraries); catn_cached_bytes
 * reports the bytes kept (host != 0: pinned host memory).  A program that
 * resets a device (cudaDeviceReset) calls catn_release_cached_memory before
 * the reset: kept blocks do not survive it, and the library cannot tell. */
catn_status catn_release_cached_memory(void);
int64_t catn_cached_bytes(int32_t host);

size_t catn_last_error(char* buf, size_t cap);

/* Library build string (arch, version). */
const char* catn_version(void);

#ifdef __cplusplus
}
#endif
#endif /* CATN_B200_H */
