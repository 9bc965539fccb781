"""Benchmark: batched spin-glass lnZ instances/s on B200 (libcatn_b200).

Workload (one "step" = one persistent-kernel pass over one batch):
  512 independent 2D spin-glass instances, open L x L square lattices with L
  drawn uniformly from {8,10,12,14,16} (64-256 spins), couplings J ~ N(0,1),
  fields h ~ N(0, 0.1^2), beta ~ U[0.5, 2.0], Dmax=32, chi=128, cutoff 1e-15,
  select=1, norm_method=1 -- seeded synthetic inputs (numpy PCG64).

  value  instances/s with the inputs already in HBM (CUDA events around the
         kernel launch; L2 flushed by a 256 MiB write between steps)
  e2e    instances/s through the public batch API per step: pinned
         host->device copy of the step's inputs (every instance's couplings,
         fields and beta; the lattices are fixed at batch creation), the
         device rebuild of the site tensors, the launch, and the
         device->host read of every instance's result (CUDA events on the
         same stream).  `e2e.full_image` times the same path with the whole
         host-built network image uploaded instead.

  grad   the other half of the metric: d lnZ / d w and d lnZ / d h (every
         <s_i s_j>, <s_k> of every instance) from one device gradient run
         of the whole batch, against the reference's pinning definition,
         which needs 1 + 2n + 4|E| contractions per instance: the pinned
         networks of the first instances are contracted in one launch and
         timed, and their measured rate prices the batch's pinned set

  plain_gpu_form  the same instances through the plain GPU form
         (baseline/plain_gpu_form.py: PyTorch FP64, one library call per
         op from a host loop, one instance at a time), a bounded sample on
         rank 0 at N=1, with its |dlnZ|/n against the engine

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU: one process per GPU (torchrun); every rank contracts its own
512-instance batch (weak scaling, no data-path collective); the time is the
max over ranks.
"""
import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = ("Ising lnZ instances/s and ∇lnZ time vs pinning, at |ΔlnZ|/n≤1e-6 vs FP64")
PARAMS = dict(Dmax=32, chi=128, cutoff=1e-15, select=1, norm_method=1)
WORKLOAD = ("512 2D spin-glass instances, L~U{8,10,12,14,16}, J~N(0,1), h~N(0,0.1^2), "
            "beta~U[0.5,2], Dmax=32, chi=128, one persistent launch")


def make_instances(count, seed):
    import __graft_entry__
    catn = __graft_entry__.load_package()
    from catn_b200 import graphs
    return graphs.spinglass_batch(count, seed)


# ----------------------------------------------------------------------------
# CPU legs (oracle port) -- run in spawned worker processes
# ----------------------------------------------------------------------------
def _oracle_one(d):
    from oracle import ising as OI, network as ON
    tn = OI.ising_network(d["n"], d["edges"], d["weights"], d["fields"], d["beta"], **PARAMS)
    lnZ, _, _ = ON.contraction(tn)
    return lnZ


def _cpu_pool(nproc):
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    os.environ["OMP_NUM_THREADS"] = "1"
    return mp.get_context("spawn").Pool(nproc)


def cpu_sample_rate(instances, seconds, nproc, pool=None):
    """Contract instances in order on `nproc` single-threaded processes until
    about `seconds` have passed; return (instances/s, count, lnZ list)."""
    own = pool is None
    pool = pool or _cpu_pool(nproc)
    t0 = time.perf_counter()
    done, lz = 0, []
    it = pool.imap(_oracle_one, instances, chunksize=1)
    for v in it:
        lz.append(v)
        done += 1
        if time.perf_counter() - t0 > seconds or done == len(instances):
            break
    dt = time.perf_counter() - t0
    if own:
        pool.terminate()
    return done / dt, done, lz


def plain_form_rate(instances, engine_lnZ, seconds):
    """Contract instances in order through the plain GPU form until about
    `seconds` have passed; return (instances/s, count, max |dlnZ|/n vs the
    engine)."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "baseline"))
    import plain_gpu_form as PG
    sys.path.pop(0)
    w = instances[0]   # warm-up: cuSOLVER/cuBLAS handles and workspaces
    PG.contraction(PG.ising_network(w["n"], w["edges"], w["weights"], w["fields"], w["beta"], **PARAMS))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    done, dev = 0, 0.0
    for d, ref in zip(instances, engine_lnZ):
        lz, _, _ = PG.contraction(PG.ising_network(d["n"], d["edges"], d["weights"], d["fields"], d["beta"],
                                                   **PARAMS))
        done += 1
        dev = max(dev, abs(lz - ref) / d["n"])
        if time.perf_counter() - t0 > seconds:
            break
    torch.cuda.synchronize()
    return done / (time.perf_counter() - t0), done, dev


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ----------------------------------------------------------------------------
# clocks
# ----------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def read_traffic():
    """DRAM bytes per launch of the persistent kernel from the committed ncu
    summary (profiles/catn_persistent_kernel_spinglass_batch.txt), if any."""
    p = os.path.join(ROOT, "profiles", "catn_persistent_kernel_spinglass_batch.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_full_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def _secondary(out, key, fn):
    """Run one secondary leg into out[key]; a failure is recorded there
    instead of ending the run before the headline line is printed."""
    try:
        out[key] = fn()
    except Exception as e:  # noqa: BLE001 -- any failure of a side leg is reported, not raised
        out[key] = {"error": f"{type(e).__name__}: {e}"}


def load_bf16_peak(key="bf16_tflops_sustained"):
    """Dense bf16 GEMM TFLOP/s from MEASURED_PEAKS.json (the sustained figure
    by default: the launches it is compared with run for seconds), or None."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        v = json.load(open(p)).get(key)
        return float(v) if v else None
    return None


# ----------------------------------------------------------------------------
def lpt_order(instances):
    """Largest instances first (by edge count), as the device work queue
    takes them, so that a pass over the batch on the host cores does not end
    on one large instance started last."""
    return sorted(range(len(instances)), key=lambda q: -len(instances[q]["edges"]))


def config_of(args, world):
    """The workload description shared by both arms (same keys, same values)."""
    return {"workload": WORKLOAD, "instances_per_gpu": args.instances, "seed": args.seed,
            "Dmax": PARAMS["Dmax"], "chi": PARAMS["chi"],
            "parallelism": f"replicas x{world} (independent instances)",
            "l2": "flushed between timed steps by a 256 MiB device write (the host-core reference arm has "
                  "no device L2)"}


def run_reference(args):
    """--impl reference: the oracle port (CPU restatement of the reference
    algorithm; Julia is unavailable) on all host cores, rank 0 only.  One
    step contracts the whole batch: every instance once, one single-threaded
    process per core pulling instances in LPT order (imap, no per-chunk
    barrier), like the device arm's work queue."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    cores = host_cores()
    insts = make_instances(args.instances, args.seed)
    order = [insts[q] for q in lpt_order(insts)]
    pool = _cpu_pool(cores)
    times = []
    for s in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        for _ in pool.imap_unordered(_oracle_one, order, chunksize=1):
            pass
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            times.append(dt)
    pool.terminate()
    t = sum(times)
    v = args.instances * args.steps / t
    out = {"impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "instances/s",
           "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(1000 * t / args.steps, 3), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": config_of(args, world),
           "cpu_baseline": {"value": round(v, 3), "unit": "instances/s", "cores": cores, "kind": "port",
                            "sample": f"the whole {args.instances}-instance batch per step, oracle port "
                                      f"(numpy/OpenBLAS FP64), {cores} single-threaded processes pulling "
                                      f"instances largest first"},
           "e2e": {"value": round(v, 3), "unit": "instances/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--instances", type=int, default=512)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-grad", action="store_true", help="skip the gradient leg")
    ap.add_argument("--plain-seconds", type=float, default=15.0,
                    help="time budget of the plain GPU form sample (0 = skip)")
    ap.add_argument("--max-slots", type=int, default=0, help="cap on CTA slots (0 = all resident)")
    ap.add_argument("--no-c2", action="store_true", help="skip the n=200 random-regular leg")
    ap.add_argument("--c4-full", action="store_true",
                    help="also run the 32x32 Gaussian lattice at full size (forward, checkpointed adjoint, one "
                         "central difference, 8 pinned edges; several minutes)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the 8x8 ferromagnet, the reduced 32x32 Gaussian-lattice and the reduced PEPS legs")
    ap.add_argument("--c2-scalar", action="store_true",
                    help="also time the n=200 leg on the scalar Jacobi route (about 40 s per beta)")
    ap.add_argument("--no-c2-oracle", action="store_true",
                    help="skip timing the FP64 oracle on beta = 1 of the n=200 random-regular leg (~25 s)")
    ap.add_argument("--arena-mb", type=int, default=64, help="device arena per slot, MiB")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    # CPU baseline first (spawned pool, before any CUDA call), rank 0 at N=1 only
    cpu = None
    cpu_lz = {}
    if rank == 0 and world == 1 and not args.no_cpu:
        cores = host_cores()
        sample = make_instances(args.instances, args.seed)
        order = lpt_order(sample)
        rate, cnt, lz = cpu_sample_rate([sample[q] for q in order], args.cpu_seconds, cores)
        cpu_lz = {order[k]: v for k, v in enumerate(lz)}
        cpu = {"value": round(rate, 3), "unit": "instances/s", "cores": cores, "kind": "port",
               "sample": f"{cnt} of the {args.instances} workload instances, largest first, "
                         f"oracle port (numpy/OpenBLAS FP64), {cores} single-threaded processes, "
                         f"~{args.cpu_seconds:.0f} s"}

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    import ctypes
    import __graft_entry__
    catn = __graft_entry__.load_package()
    from catn_b200 import _lib as catn_lib
    insts = make_instances(args.instances, args.seed + 7919 * rank)
    batch = catn.IsingBatch(insts, slot_arena_bytes=args.arena_mb << 20, max_slots=args.max_slots, **PARAMS)
    stream = torch.cuda.current_stream()
    sh = ct_stream(stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def device_step():
        batch.launch(sh)

    # warm-up (full API path, checks every instance)
    batch.upload(sh)
    for _ in range(args.warmup):
        batch.launch(sh)
        batch.fetch(sh)
    res = batch.fetch(sh)
    res_ref = [catn_lib.Result.from_buffer_copy(x) for x in res]
    flops = sum(r.flops for r in res)
    nbytes = sum(r.bytes for r in res)
    steps_per_inst = [r.nsteps for r in res]
    # --- device-resident timing ---
    times = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1.0)
            if dist:
                dist.barrier()
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            device_step()
            b.record(stream)
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b) / 1000.0)
        batch.fetch(sh)
        # --- end-to-end timing through the public API ---
        # the step's inputs: every instance's couplings, fields and beta in
        # pinned host memory (the lattices were fixed at batch creation)
        pw = torch.tensor(np.concatenate([np.asarray(d["weights"], float) for d in insts]),
                          dtype=torch.float64).pin_memory()
        ph = torch.tensor(np.concatenate([np.asarray(d["fields"], float) for d in insts]),
                          dtype=torch.float64).pin_memory()
        pb = torch.tensor([float(d["beta"]) for d in insts], dtype=torch.float64).pin_memory()
        pw_np, ph_np, pb_np = pw.numpy(), ph.numpy(), pb.numpy()

        def e2e_run(full_image):
            ts = []
            for _ in range(args.steps):
                flush.fill_(1.0)
                if dist:
                    dist.barrier()
                torch.cuda.synchronize()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                if full_image:
                    batch.upload(sh)
                else:
                    batch.set_params(pw_np, ph_np, pb_np, sh)
                batch.launch(sh)
                batch.fetch(sh)
                b.record(stream)
                torch.cuda.synchronize()
                ts.append(a.elapsed_time(b) / 1000.0)
            return ts

        e2e_times = e2e_run(False)
        e2e_res = batch.fetch(sh)
        e2e_check = max(abs(x.lnZ - y.lnZ) / max(1.0, abs(y.lnZ)) for x, y in zip(e2e_res, res_ref))
        e2e_full_times = e2e_run(True)   # last: leaves the host-built networks on the device
    total = sum(times)
    total_e2e = sum(e2e_times)
    total_full = sum(e2e_full_times)
    if dist:
        t = torch.tensor([total, total_e2e, total_full], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total, total_e2e, total_full = float(t[0]), float(t[1]), float(t[2])
    units = args.instances * world * args.steps
    value = units / total
    e2e_value = units / total_e2e
    if rank != 0:
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    peak, peak_kind = load_peaks()
    # error against the FP64 oracle on the instances the CPU leg contracted
    accuracy = {"vs": "FP64 oracle (numpy/OpenBLAS restatement of the reference algorithm)",
                "instances_compared": len(cpu_lz)}
    if cpu_lz:
        d_or = [abs(res_ref[q].lnZ - v) / insts[q]["n"] for q, v in cpu_lz.items()]
        accuracy["max_abs_dlnZ_per_spin"] = float(max(d_or))
        accuracy["median_abs_dlnZ_per_spin"] = float(statistics.median(d_or))
        accuracy["bar"] = 1e-6
        accuracy["within_bar"] = bool(max(d_or) <= 1e-6)
    fp64_peak = measure_dgemm_tflops()
    avg = total / args.steps
    achieved_gbs = nbytes / avg / 1e9
    traffic = read_traffic()
    out = {
        "metric": METRIC, "value": round(value, 3), "unit": "instances/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * avg, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_of(args, world),
        "engine": {"slots": batch.slots, "contraction_steps_total": int(sum(steps_per_inst)),
                   "statuses_nonzero": int(sum(1 for r in res_ref if r.status != 0))},
        "accuracy": accuracy,
        "e2e": {"value": round(e2e_value, 3), "unit": "instances/s",
                "h2d_bytes_per_step": int(batch.param_bytes),
                "d2h_bytes_per_step": int(args.instances * ctypes.sizeof(catn_lib.Result)),
                "inputs": "couplings, fields and beta of every instance (pinned host -> device); site tensors "
                          "rebuilt on the device (catn_ising_batch_set_params)",
                "max_rel_dlnZ_vs_host_built": float(e2e_check),
                "full_image": {"value": round(units / total_full, 3), "unit": "instances/s",
                               "h2d_bytes_per_step": int(batch.input_bytes),
                               "inputs": "the whole host-built network image (catn_batch_upload)"}},
        "gpu_launches": 4 * args.steps,
        "roofline": {"bound": "hbm", "achieved": round(achieved_gbs, 3), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved_gbs / peak, 6), "traffic": traffic,
                     "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)",
                     "algorithmic_bytes_per_launch": nbytes,
                     "algorithmic_fp64_flops_per_launch": flops,
                     "achieved_fp64_tflops": round(flops / avg / 1e12, 4),
                     "fp64": {"achieved": round(flops / avg / 1e12, 4), "peak": fp64_peak, "unit": "TFLOP/s",
                              "frac": round(flops / avg / 1e12 / fp64_peak, 5) if fp64_peak else None,
                              "peak_source": "cuBLAS DGEMM 8192^3 (torch.matmul float64), best of 5, "
                                             "measured in this run on this GPU"}},
        "clocks": clk.summary(),
    }
    if cpu:
        out["cpu_baseline"] = cpu
    if world == 1 and not args.no_grad:
        _secondary(out, "grad", lambda: grad_leg(catn, batch, insts, value, stream, sh))

    def plain_leg():
        rate, cnt, dev = plain_form_rate(insts, [r.lnZ for r in res], args.plain_seconds)
        return {
            "value": round(rate, 3), "unit": "instances/s", "value_over_plain": round(value / rate, 1),
            "max_abs_dlnZ_per_spin_vs_engine": dev,
            "sample": f"first {cnt} of the {args.instances} workload instances in order, one at a time, "
                      f"PyTorch FP64 on cuda:{local} (torch.linalg.svd/qr + einsum per op, host loop), "
                      f"~{args.plain_seconds:.0f} s wall clock"}
    if world == 1 and args.plain_seconds > 0:
        _secondary(out, "plain_gpu_form", plain_leg)
    if world == 1 and not args.no_c2:
        _secondary(out, "rrg200", lambda: c2_leg(catn, args, fp64_peak, load_bf16_peak()))
    if world == 1 and args.c4_full:
        _secondary(out, "gaussian_lattice_32", lambda: c4_full_leg(catn))
    if world == 1 and not args.no_configs:
        _secondary(out, "ferro8", lambda: c1_leg(catn))
        _secondary(out, "gaussian_lattice_reduced", lambda: c4_reduced_leg(catn))
        _secondary(out, "peps_reduced", lambda: peps_reduced_leg(catn))
    print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def _oracle_rrg200(beta):
    """FP64 oracle on the n=200 random-regular configuration (spawned
    process, all host cores to BLAS); returns (lnZ, seconds)."""
    from oracle import ising as OI, network as ON
    d = json.load(open(os.path.join(ROOT, "tests", "golden", "rrg200.json")))
    t0 = time.perf_counter()
    tn = OI.ising_network(d["n"], d["edges"], d["weights"], d["fields"], beta, **d["params"])
    lnZ, _, _ = ON.contraction(tn)
    return lnZ, time.perf_counter() - t0


def c2_leg(catn, args, fp64_peak=None, bf16_peak=None):
    """The n=200 random 3-regular +-1 spin glass (300 edges, h ~ N(0, 0.1^2),
    beta in {0.5, 1, 1.5}, Dmax 32, chi 128), one network per beta through
    the public API (host image in, results out), in two forms: FP64 on the
    block Jacobi route and the split precision form (3xTF32 tensor-core
    products, block route); with --c2-scalar also FP64 on the scalar Jacobi
    route.  The FP64 oracle is timed on beta = 1 on the host cores.  Errors are
    against the FP64 oracle's values frozen in tests/golden/rrg200.json (made
    by tests/golden/make_golden.py); the trace must equal the oracle's.
    Rates: algorithmic FLOPs of the contraction (the same per-step
    convention as the batch's roofline) per second, against the measured
    DGEMM rate (FP64 forms) or the TF32 rate (split form)."""
    d = json.load(open(os.path.join(ROOT, "tests", "golden", "rrg200.json")))
    edges = [tuple(e) for e in d["edges"]]
    res = {"workload": "random 3-regular +-1 spin glass, n=200 (300 edges), h~N(0,0.1^2), beta in {0.5,1,1.5}, "
                       "Dmax=32, chi=128, seed 200 (tests/golden/rrg200.json)",
           "timing": "host wall clock around catn.contraction (device move done before; the launch and the "
                     "result read-back inside)",
           "forms": {}}
    forms = ([("fp64_scalar", dict(svd_route="scalar"), [1.0])] if args.c2_scalar else []) + \
            [("fp64_block", dict(svd_route="block"), d["betas"]),
             ("split", dict(svd_route="block", precision="split"), d["betas"])]
    for name, kw, betas in forms:
        per = []
        for beta in betas:
            k = d["betas"].index(beta)
            ref = d["oracle"][k]
            tn = catn.ising_network(d["n"], edges, d["weights"], d["fields"], beta, **d["params"], **kw)
            catn.adapt(catn.B200, tn, trace=True)
            t0 = time.perf_counter()
            lnZ, err, psi = catn.contraction(tn, trace=True)
            dt = time.perf_counter() - t0
            rows = [[int(x) for x in r[:7]] for r in tn.trace]
            per.append({"beta": beta, "s": round(dt, 3), "abs_dlnZ_per_spin": abs(lnZ - ref["lnZ"]) / d["n"],
                        "trace_identical": rows == ref["trace"], "err": err, "oracle_err": ref["err"],
                        "algorithmic_tflops": round(tn.result.flops / dt / 1e12, 4)})
        rate = sum(p["algorithmic_tflops"] for p in per) / len(per)
        if name == "split":
            # the tensor pipe runs TF32 at half the bf16 rate; the split products
            # are three TF32 products each
            pk, src = (bf16_peak / 2, "half the measured sustained bf16 GEMM rate (MEASURED_PEAKS.json), "
                                      "the TF32 rate") \
                if bf16_peak else (None, None)
        else:
            pk, src = fp64_peak, "cuBLAS DGEMM measured in this run"
        res["forms"][name] = {"s_per_beta": round(sum(p["s"] for p in per) / len(per), 3),
                              "algorithmic_tflops": round(rate, 4),
                              "peak_tflops": pk, "peak_source": src,
                              "frac": round(rate / pk, 6) if pk else None,
                              "max_abs_dlnZ_per_spin": max(p["abs_dlnZ_per_spin"] for p in per),
                              "traces_identical": all(p["trace_identical"] for p in per), "runs": per}
    if not args.no_c2_oracle:
        with mp.get_context("spawn").Pool(1) as pool:
            lz, secs = pool.apply(_oracle_rrg200, (1.0,))
        res["oracle_fp64_cpu"] = {"beta": 1.0, "s": round(secs, 3), "cores": host_cores(),
                                  "what": "the oracle port (numpy/OpenBLAS, all cores to BLAS), same network"}
        b1 = [p["s"] for p in res["forms"]["fp64_block"]["runs"] if p["beta"] == 1.0]
        if b1:
            res["fp64_block_speedup_vs_oracle_at_beta_1"] = round(secs / b1[0], 2)
    return res


def c1_leg(catn):
    """The 8 x 8 open ferromagnet (w = 1, h = 0, beta = 0.44, Dmax 20, chi
    200), one network through the public API: latency of one contraction,
    lnZ per site and free energy (ising.jl:239-244), the error against the
    transfer-matrix value and the trace against the FP64 oracle's, both
    frozen in tests/golden/config1_ferro8.json, and the HBM fraction of the
    one launch (algorithmic bytes / CUDA-event time)."""
    import torch
    d = json.load(open(os.path.join(ROOT, "tests", "golden", "config1_ferro8.json")))
    edges = [tuple(e) for e in d["edges"]]
    times, out = [], None
    for rep in range(4):
        tn = catn.ising_network(d["n"], edges, d["weights"], d["fields"], d["beta"], **d["params"])
        catn.adapt(catn.B200, tn, trace=True)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        a.record()
        lnZ, err, psi = catn.contraction(tn, trace=True)
        b.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        if rep > 0:   # the first contraction is a warm-up
            times.append((a.elapsed_time(b) / 1e3, wall))
        out = (tn, lnZ, err)
    tn, lnZ, err = out
    dev_s = sum(t[0] for t in times) / len(times)
    rows = [[int(x) for x in r[:7]] for r in tn.trace]
    nbytes = tn.result.bytes
    peak, _ = load_peaks()
    return {"workload": "8x8 open square lattice, w=1, h=0, beta=0.44, Dmax=20, chi=200 (tests/golden/config1_ferro8.json)",
            "ms_per_contraction": round(1e3 * dev_s, 3),
            "ms_per_contraction_wall": round(1e3 * sum(t[1] for t in times) / len(times), 3),
            "lnZ_per_site": lnZ / d["n"], "free_energy_per_site": -lnZ / d["n"] / d["beta"],
            "abs_dlnZ_per_site_vs_transfer_matrix": abs(lnZ - d["exact_lnZ"]) / d["n"],
            "abs_dlnZ_per_site_vs_oracle": abs(lnZ - d["oracle"]["lnZ"]) / d["n"],
            "trace_identical_to_oracle": rows == d["oracle"]["trace"], "err": err,
            "roofline": {"bound": "hbm", "achieved": round(nbytes / dev_s / 1e9, 4), "peak": peak, "unit": "GB/s",
                         "frac": round(nbytes / dev_s / 1e9 / peak, 7) if peak else None,
                         "algorithmic_bytes": nbytes},
            "timing": "CUDA events around catn.contraction (upload, one launch, read-back), mean of 3 after one warm-up"}


def _oracle_fixture_time(name):
    """FP64 oracle on a frozen configuration (spawned process, all host cores
    to BLAS); returns (lnZ, seconds)."""
    from oracle import ising as OI, network as ON
    d = json.load(open(os.path.join(ROOT, "tests", "golden", name + ".json")))
    t0 = time.perf_counter()
    if name == "peps6":
        import __graft_entry__
        __graft_entry__.load_package()
        from catn_b200 import graphs
        _, _, et, ei = graphs.peps_double_layer(d["L"], d["D"], d["d"], np.random.default_rng(d["seed"]))
        tn = ON.TensorNetwork.from_tensors(et, ei, **d["params"])
    else:
        tn = OI.ising_network(d["n"], d["edges"], d["weights"], d["fields"], d["beta"], **d["params"])
    lnZ, _, _ = ON.contraction(tn)
    return lnZ, time.perf_counter() - t0


def _time_oracle(name):
    with mp.get_context("spawn").Pool(1) as pool:
        lz, secs = pool.apply(_oracle_fixture_time, (name,))
    return {"s": round(secs, 3), "lnZ": lz, "cores": host_cores(),
            "what": "the oracle port (numpy/OpenBLAS, all cores to BLAS), same network"}


def c4_reduced_leg(catn):
    """The 32 x 32 Gaussian lattice configuration (J ~ N(0,1), h ~ N(0,0.2^2),
    beta 1, Dmax 48, chi 256) at L = 10 (inputs and the FP64 oracle's lnZ and
    trace frozen in tests/golden/gaussian10.json): the forward contraction
    against the oracle, the device adjoint of lnZ (whole tape, and
    checkpointed every 64 steps), and the reference's pinning definition of
    every <s_k> and <s_i s_j> (1 + 2n + 4|E| networks, all of them: as one
    batch, and one network at a time as the reference's loop runs them),
    each timed through the public calls; the observables of the two routes
    are compared on every spin and edge."""
    d = json.load(open(os.path.join(ROOT, "tests", "golden", "gaussian10.json")))
    L, seed, n, beta = d["L"], 4, d["n"], d["beta"]
    edges = [tuple(e) for e in d["edges"]]
    w, h = np.array(d["weights"]), np.array(d["fields"])
    kw = dict(Dmax=48, chi=256)
    catn.contraction(catn.ising_network(n, edges, w, h, beta, **kw))   # warm-up
    t0 = time.perf_counter()
    lnZ, err, _ = catn.contraction(catn.ising_network(n, edges, w, h, beta, **kw))
    t_fwd = time.perf_counter() - t0
    grads = {}
    for k in (0, 64):
        net = catn.ising_network(n, edges, w, h, beta, **kw)
        catn.gradient(net, ckpt_interval=k)   # warm-up (allocates the gradient slot)
        t0 = time.perf_counter()
        lz_g, dw, dh = catn.gradient(net, ckpt_interval=k)
        grads[k] = (time.perf_counter() - t0, lz_g, dw, dh)
    inst = dict(n=n, edges=edges, weights=w, fields=h, beta=beta)
    pins = _pin_sets(inst)
    b = catn.IsingBatch([dict(inst, pos1=p1, val1=v1, pos2=p2, val2=v2) for (p1, v1, p2, v2) in pins], **kw)
    b.run()   # warm-up (allocates the slots)
    t0 = time.perf_counter()
    b.run()
    t_pin = time.perf_counter() - t0
    lz = b.lnZ()
    z1 = np.exp(lz[1:1 + 2 * n] - lz[0]).reshape(n, 2)
    m_pin = z1[:, 1] - z1[:, 0]   # val 2 pins spin +1, val 1 spin -1 (ising.jl:255-290)
    z2 = np.exp(lz[1 + 2 * n:] - lz[0]).reshape(len(edges), 2, 2)
    c_pin = z2[:, 0, 0] - z2[:, 0, 1] - z2[:, 1, 0] + z2[:, 1, 1]
    t_adj, lz_g, dw, dh = grads[0]
    # the reference's loop: every pinned network built and contracted on its
    # own (ising.jl:276-289, 321-337), through the same public calls
    t0 = time.perf_counter()
    lz_seq = [catn.contraction(catn.ising_network(n, edges, w, h, beta, pos1=p1, val1=v1, pos2=p2, val2=v2, **kw))[0]
              for (p1, v1, p2, v2) in pins]
    t_seq = time.perf_counter() - t0
    tn = catn.ising_network(n, edges, w, h, beta, **kw)
    catn.adapt(catn.B200, tn, trace=True)
    lz_t = catn.contraction(tn, trace=True)[0]
    rows = [[int(x) for x in r_[:7]] for r_ in tn.trace]
    vs_oracle = {"abs_dlnZ_per_site": abs(lz_t - d["oracle"]["lnZ"]) / n,
                 "trace_identical": rows == d["oracle"]["trace"], "oracle_cpu": _time_oracle("gaussian10")}
    return {"workload": f"{L}x{L} open lattice (the 32x32 configuration reduced), J~N(0,1), h~N(0,0.2^2), beta=1, "
                        f"Dmax=48, chi=256, seed {seed} (tests/golden/gaussian10.json)",
            "forward_s": round(t_fwd, 4), "lnZ": lnZ, "err": err, "vs_oracle": vs_oracle,
            "adjoint_s": round(t_adj, 4), "adjoint_ckpt64_s": round(grads[64][0], 4),
            "ckpt64_gradients_identical": bool(np.array_equal(grads[64][2], dw) and np.array_equal(grads[64][3], dh)),
            "pinning_networks": len(pins), "pinning_s": round(t_pin, 4),
            "speedup_adjoint_vs_pinning_batched": round(t_pin / t_adj, 2),
            "pinning_sequential_s": round(t_seq, 3),
            "speedup_adjoint_vs_pinning_sequential": round(t_seq / t_adj, 1),
            "max_abs_dlnZ_sequential_vs_batched": float(np.max(np.abs(np.array(lz_seq) - lz))),
            "max_abs_diff_magnetization": float(np.max(np.abs(dh / beta - m_pin))),
            "max_abs_diff_correlation": float(np.max(np.abs(dw / beta - c_pin))),
            "timing": "host wall clock around the public calls (network upload, launches and read-back inside), "
                      "after one warm-up call of each; pinning batched = one IsingBatch.run() over every pinned network, "
                      "sequential = ising_network + contraction per pinned network"}


def peps_reduced_leg(catn):
    """The 16 x 16 PEPS norm configuration reduced: the fused double layer of
    a random real L x L PEPS (d = 2, bond D, graphs.peps_double_layer, the
    construction of examples/peps_norm.jl:71-81) contracted as a
    TensorNetwork at Dmax / chi, in FP64 on the scalar and the block Jacobi
    routes and in split precision, each timed through the public calls; every
    form's lnZ and trace against the FP64 oracle's (frozen in
    tests/golden/peps6.json), whose own time on the host cores is measured."""
    from catn_b200 import graphs
    g = json.load(open(os.path.join(ROOT, "tests", "golden", "peps6.json")))
    L, D, seed, Dmax, chi = g["L"], g["D"], g["seed"], g["params"]["Dmax"], g["params"]["chi"]
    _, _, et, ei = graphs.peps_double_layer(L, D, g["d"], np.random.default_rng(seed))
    out = {"workload": f"{L}x{L} PEPS double layer, d=2, D={D} (bonds {D * D}), Dmax={Dmax}, chi={chi}, seed {seed}",
           "timing": "host wall clock around TensorNetwork + catn.contraction", "forms": {}}
    ref = None
    for name, kw in (("fp64_scalar", dict(svd_route="scalar")), ("fp64_block", dict(svd_route="block")),
                     ("split", dict(precision="split"))):
        t0 = time.perf_counter()
        net = catn.TensorNetwork(et, ei, Dmax=Dmax, chi=chi, **kw)
        catn.adapt(catn.B200, net, trace=True)
        lnZ, err, psi = catn.contraction(net, trace=True)
        dt = time.perf_counter() - t0
        ref = lnZ if ref is None else ref
        rows = [[int(x) for x in r_[:7]] for r_ in net.trace]
        out["forms"][name] = {"s": round(dt, 3), "lnZ": lnZ, "truncation_err": err, "psi": psi,
                              "abs_dlnZ_vs_fp64_scalar": abs(lnZ - ref),
                              "abs_dlnZ_vs_oracle": abs(lnZ - g["oracle"]["lnZ"]),
                              "trace_identical_to_oracle": rows == g["oracle"]["trace"],
                              "algorithmic_tflops": round(net.result.flops / dt / 1e12, 5)}
    out["oracle_cpu"] = _time_oracle("peps6")
    return out


def c4_full_leg(catn, L=32, seed=32, fd_edges=1, pin_edges=4):
    """The 32 x 32 Gaussian lattice at full size (J ~ N(0,1), h ~ N(0,0.2^2),
    beta 1, Dmax 48, chi 256): the forward contraction (FP64, and split
    precision against it), the checkpointed
    adjoint of lnZ (a checkpoint every 64 steps), central differences (step
    1e-5) on `fd_edges` couplings, and pinning of `pin_edges` edges (4
    networks each, one batch: one CTA per network, no helper CTAs), all
    through the public calls.  Progress goes
    to stderr as each part ends."""
    from catn_b200.graphs import square_edges
    r = np.random.default_rng(seed)
    n = L * L
    edges = square_edges(L)
    w, h, beta = r.normal(size=len(edges)), r.normal(0, 0.2, n), 1.0
    kw = dict(Dmax=48, chi=256)
    out = {"workload": f"{L}x{L} open lattice ({len(edges)} edges), J~N(0,1), h~N(0,0.2^2), beta=1, Dmax=48, chi=256, "
                       f"seed {seed}",
           "timing": "host wall clock around the public calls (network upload, launches and read-back inside)"}
    t0 = time.perf_counter()
    net = catn.ising_network(n, edges, w, h, beta, **kw)
    lnZ, err, _ = catn.contraction(net)
    t_fwd = time.perf_counter() - t0
    out.update(forward_s=round(t_fwd, 3), lnZ=lnZ, lnZ_per_site=lnZ / n, err=err,
               maxdim_intermediate=net.maxdim_intermediate,
               forward_engine_ms=round(net.result.prof[0] / 1.965e6, 1), forward_arena_peak=net.result.arena_peak)
    print("c4 forward", out["forward_s"], lnZ, err, file=sys.stderr, flush=True)
    # the split-precision form (3xTF32 tensor-core merges and block-route Grams)
    t0 = time.perf_counter()
    net_s = catn.ising_network(n, edges, w, h, beta, precision="split", **kw)
    lnZ_s, err_s, _ = catn.contraction(net_s)
    out["split"] = {"forward_s": round(time.perf_counter() - t0, 3), "lnZ": lnZ_s, "err": err_s,
                    "abs_dlnZ_per_site_vs_fp64": abs(lnZ_s - lnZ) / n,
                    "engine_ms": round(net_s.result.prof[0] / 1.965e6, 1)}
    print("c4 split forward", out["split"], file=sys.stderr, flush=True)
    t0 = time.perf_counter()
    lz_g, dw, dh = catn.gradient(catn.ising_network(n, edges, w, h, beta, **kw), ckpt_interval=64)
    t_adj = time.perf_counter() - t0
    out.update(adjoint_ckpt64_s=round(t_adj, 3), adjoint_lnZ_minus_forward=lz_g - lnZ)
    print("c4 adjoint", out["adjoint_ckpt64_s"], file=sys.stderr, flush=True)
    fd = []
    for q in r.choice(len(edges), size=fd_edges, replace=False).tolist():
        eps = 1e-5
        wp, wm = w.copy(), w.copy()
        wp[q] += eps
        wm[q] -= eps
        lp = catn.contraction(catn.ising_network(n, edges, wp, h, beta, **kw))[0]
        lm = catn.contraction(catn.ising_network(n, edges, wm, h, beta, **kw))[0]
        fd.append({"edge": q, "fd": (lp - lm) / (2 * eps), "adjoint": float(dw[q]),
                   "abs_diff": abs((lp - lm) / (2 * eps) - float(dw[q]))})
        print("c4 fd", fd[-1], file=sys.stderr, flush=True)
    out["central_differences"] = fd
    subset = sorted(r.choice(len(edges), size=pin_edges, replace=False).tolist())
    insts = [dict(n=n, edges=edges, weights=w, fields=h, beta=beta)]
    for q in subset:
        m, nn = edges[q]
        for v1 in (1, 2):
            for v2 in (1, 2):
                insts.append(dict(n=n, edges=edges, weights=w, fields=h, beta=beta, pos1=m, val1=v1, pos2=nn, val2=v2))
    # each pinned network's slot gets 1.5x the arena the forward run peaked at
    arena = max(1 << 30, int(1.5 * net.result.arena_peak) // 256 * 256)
    t0 = time.perf_counter()
    b = catn.IsingBatch(insts, slot_arena_bytes=arena, **kw)
    b.run()
    t_pin = time.perf_counter() - t0
    lz = b.lnZ()
    p = np.exp(lz[1:] - lz[0]).reshape(len(subset), 2, 2)
    c_pin = p[:, 0, 0] - p[:, 0, 1] - p[:, 1, 0] + p[:, 1, 1]
    npin = 1 + 2 * n + 4 * len(edges)
    out.update(pinning_subset_edges=len(subset), pinning_subset_networks=len(insts),
               pinning_subset_s=round(t_pin, 3), pinning_slots=b.slots, pinning_slot_arena=arena,
               max_abs_diff_correlation_vs_adjoint=float(np.max(np.abs(dw[subset] / beta - c_pin))),
               pinning_networks_full_definition=npin,
               pinning_full_s_at_subset_rate=round(t_pin / len(insts) * npin, 1),
               speedup_adjoint_vs_pinning_at_subset_rate=round(t_pin / len(insts) * npin / t_adj, 1),
               speedup_adjoint_vs_pinning_sequential_at_forward_time=round(npin * t_fwd / t_adj, 1))
    print("c4 pinning", t_pin, file=sys.stderr, flush=True)
    return out


def _pin_sets(d):
    """The reference's pinned networks of one instance: the unpinned one,
    both values of every spin (ising.jl:263-290) and the four value pairs of
    every edge (ising.jl:309-339)."""
    pins = [(0, 0, 0, 0)] + [(k, v, 0, 0) for k in range(1, d["n"] + 1) for v in (1, 2)]
    for (m, nn) in d["edges"]:
        for v1 in (1, 2):
            for v2 in (1, 2):
                pins.append((int(m), v1, int(nn), v2))
    return pins


def grad_leg(catn, batch, insts, forward_rate, stream, sh, sample=4):
    """Adjoint of the whole batch (one launch) against pinning, both measured."""
    import torch
    batch.grad_launch(sh)   # first call allocates the gradient slots
    batch.grad_fetch(sh)
    times = []
    for _ in range(3):
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        batch.grad_launch(sh)
        res, dw, dh = batch.grad_fetch(sh)
        b.record(stream)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b) / 1000.0)
    t_grad = sum(times) / len(times)
    pin = [1 + 2 * d["n"] + 4 * len(d["edges"]) for d in insts]
    # measured pinning: every pinned network of the first `sample` instances
    # in ONE batch launch (upload, launch and read-back inside CUDA events)
    kw = dict(PARAMS)
    pinned, owner = [], []
    for q in range(sample):
        d = insts[q]
        for p in _pin_sets(d):
            pinned.append(dict(n=d["n"], edges=d["edges"], weights=d["weights"], fields=d["fields"], beta=d["beta"],
                               pos1=p[0], val1=p[1], pos2=p[2], val2=p[3]))
            owner.append(q)
    pb = catn.IsingBatch(pinned, **kw)
    pb.upload(sh)
    pb.launch(sh)
    pb.fetch(sh)
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    pb.upload(sh)
    pb.launch(sh)
    pres = pb.fetch(sh)
    b.record(stream)
    torch.cuda.synchronize()
    t_pin_sample = a.elapsed_time(b) / 1000.0
    lz = np.array([r.lnZ for r in pres])
    pin_rate = len(pinned) / t_pin_sample
    # observables of the sample from pinning vs from the batch's adjoint run
    arr = batch._arrays
    dev, pos = 0.0, 0
    for q in range(sample):
        d = insts[q]
        n, ne = d["n"], len(d["edges"])
        z0 = lz[pos]
        pm = np.exp(lz[pos + 1:pos + 1 + 2 * n] - z0).reshape(n, 2)
        pc = np.exp(lz[pos + 1 + 2 * n:pos + 1 + 2 * n + 4 * ne] - z0).reshape(ne, 2, 2)
        pos += 1 + 2 * n + 4 * ne
        m_pin = pm[:, 1] - pm[:, 0]
        c_pin = pc[:, 0, 0] - pc[:, 0, 1] - pc[:, 1, 0] + pc[:, 1, 1]
        gh = dh[arr[1][q]:arr[1][q + 1]] / d["beta"]
        gw = dw[arr[2][q]:arr[2][q + 1]] / d["beta"]
        dev = max(dev, float(np.max(np.abs(gh - m_pin))), float(np.max(np.abs(gw - c_pin))))
    t_pin_batch = sum(pin) / pin_rate
    return {
        "what": "d lnZ/d w_e = beta <s_i s_j> for every edge and d lnZ/d h_k = beta <s_k> for every spin of "
                "every instance, one device gradient run (taped forward + backward) of the whole batch, against "
                "the reference's pinning definition (1 + 2n + 4|E| contractions per instance)",
        "adjoint_ms_per_batch": round(1000 * t_grad, 3),
        "adjoint_instances_per_s": round(len(insts) / t_grad, 3),
        "pinning_contractions_per_batch": int(sum(pin)),
        "pinning_measured": {"instances": sample, "contractions": len(pinned),
                             "ms": round(1000 * t_pin_sample, 3),
                             "contractions_per_s": round(pin_rate, 3),
                             "max_abs_observable_diff_vs_adjoint": dev},
        "pinning_ms_per_batch_at_measured_rate": round(1000 * t_pin_batch, 3),
        "speedup_vs_pinning": round(t_pin_batch / t_grad, 1),
        "timing": "CUDA events: adjoint = catn_batch_grad_launch (input upload + one launch) + read-back of "
                  "results and gradients, mean of 3; pinning = upload + one launch + read-back of every pinned "
                  "network of the first instances of the batch, whose measured rate prices the batch's pinned set",
    }


def measure_dgemm_tflops():
    """FP64 denominator: cuBLAS DGEMM 8192^3 on this GPU, best of 5 (CUDA
    events).  The measured-peaks file holds no FP64 figure."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    best = None
    for _ in range(6):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1000.0
        best = t if best is None else min(best, t)
    del a, b
    torch.cuda.empty_cache()
    return round(2.0 * n ** 3 / best / 1e12, 3)


def ct_stream(stream):
    import ctypes
    return ctypes.c_void_p(stream.cuda_stream)


if __name__ == "__main__":
    main()
