"""ctypes binding of libcatn_b200.so (the C ABI declared in include/catn_b200.h).

The shared library is the only compute path: importing the package works
without it (so that tests can inspect the package on a CPU-only machine), but
every call that contracts a network raises ``CatnError`` if the library or a
CUDA device is missing.  There is no CPU fallback.
"""
import ctypes as ct
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcatn_b200.so")

CATN_OK, CATN_EINVAL, CATN_ENOMEM, CATN_ENOCONV, CATN_ETIMEOUT, CATN_ECUDA, CATN_ESTATE = range(7)


class CatnError(RuntimeError):
    """Error raised for a non-zero catn_status (the reference raises Julia
    exceptions via ``error(...)``/``@assert`` at the same points)."""

    def __init__(self, status, msg):
        super().__init__(f"[catn status {status}] {msg}")
        self.status = status


class Params(ct.Structure):
    """``catn_params``: keyword arguments of TensorNetwork / ising_network."""
    _fields_ = [("Dmax", ct.c_int32), ("chi", ct.c_int32), ("cutoff", ct.c_double),
                ("norm_method", ct.c_int32), ("select", ct.c_int32), ("reverse", ct.c_int32),
                ("svdopt", ct.c_int32), ("swapopt", ct.c_int32), ("compress", ct.c_int32),
                ("cut_bond", ct.c_int32), ("seed", ct.c_int32), ("trace", ct.c_int32), ("rsvd", ct.c_int32),
                ("rsvd_min_dim", ct.c_int32), ("precision", ct.c_int32), ("svd_route", ct.c_int32),
                ("ckpt_interval", ct.c_int32), ("braket_loops", ct.c_int32)]


class Tuning(ct.Structure):
    """``catn_tuning``: the process-wide launch-shape and route table."""
    _fields_ = [("helper_ctas", ct.c_int32), ("grad_helper_ctas", ct.c_int32),
                ("shared_jacobi_min_n", ct.c_int32), ("block_min_n", ct.c_int32),
                ("shared_house_min", ct.c_int64), ("blocked_qr_min_n", ct.c_int32), ("reserved", ct.c_int32)]


class Result(ct.Structure):
    """``catn_result``."""
    _fields_ = [("lnZ", ct.c_double), ("err", ct.c_double), ("psi", ct.c_double),
                ("sign", ct.c_double), ("maxdim", ct.c_int32), ("status", ct.c_int32),
                ("nsteps", ct.c_int32), ("jacobi_max", ct.c_int32), ("arena_peak", ct.c_int64),
                ("flops", ct.c_double), ("bytes", ct.c_double), ("prof", ct.c_double * 24)]


# Every exported symbol with its ctypes signature (argtypes, restype).
_P = ct.c_void_p
SIGNATURES = {
    "catn_params_default": ([ct.POINTER(Params)], None),
    "catn_net_create_mps": ([ct.POINTER(Params), ct.c_int32, _P, _P, _P, _P, _P, _P, ct.c_int64,
                             ct.POINTER(ct.c_void_p)], ct.c_int),
    "catn_net_create_dense": ([ct.POINTER(Params), ct.c_int32, _P, _P, _P, _P, ct.c_int64,
                               ct.POINTER(ct.c_void_p)], ct.c_int),
    "catn_contract": ([ct.c_void_p, ct.POINTER(Result), _P, ct.c_int32], ct.c_int),
    "catn_cut_bondim": ([ct.c_void_p, ct.c_int32, ct.c_int32, ct.c_int32, ct.POINTER(ct.c_double)], ct.c_int),
    "catn_result_tensor": ([ct.c_void_p, _P, ct.c_int64, ct.POINTER(ct.c_int64),
                            ct.POINTER(ct.c_int32), _P], ct.c_int),
    "catn_net_destroy": ([ct.c_void_p], ct.c_int),
    "catn_ising_create": ([ct.POINTER(Params), ct.c_int32, ct.c_int32, _P, _P, _P, ct.c_double,
                           ct.c_int32, ct.c_int32, ct.c_int32, ct.c_int32, ct.c_int64,
                           ct.POINTER(ct.c_void_p)], ct.c_int),
    "catn_ising_batch_create": ([ct.POINTER(Params), ct.c_int32, _P, _P, _P, _P, _P, _P, _P, _P,
                                 ct.c_int64, ct.c_int32, ct.POINTER(ct.c_void_p)], ct.c_int),
    "catn_batch_run": ([ct.c_void_p, _P], ct.c_int),
    "catn_batch_launch": ([ct.c_void_p, ct.c_void_p], ct.c_int),
    "catn_batch_upload": ([ct.c_void_p, ct.c_void_p], ct.c_int),
    "catn_batch_results": ([ct.c_void_p, _P, ct.c_void_p], ct.c_int),
    "catn_batch_slots": ([ct.c_void_p], ct.c_int32),
    "catn_batch_input_bytes": ([ct.c_void_p], ct.c_int64),
    "catn_batch_destroy": ([ct.c_void_p], ct.c_int),
    "catn_ising_batch_set_params": ([ct.c_void_p, _P, _P, _P, ct.c_void_p], ct.c_int),
    "catn_ising_batch_randomize": ([ct.c_void_p, ct.c_uint64, ct.c_double, ct.c_double, ct.c_void_p], ct.c_int),
    "catn_ising_batch_get_params": ([ct.c_void_p, _P, _P, _P], ct.c_int),
    "catn_ising_batch_param_bytes": ([ct.c_void_p], ct.c_int64),
    "catn_braket_create": ([ct.POINTER(Params), ct.c_int32, _P, _P, _P, _P, ct.c_int64, ct.POINTER(ct.c_void_p)],
                           ct.c_int),
    "catn_ising_grad": ([ct.c_void_p, ct.POINTER(Result), _P, _P, ct.c_int32], ct.c_int),
    "catn_batch_grad_launch": ([ct.c_void_p, _P], ct.c_int),
    "catn_batch_grad_results": ([ct.c_void_p, _P, _P, _P, _P], ct.c_int),
    "catn_ising_contract_static": ([ct.POINTER(Params), ct.c_int32, ct.c_int32, _P, _P, _P, ct.c_double,
                                    ct.c_int32, ct.c_int32, ct.c_int32, ct.c_int32, ct.c_void_p,
                                    ct.POINTER(Result)], ct.c_int),
    "catn_tc_matmul": ([ct.c_int32, ct.c_int32, ct.c_int32, _P, _P, _P], ct.c_int),
    "catn_tuning_get": ([ct.POINTER(Tuning)], ct.c_int),
    "catn_tuning_set": ([ct.POINTER(Tuning)], ct.c_int),
    "catn_last_error": ([ct.c_char_p, ct.c_size_t], ct.c_size_t),
    "catn_release_cached_memory": ([], ct.c_int),
    "catn_cached_bytes": ([ct.c_int32], ct.c_int64),
    "catn_version": ([], ct.c_char_p),
}

_lib = None


def load(path=None):
    """Load (once) and return the library; raise CatnError if it is absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or os.environ.get("CATN_B200_LIB") or LIB_PATH
    if not os.path.exists(p):
        raise CatnError(CATN_ECUDA, f"libcatn_b200.so not built ({p}); run __graft_entry__.build()")
    lib = ct.CDLL(p)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if path is None:
        _lib = lib
        _apply_committed_tuning(lib)
    return lib


TUNING_PATH = os.path.join(_HERE, "tuning_b200.json")


def _apply_committed_tuning(lib):
    """Install the autotuner's table (tune.py) if one is saved beside the
    package; entries absent from it keep the built-in defaults."""
    if not os.path.exists(TUNING_PATH):
        return
    import json
    with open(TUNING_PATH) as f:
        table = json.load(f).get("table", {})
    t = Tuning()
    check(lib, lib.catn_tuning_get(ct.byref(t)))
    for name, _ in Tuning._fields_:
        if name in table:
            setattr(t, name, int(table[name]))
    check(lib, lib.catn_tuning_set(ct.byref(t)))


def last_error(lib):
    buf = ct.create_string_buffer(1024)
    lib.catn_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(lib, status):
    if status != CATN_OK:
        raise CatnError(status, last_error(lib))


def ptr(a):
    return a.ctypes.data_as(ct.c_void_p) if a is not None else None


PRECISIONS = {"fp64": 0, "split": 1}
SVD_ROUTES = {"auto": 0, "scalar": 1, "block": 2}


def make_params(Dmax=32, chi=32, cutoff=1e-15, norm_method=1, select=1, reverse=True, svdopt=True,
                swapopt=True, compress=False, cut_bond=False, seed=1, trace=False, rsvd=0, rsvd_min_dim=0,
                precision="fp64", svd_route="auto", ckpt_interval=0, braket_loops=False):
    """``catn_params`` from the reference's keywords plus the engine's own:
    ``rsvd`` / ``rsvd_min_dim`` (randomized swap route), ``precision``
    ("fp64" or "split"), ``svd_route`` ("auto", "scalar", "block") and
    ``ckpt_interval`` (gradient runs: steps between checkpoints, 0 = whole
    tape) and ``braket_loops`` (BraKet networks with cycles)."""
    prec = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    route = SVD_ROUTES[svd_route] if isinstance(svd_route, str) else int(svd_route)
    return Params(int(Dmax), int(chi), float(cutoff), int(norm_method), int(select), int(bool(reverse)),
                  int(bool(svdopt)), int(bool(swapopt)), int(bool(compress)), int(bool(cut_bond)),
                  int(seed), int(bool(trace)), int(rsvd), int(rsvd_min_dim), prec, route, int(ckpt_interval),
                  int(bool(braket_loops)))
