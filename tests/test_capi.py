"""The C ABI library: loads on a CPU-only machine, exports every symbol that
include/catn_b200.h declares (with the ctypes signatures the package binds),
and fails loudly -- an error status, never a CPU fallback -- when no CUDA
device is present."""
import ctypes as ct
import os
import re
import subprocess

import pytest

from catn_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "catn_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(catn_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_bound_symbols():
    assert set(declared_symbols()) == set(L.SIGNATURES)


def test_library_exports_every_declared_symbol():
    lib = L.load()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (catn_[a-z0-9_]+)\b", out))
    assert set(declared_symbols()) <= exported


def test_params_default_matches_reference_kwargs():
    lib = L.load()
    p = L.Params()
    lib.catn_params_default(ct.byref(p))
    # TensorNetwork defaults (tensor_network.jl:41-54)
    assert (p.Dmax, p.chi, p.cutoff, p.norm_method, p.select) == (32, 32, 1e-15, 1, 1)
    assert (p.reverse, p.svdopt, p.swapopt, p.compress, p.cut_bond, p.seed) == (1, 1, 1, 0, 0, 1)
    assert lib.catn_version().startswith(b"catn_b200")


def test_invalid_params_rejected():
    lib = L.load()
    p = L.make_params(Dmax=0)
    h = ct.c_void_p()
    e = (ct.c_int32 * 2)(1, 2)
    w = (ct.c_double * 1)(1.0)
    f = (ct.c_double * 2)(0.0, 0.0)
    st = lib.catn_ising_create(ct.byref(p), 2, 1, e, w, f, 1.0, 0, 0, 0, 0, 0, ct.byref(h))
    assert st == L.CATN_EINVAL
    assert "Dmax" in L.last_error(lib)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device behaviour")
def test_no_device_fails_loudly(catn):
    tn = catn.ising_network(3, [(1, 2), (2, 3)], [1.0, 1.0], [0.0] * 3, 0.5, Dmax=-1, chi=100)
    with pytest.raises(catn.CatnError) as ei:
        catn.contraction(tn)
    assert ei.value.status == L.CATN_ECUDA
