"""Host-side behaviour of the Python mirror that needs no device: label
resolution, input dtypes, and the errors the reference raises while building
a network (src/tensor_network.jl:56-116)."""
import numpy as np
import pytest


def test_float32_tensors_are_contracted_in_fp64(catn):
    """The reference's Float32 path (test/test_gpu.jl:66-73) contracts at
    Float32 precision; the device engine takes the same tensors in FP64."""
    r = np.random.default_rng(1)
    ts = [r.normal(size=(3, 4)).astype(np.float32), r.normal(size=(4, 5)).astype(np.float32),
          r.normal(size=(5, 3)).astype(np.float32)]
    tn = catn.TensorNetwork(ts, [["a", "b"], ["b", "c"], ["c", "a"]], Dmax=-1, chi=10_000)
    assert all(t.dtype == np.float64 for t in tn.tensors)
    assert all(np.array_equal(a, b.astype(np.float64)) for a, b in zip(tn.tensors, ts))
    assert tn.neighbors == [[3, 2], [1, 3], [2, 1]]   # a label's other end, per leg


def test_complex_tensors_are_rejected(catn):
    ts = [np.ones((2, 2), dtype=complex), np.ones((2, 2))]
    with pytest.raises(NotImplementedError):
        catn.TensorNetwork(ts, [["a", "b"], ["b", "a"]])


@pytest.mark.parametrize("ixs,msg", [
    ([["a", "a"], ["a", "b"]], "Self-loop"),
    ([["a", "b"], ["a", "b"], ["a", "c"]], "appears in 3 tensors"),
])
def test_label_errors(catn, ixs, msg):
    ts = [np.ones((2,) * len(ix)) for ix in ixs]
    with pytest.raises(ValueError, match=msg):
        catn.TensorNetwork(ts, ixs)


def test_open_legs_get_negative_sentinels(catn):
    ts = [np.ones((2, 3)), np.ones((3, 4))]
    tn = catn.TensorNetwork(ts, [["p", "b"], ["b", "q"]])
    assert tn.neighbors[0][1] == 2 and tn.neighbors[1][0] == 1
    assert tn.neighbors[0][0] < 0 and tn.neighbors[1][1] < 0 and tn.neighbors[0][0] != tn.neighbors[1][1]
