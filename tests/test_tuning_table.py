"""The process-wide tuning table through the C ABI (no GPU needed): the
built-in defaults, a round trip through catn_tuning_set / _get, rejection of
invalid entries, and the tuner's save / load of a table."""
import pytest


@pytest.fixture
def tune():
    from catn_b200 import tune as T
    saved = T.get()
    yield T
    T.apply(saved)


def test_builtin_defaults(tune):
    t = tune.get()
    assert t["helper_ctas"] == 16 and t["shared_jacobi_min_n"] == 128
    assert t["block_min_n"] == 192 and t["shared_house_min"] == 1 << 20
    assert t["blocked_qr_min_n"] == 1 << 30   # the blocked QR is off unless a table turns it on


def test_round_trip(tune):
    want = dict(helper_ctas=8, grad_helper_ctas=4, shared_jacobi_min_n=96, block_min_n=128,
                shared_house_min=1 << 18, blocked_qr_min_n=256)
    got = tune.apply(want)
    assert {k: got[k] for k in want} == want
    assert {k: tune.get()[k] for k in want} == want


@pytest.mark.parametrize("bad", [dict(block_min_n=2), dict(helper_ctas=5000), dict(grad_helper_ctas=4097)])
def test_invalid_entries_rejected(tune, bad):
    from catn_b200 import CatnError
    before = tune.get()
    with pytest.raises(CatnError):
        tune.apply(bad)
    assert tune.get() == before


def test_save_and_load(tune, tmp_path):
    p = tmp_path / "tuning.json"
    res = {"table": dict(tune.get(), helper_ctas=12), "measurements": {}, "device": "test"}
    tune.save(res, str(p))
    assert tune.load(str(p))["table"]["helper_ctas"] == 12
