"""The decoder's own exp/log (sg_math.h): accuracy against mpmath and
agreement with the system libm that the reference uses."""
import numpy as np
import pytest

from oracle_api import Oracle


def _ulp_err(x, y_exact):
    import mpmath as mp

    y = float(x)
    u = mp.mpf(np.spacing(abs(y)))
    return float(abs(mp.mpf(y) - y_exact) / u)


@pytest.fixture(scope="module")
def twin(oracle_paths):
    return Oracle(oracle_paths["twin"])


@pytest.fixture(scope="module")
def libm(oracle_paths):
    return Oracle(oracle_paths["libm"])


def test_exp_log_accuracy_vs_mpmath(twin):
    import mpmath as mp

    mp.mp.prec = 120
    rng = np.random.default_rng(3)
    worst_e = worst_l = 0.0
    for x in np.concatenate([rng.uniform(-50, 50, 1500), rng.uniform(-740, 0, 500), rng.uniform(-1e-3, 1e-3, 300)]):
        worst_e = max(worst_e, _ulp_err(twin.lib.sgo_exp(float(x)), mp.exp(mp.mpf(float(x)))))
    for x in np.concatenate([rng.uniform(0.5, 1.5, 1500), np.exp(rng.uniform(-92, 50, 700)),
                             1 + rng.uniform(-2e-3, 2e-3, 300)]):
        worst_l = max(worst_l, _ulp_err(twin.lib.sgo_log(float(x)), mp.log(mp.mpf(float(x)))))
    assert worst_e < 0.52, worst_e
    assert worst_l < 0.52, worst_l


def test_special_values(twin):
    e, l = twin.lib.sgo_exp, twin.lib.sgo_log
    assert e(0.0) == 1.0 and e(-800.0) == 0.0 and e(800.0) == float("inf")
    assert np.isnan(e(float("nan")))
    assert l(1.0) == 0.0 and l(0.0) == float("-inf") and np.isnan(l(-1.0))
    assert l(float("inf")) == float("inf")
    assert l(1e-310) == np.log(1e-310)  # subnormal input


def test_agreement_with_libm(twin, libm):
    """Within 1 ulp everywhere and equal on all but ~1e-3 of arguments."""
    rng = np.random.default_rng(11)
    xs = rng.uniform(-50, 50, 20000)
    a = np.array([twin.lib.sgo_exp(float(x)) for x in xs])
    b = np.array([libm.lib.sgo_exp(float(x)) for x in xs])
    d = np.abs(a.view(np.int64) - b.view(np.int64))
    assert d.max() <= 1 and (d != 0).mean() < 3e-3
    ys = rng.uniform(0.5, 2.0, 20000)
    a = np.array([twin.lib.sgo_log(float(y)) for y in ys])
    b = np.array([libm.lib.sgo_log(float(y)) for y in ys])
    d = np.abs(a.view(np.int64) - b.view(np.int64))
    assert d.max() <= 1 and (d != 0).mean() < 5e-3
