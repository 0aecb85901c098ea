"""The decoder's exp and log.

In its reference-exact mode the kernel evaluates exp/log with the correctly
rounded routines of sogrand_b200/csrc/sg_crmath.h (the same source on host
and device, built into the twin_cr oracle).  They are checked here on the
host, through that oracle,
against two independent references: mpmath at 200 bits, and the binary128
checker of oracle/crq.h (libsg_oracle_crq.so) on large samples, on the
structured arguments the decoder produces (1 +- m 2^-52: JacLog of large
|LLR|), on subnormal and overflow boundaries, and with the slow paths forced.
The table-driven routines of sg_math.h -- the default decoder's, and the
input generator's -- are checked for their 0.51 ulp bound."""
import ctypes as C

import numpy as np
import pytest

from oracle_api import Oracle


def _ulp_err(y, y_exact):
    import mpmath as mp

    u = mp.mpf(np.spacing(abs(float(y_exact))))
    return float(abs(mp.mpf(float(y)) - y_exact) / u)


@pytest.fixture(scope="module")
def twin(oracle_paths):
    o = Oracle(oracle_paths["twin_cr"])
    for name in ("sgo_exp_cr_slow", "sgo_log_cr_slow", "sgo_exp_tab", "sgo_log_tab"):
        f = getattr(o.lib, name)
        f.restype = C.c_double
        f.argtypes = [C.c_double]
    return o


@pytest.fixture(scope="module")
def libm(oracle_paths):
    return Oracle(oracle_paths["libm"])


@pytest.fixture(scope="module")
def crq(oracle_paths):
    if oracle_paths.get("crq") is None:
        pytest.skip("libsg_oracle_crq.so (needs libquadmath) not built")
    return Oracle(oracle_paths["crq"])


def _exp_args(rng, n):
    return np.concatenate([
        -rng.uniform(0, 60, n),                 # the guess loop's exp(-PM)
        rng.uniform(-50, 50, n),                # JacLog
        rng.uniform(-745.2, 709.8, n // 4),     # whole range
        rng.uniform(-745.2, -707.0, n // 8),    # subnormal results
        rng.uniform(705.0, 709.8, n // 8),      # near overflow
        rng.uniform(-1e-12, 1e-12, n // 8),     # near 1
    ])


def _log_args(rng, n):
    sub = np.frombuffer(rng.integers(1, 1 << 52, n // 8, dtype=np.int64).tobytes(), np.float64)
    return np.concatenate([
        1.0 + np.exp(-rng.uniform(0, 40, n)),   # JacLog arguments
        np.exp(-rng.uniform(0, 92.1, n)),       # soft output p0, p1
        np.exp(rng.uniform(-700, 700, n // 4)),
        1.0 + rng.uniform(-0.01, 0.01, n // 4),
        sub,
    ])


def _differ(f, g, xs):
    a = np.array([f(float(x)) for x in xs])
    b = np.array([g(float(x)) for x in xs])
    return np.flatnonzero(a.view(np.int64) != b.view(np.int64))


def test_correctly_rounded_vs_mpmath(twin):
    import mpmath as mp

    mp.mp.prec = 200
    rng = np.random.default_rng(3)
    for x in _exp_args(rng, 400):
        ex = mp.exp(mp.mpf(float(x)))
        if ex < mp.mpf(2) ** -1022:  # subnormal: the grid is absolute
            assert abs(mp.mpf(twin.lib.sgo_exp(float(x))) - ex) <= mp.mpf(2) ** -1075, x
        else:
            assert _ulp_err(twin.lib.sgo_exp(float(x)), ex) <= 0.5, x
    for x in _log_args(rng, 400):
        assert _ulp_err(twin.lib.sgo_log(float(x)), mp.log(mp.mpf(float(x)))) <= 0.5, x


def test_correctly_rounded_vs_binary128(twin, crq):
    rng = np.random.default_rng(17)
    xs = _exp_args(rng, 40000)
    bad = _differ(twin.lib.sgo_exp, crq.lib.sgo_exp, xs)
    assert bad.size == 0, [float(xs[i]).hex() for i in bad[:5]]
    ys = _log_args(rng, 40000)
    bad = _differ(twin.lib.sgo_log, crq.lib.sgo_log, ys)
    assert bad.size == 0, [float(ys[i]).hex() for i in bad[:5]]


def test_structured_log_arguments(twin, crq):
    """1 + m 2^-52 and 1 - m 2^-53: log(1 + e^-|L|) for |L| between 30 and
    50 takes these values, and many have exact images within 2^-105 of a
    midpoint."""
    m = np.arange(1, 1 << 15, dtype=np.float64)
    for xs in (1.0 + m * 2.0 ** -52, 1.0 - m * 2.0 ** -53, 1.0 + m * 2.0 ** -40):
        bad = _differ(twin.lib.sgo_log, crq.lib.sgo_log, xs)
        assert bad.size == 0, [float(xs[i]).hex() for i in bad[:5]]


def test_slow_paths_alone(twin, crq):
    """The double-double slow paths, run on every argument (normally about
    one in 2^12), give the correctly rounded result too."""
    rng = np.random.default_rng(23)
    xs = _exp_args(rng, 5000)
    bad = _differ(twin.lib.sgo_exp_cr_slow, crq.lib.sgo_exp, xs)
    assert bad.size == 0, [float(xs[i]).hex() for i in bad[:5]]
    ys = _log_args(rng, 5000)
    bad = _differ(twin.lib.sgo_log_cr_slow, crq.lib.sgo_log, ys)
    assert bad.size == 0, [float(ys[i]).hex() for i in bad[:5]]


def test_special_values(twin):
    e, l = twin.lib.sgo_exp, twin.lib.sgo_log
    assert e(0.0) == 1.0 and e(-0.0) == 1.0 and e(-800.0) == 0.0 and e(800.0) == float("inf")
    assert np.isnan(e(float("nan"))) and e(float("-inf")) == 0.0 and e(float("inf")) == float("inf")
    assert e(float.fromhex("0x1.62e42fefa39efp+9")) < float("inf")
    assert e(float.fromhex("0x1.62e42fefa39f0p+9")) == float("inf")
    assert e(float.fromhex("-0x1.74910d52d3051p+9")) == 5e-324
    assert e(float.fromhex("-0x1.74910d52d3052p+9")) == 0.0
    assert l(1.0) == 0.0 and l(0.0) == float("-inf") and np.isnan(l(-1.0)) and np.isnan(l(float("nan")))
    assert l(float("inf")) == float("inf")
    assert l(5e-324) == np.log(5e-324) and l(1e-310) == np.log(1e-310)  # subnormal inputs


def test_table_routines_accuracy(twin):
    """sg_math.h's table-driven exp/log: < 0.51 ulp."""
    import mpmath as mp

    mp.mp.prec = 120
    rng = np.random.default_rng(3)
    worst_e = worst_l = 0.0
    for x in np.concatenate([rng.uniform(-50, 50, 1500), rng.uniform(-740, 0, 500), rng.uniform(-1e-3, 1e-3, 300)]):
        worst_e = max(worst_e, _ulp_err(twin.lib.sgo_exp_tab(float(x)), mp.exp(mp.mpf(float(x)))))
    for x in np.concatenate([rng.uniform(0.5, 1.5, 1500), np.exp(rng.uniform(-92, 50, 700)),
                             1 + rng.uniform(-2e-3, 2e-3, 300)]):
        worst_l = max(worst_l, _ulp_err(twin.lib.sgo_log_tab(float(x)), mp.log(mp.mpf(float(x)))))
    assert worst_e < 0.52, worst_e
    assert worst_l < 0.52, worst_l


def test_agreement_with_glibc(twin, libm):
    """glibc's exp/log (the reference's libm here) are not correctly rounded:
    they differ from the correctly rounded ones by one ulp on a small
    fraction of arguments, never more."""
    rng = np.random.default_rng(11)
    xs = rng.uniform(-50, 50, 20000)
    a = np.array([twin.lib.sgo_exp(float(x)) for x in xs])
    b = np.array([libm.lib.sgo_exp(float(x)) for x in xs])
    d = np.abs(a.view(np.int64) - b.view(np.int64))
    assert d.max() <= 1 and (d != 0).mean() < 2e-3
    ys = rng.uniform(0.5, 2.0, 20000)
    a = np.array([twin.lib.sgo_log(float(y)) for y in ys])
    b = np.array([libm.lib.sgo_log(float(y)) for y in ys])
    d = np.abs(a.view(np.int64) - b.view(np.int64))
    assert d.max() <= 1 and (d != 0).mean() < 2e-3
