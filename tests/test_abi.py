"""The C-ABI library loads and exports every symbol include/sogrand_b200.h
declares; argument errors are reported without touching a GPU."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "sogrand_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(sg):
    from sogrand_b200 import _lib

    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.symbols()), "binding and header disagree"
    nm = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (sg_[a-z0-9_]+)", nm))
    assert set(names) <= exported


def test_version_and_status_strings(sg):
    from sogrand_b200 import _lib

    lib = _lib.load()
    assert b"sm_100a" in lib.sg_version()
    assert lib.sg_status_string(0) == b"ok"
    assert lib.sg_status_string(3) == b"non-finite input"


def test_params_default_is_reference(sg):
    p = sg.params()
    assert (p.L, p.Imax, p.Tmax) == (3, 30, (1 << 64) - 1)
    assert p.thres == 1.0 - 1e-5
    assert all(a == 0.7 for a in p.alpha)


def test_reference_alpha_mapping(sg):
    a = np.arange(100, dtype=np.float64)
    ph = sg.reference_alpha(a)
    # iteration 1: columns alpha[0], rows alpha[1], slices alpha[1]
    assert list(ph[:6]) == [0, 1, 1, 2, 3, 3]


@pytest.mark.parametrize("field,value", [("L", 0), ("L", 9), ("Imax", 0), ("Imax", 51)])
def test_bad_params_rejected_before_gpu(sg, field, value):
    from sogrand_b200 import _lib

    p = sg.params()
    setattr(p, field, value)
    lib = _lib.load()
    st = lib.sg_decode_device(None, 1, C.byref(p), None, None, None, None)
    assert st == 1
    assert b"must be in" in lib.sg_last_error()


def test_nonfinite_alpha_rejected(sg):
    from sogrand_b200 import _lib

    p = sg.params()
    p.alpha[5] = float("nan")
    assert _lib.load().sg_decode_host(None, 1, C.byref(p), None, None, None) == 1


def test_zero_codewords_is_ok(sg):
    from sogrand_b200 import _lib

    p = sg.params()
    assert _lib.load().sg_decode_device(None, 0, C.byref(p), None, None, None, None) == 0


def test_missing_input_file_is_io_error(sg, tmp_path):
    with pytest.raises(sg.SograndError) as e:
        sg.decode_file(str(tmp_path / "nope.bin"), str(tmp_path / "out.bin"))
    assert e.value.status == 4


def test_cli_usage(sg):
    exe = os.path.join(ROOT, "sogrand_b200", "bin", "cubic_decoder")
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 1
    assert r.stderr.startswith("Usage: ") and "<input_llr_file> <output_file>" in r.stderr


def test_wilson_interval(sg):
    lo, hi = sg.wilson_interval(0, 1000)
    assert lo == 0.0 and 0.0038 < hi < 0.0039
    lo, hi = sg.wilson_interval(50, 100)
    assert abs(lo - 0.40383) < 1e-4 and abs(hi - 0.59617) < 1e-4
    assert sg.wilson_interval(7, 7)[1] == 1.0
    with pytest.raises(sg.SograndError):
        sg.wilson_interval(5, 4)


def test_wait_limit_is_clamped(sg):
    """The device wait limit is process state only; no GPU is touched."""
    from sogrand_b200 import _lib

    lib = _lib.load()
    old = lib.sg_get_wait_limit()
    assert old == 1 << 22
    try:
        assert lib.sg_set_wait_limit(1 << 40) == 0
        assert lib.sg_get_wait_limit() == 1 << 22
        assert lib.sg_set_wait_limit(5) == 0 and lib.sg_get_wait_limit() == 5
    finally:
        lib.sg_set_wait_limit(old)


def test_autograd_wrapper_rejects_misshapen_tensors(sg):
    """The differentiable decode checks dtype, device and layout before it
    hands pointers to the C ABI (no GPU needed to see the rejection)."""
    import torch

    from sogrand_b200 import diff

    alpha = torch.full((90,), 0.7, dtype=torch.float64)
    bits = torch.zeros((2, 4096), dtype=torch.uint8)
    for bad in (torch.zeros((2, 4096), dtype=torch.float32), torch.zeros((2, 4096), dtype=torch.float64),
                torch.zeros((4096, 2), dtype=torch.float64).t()):
        with pytest.raises(ValueError):
            diff.decode_bce(alpha, bad, bits)
