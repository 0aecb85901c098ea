"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def _ensure_built(target_dir, files):
    if not all(os.path.exists(os.path.join(target_dir, f)) for f in files):
        subprocess.run(["make", "-C", target_dir], check=True, capture_output=True)


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def kat():
    return dict(np.load(os.path.join(GOLDEN, "kat_lines.npz")))


@pytest.fixture(scope="session")
def oracle_paths():
    """The CPU checkers (built from oracle/ if missing): "libm" (glibc
    exp/log), "twin" and "twin_cr" (the decoder's table-driven and correctly
    rounded exp/log); "crq" (the binary128 checker, needs libquadmath) is
    None where it cannot be built."""
    d = os.path.join(ROOT, "oracle")
    _ensure_built(d, ["libsg_oracle.so", "libsg_oracle_twin.so", "libsg_oracle_twin_cr.so"])
    crq = os.path.join(d, "libsg_oracle_crq.so")
    if not os.path.exists(crq):
        subprocess.run(["make", "-C", d, "crq"], capture_output=True)
    return {"libm": os.path.join(d, "libsg_oracle.so"), "twin": os.path.join(d, "libsg_oracle_twin.so"),
            "twin_cr": os.path.join(d, "libsg_oracle_twin_cr.so"), "crq": crq if os.path.exists(crq) else None}


@pytest.fixture(scope="session")
def sg():
    import sogrand_b200

    return sogrand_b200


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture
def cr_mode(sg):
    """The decoder's reference-exact math mode (correctly rounded exp/log)
    for one test."""
    old = sg.get_math_mode()
    sg.set_math_mode(1)
    yield
    sg.set_math_mode(old)
