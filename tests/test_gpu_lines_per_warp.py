"""The two-lines-per-warp kernel configurations (16 lanes per line,
sg_line16.cuh) give exactly the results of the 32-lane line decoder: on the
cases that take the decoder's rarer paths (Tmax cuts, list sizes, tied
magnitudes and the exact quicksort, lines that search deep into the order
tables, checkpoints of the differentiable forward) and, in the
reference-exact math mode, against the reference's own fixtures."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DEFAULT = "w16-gmem-g2"


def _l2_variants():
    from sogrand_b200 import autotune

    names = [n for n in autotune.variants() if "-l2-" in n]
    assert len(names) >= 3
    return names


def _decode(sg, torch, name, dllr, p):
    from sogrand_b200 import autotune

    autotune.set_variant(name)
    db, draw, dl = sg.decode(dllr, p, want_lapp=True)
    torch.cuda.synchronize()
    return db.cpu().numpy(), draw.cpu().numpy(), dl.cpu().numpy()


def _cases(sg):
    """(label, cubes, params) for the rarer paths of the line decoder."""
    _, noisy = sg.gen_llr(4711, 0, 48, ebn0_db=1.25)
    info = sg.gen_info(4712, 0, 24)
    code = sg.encode(info).astype(np.float64)
    rng = np.random.default_rng(4713)
    # magnitudes on a coarse grid: most lines hold tied reliabilities
    tied = np.round(np.abs(rng.normal(1.0, 0.8, code.shape)) * 2.0) / 2.0 + 0.5
    tied = (1.0 - 2.0 * code) * tied
    flip = rng.random(code.shape) < 0.06
    tied[flip] = -tied[flip]
    # large magnitudes of several spreads with flipped signs: high IC, deep searches
    mag = rng.uniform(12.0, 30.0, (24, 1)) + rng.uniform(0.0, 1.0, code.shape) * np.repeat([2.0, 6.0, 12.0, 24.0], 6)[:, None]
    deep = (1.0 - 2.0 * code) * mag
    flip = rng.random(code.shape) < 0.01
    deep[flip] = -deep[flip]
    return [
        ("1.25 dB", noisy, sg.params()),
        ("Tmax 10", noisy, sg.params(Tmax=10)),
        ("Tmax 100", noisy, sg.params(Tmax=100)),
        ("Tmax 1000", noisy, sg.params(Tmax=1000)),
        ("L 1", noisy, sg.params(L=1)),
        ("L 4", noisy, sg.params(L=4)),
        ("tied magnitudes", np.ascontiguousarray(tied), sg.params()),
        ("high IC", np.ascontiguousarray(deep), sg.params()),
    ]


def test_l2_variants_equal_32_lane_decoder(cuda, sg):
    from sogrand_b200 import autotune

    torch = cuda
    before = autotune.get_variant()
    try:
        for label, llr, p in _cases(sg):
            dllr = torch.from_numpy(llr).cuda()
            want = _decode(sg, torch, DEFAULT, dllr, p)
            for name in _l2_variants():
                got = _decode(sg, torch, name, dllr, p)
                assert np.array_equal(got[0], want[0]), (label, name, "bits")
                assert np.array_equal(got[1], want[1]), (label, name, "statistics")
                assert np.array_equal(got[2].view(np.int64), want[2].view(np.int64)), (label, name, "L_APP")
    finally:
        autotune.set_variant(before)


def test_l2_variants_forward_checkpoints(cuda, sg):
    """The differentiable forward (sg_forward_device) runs the selected
    configuration: the same outputs and the same checkpoints of L_E entering
    every phase a codeword ran (later phases are never written)."""
    from sogrand_b200 import autotune, diff

    torch = cuda
    _, llr = sg.gen_llr(4714, 0, 16, ebn0_db=1.5, device="cuda")
    p = sg.params(Imax=10)
    before = autotune.get_variant()
    try:
        autotune.set_variant(DEFAULT)
        want = diff.forward_raw(llr, p)
        torch.cuda.synchronize()
        phases = sg.stats_from_device(want[1])["phases"]
        assert phases.min() >= 1
        for name in _l2_variants():
            autotune.set_variant(name)
            got = diff.forward_raw(llr, p)
            torch.cuda.synchronize()
            for a, b in zip(got[:3], want[:3]):
                assert torch.equal(a, b), name
            for i, n_ph in enumerate(phases):
                assert torch.equal(got[3][i, :n_ph], want[3][i, :n_ph]), (name, i)
    finally:
        autotune.set_variant(before)


@pytest.mark.parametrize("name", ["cfg1_2dB_100", "snr_1.5dB"])
def test_l2_variants_reference_exact_mode(cuda, sg, golden, cr_mode, name):
    """Math mode 1: every defined codeword equals the reference under a
    correctly rounded libm (bits, iterations, NG, NG_p, convergence)."""
    from sogrand_b200 import autotune

    torch = cuda
    e = golden["sets"][name]
    _, llr = sg.gen_llr(e["seed"], 0, e["n_cw"], ebn0_db=e["ebn0_db"])
    want = e["ref_cr"]
    dllr = torch.from_numpy(llr).cuda()
    before = autotune.get_variant()
    try:
        for v in _l2_variants():
            bits, raw, _ = _decode(sg, torch, v, dllr, sg.params(Tmax=e["Tmax"]))
            st = sg.stats_from_device(torch.from_numpy(raw))
            for i in range(e["n_cw"]):
                if want["undefined_lines"][i]:
                    continue
                got = (bits[i].tobytes().hex(), float(st["iterations"][i]), int(st["ng"][i]), int(st["ng_p"][i]),
                       int(st["converged"][i]))
                assert got == (want["bits"][i], want["iterations"][i], want["ng"][i], want["ng_p"][i],
                               want["converged"][i]), (v, i)
    finally:
        autotune.set_variant(before)
