"""The C FP64 adjoint (oracle) against central finite differences of the
forward loss, on the branch of the forward pass."""
import numpy as np
import pytest

from oracle_api import adjoint, forward_loss


@pytest.mark.timeout(600)
def test_c_adjoint_matches_finite_differences(sg, oracle_paths):
    info, llr = sg.gen_llr(31337, 0, 1, ebn0_db=1.5)
    bits = sg.encode(info)[0]
    imax = 3
    alpha = np.full(150, 0.7)
    loss, ga, gl = adjoint(oracle_paths["twin"], llr[0], bits, Imax=imax, alpha=alpha)
    assert np.isfinite(loss) and loss > 0
    assert np.abs(ga).max() > 0
    h = 1e-6
    checked = 0
    for ph in range(3 * imax):
        if ga[ph] == 0:
            continue
        up, dn = alpha.copy(), alpha.copy()
        up[ph] += h
        dn[ph] -= h
        fd = (forward_loss(oracle_paths["twin"], llr[0], bits, Imax=imax, alpha=up)
              - forward_loss(oracle_paths["twin"], llr[0], bits, Imax=imax, alpha=dn)) / (2 * h)
        assert abs(fd - ga[ph]) <= 1e-4 * max(1.0, abs(ga[ph])), (ph, fd, ga[ph])
        checked += 1
    assert checked >= 3
    # channel-LLR gradient at a few positions
    rng = np.random.default_rng(0)
    for q in rng.choice(4096, 4, replace=False):
        up, dn = llr[0].copy(), llr[0].copy()
        up[q] += h
        dn[q] -= h
        fd = (forward_loss(oracle_paths["twin"], up, bits, Imax=imax, alpha=alpha)
              - forward_loss(oracle_paths["twin"], dn, bits, Imax=imax, alpha=alpha)) / (2 * h)
        assert abs(fd - gl[q]) <= 1e-4 * max(1.0, abs(gl[q])), (q, fd, gl[q])


@pytest.mark.timeout(600)
def test_c_adjoint_phase_loss_matches_finite_differences(sg, oracle_paths):
    """The BCE summed over every phase's APP (loss_mode 1): its loss, as the
    adjoint reports it, differenced in alpha."""
    info, llr = sg.gen_llr(31338, 0, 1, ebn0_db=1.5)
    bits = sg.encode(info)[0]
    imax = 3
    alpha = np.full(150, 0.7)
    loss, ga, _ = adjoint(oracle_paths["twin"], llr[0], bits, loss_mode=1, Imax=imax, alpha=alpha)
    final, _, _ = adjoint(oracle_paths["twin"], llr[0], bits, loss_mode=0, Imax=imax, alpha=alpha)
    assert loss > final > 0
    h = 1e-6
    checked = 0
    for ph in range(3 * imax):
        if ga[ph] == 0:
            continue
        up, dn = alpha.copy(), alpha.copy()
        up[ph] += h
        dn[ph] -= h
        lu = adjoint(oracle_paths["twin"], llr[0], bits, loss_mode=1, Imax=imax, alpha=up)[0]
        ld = adjoint(oracle_paths["twin"], llr[0], bits, loss_mode=1, Imax=imax, alpha=dn)[0]
        fd = (lu - ld) / (2 * h)
        assert abs(fd - ga[ph]) <= 1e-4 * max(1.0, abs(ga[ph])), (ph, fd, ga[ph])
        checked += 1
    assert checked >= 3
