"""GPU adjoint (sg_forward_device / sg_backward_device): against the C FP64
adjoint of the oracle and against central finite differences."""
import multiprocessing as mp

import numpy as np
import pytest

from oracle_api import adjoint

pytestmark = pytest.mark.gpu


def _c_adjoint(args):
    path, llr, bits, imax, mode = args
    return adjoint(path, llr, bits, loss_mode=mode, Imax=imax)


@pytest.mark.parametrize("imax,mode", [(3, 0), (30, 0), (3, 1), (30, 1)])
def test_gpu_adjoint_matches_c_adjoint(cuda, sg, oracle_paths, imax, mode):
    """Loss and gradients of the final APP's BCE (mode 0) and of the BCE
    summed over every phase's APP (mode 1)."""
    torch = cuda
    from sogrand_b200 import diff

    info, llr = sg.gen_llr(4242, 0, 4, ebn0_db=1.5)
    bits = sg.encode(info)
    p = sg.params(Imax=imax)
    d = torch.from_numpy(llr).cuda()
    db = torch.from_numpy(bits).cuda()
    _, stats, lapp, ckpt = diff.forward_raw(d, p)
    loss, ga, gl = diff.backward_raw(d, db, p, stats, ckpt, want_llr=True, loss_mode=mode)
    torch.cuda.synchronize()
    with mp.get_context("spawn").Pool(4) as pool:
        ref = pool.map(_c_adjoint, [(oracle_paths["twin"], llr[i], bits[i], imax, mode) for i in range(4)])
    for i, (cl, cga, cgl) in enumerate(ref):
        assert abs(loss[i].item() - cl) <= 1e-12 * abs(cl)
        g = ga[i].cpu().numpy()
        assert np.abs(g - cga).max() <= 1e-9 * max(1.0, np.abs(cga).max()), (i, np.abs(g - cga).max())
        h = gl[i].cpu().numpy()
        assert np.abs(h - cgl).max() <= 1e-9 * max(1.0, np.abs(cgl).max())
    # the decoded L_APP of the forward equals the plain decoder's
    _, _, lp = sg.decode(d, p, want_lapp=True)
    assert torch.equal(lp, lapp)


def test_gpu_adjoint_finite_differences_64_codewords(cuda, sg):
    """d loss / d alpha on 64 codewords at 1.5 dB vs central differences with
    step 1e-6, per codeword.  The loss is piecewise smooth: a (codeword,
    phase) pair whose branch flips between alpha - h and alpha + h (its
    guess count or phase count changes) is counted and excluded; on the rest
    the adjoint must match."""
    torch = cuda
    from sogrand_b200 import diff

    imax = 30
    info, llr = sg.gen_llr(2718, 0, 64, ebn0_db=1.5, device="cuda")
    cb = diff.code_bits_for(info, "cuda")
    sgn = cb.to(torch.float64) * 2 - 1
    base = np.full(150, 0.7)

    def run(a):
        p = sg.params(Imax=imax, alpha=a)
        _, st, lapp, ck = diff.forward_raw(llr, p)
        loss = torch.nn.functional.softplus(sgn * lapp).sum(dim=1)
        return p, st, ck, loss.cpu().numpy(), sg.stats_from_device(st)

    p0, st0, ck0, loss0, s0 = run(base)
    closs, ga, _ = diff.backward_raw(llr, cb, p0, st0, ck0)
    assert np.allclose(closs.cpu().numpy(), loss0, rtol=1e-12)
    ga = ga.cpu().numpy()
    h = 1e-6
    rel, flipped, pairs = [], 0, 0
    for ph in range(1, 3 * imax):
        if not ga[:, ph].any():
            continue
        up, dn = base.copy(), base.copy()
        up[ph] += h
        dn[ph] -= h
        _, _, _, lu, su = run(up)
        _, _, _, ld, sd = run(dn)
        same = (su["ng"] == sd["ng"]) & (su["phases"] == sd["phases"]) & (su["ng"] == s0["ng"])
        flipped += int((~same & (ga[:, ph] != 0)).sum())
        pairs += int((ga[:, ph] != 0).sum())
        fd = ((lu - ld) / (2 * h))[same].sum()
        ad = ga[same, ph].sum()
        if ad != 0:
            rel.append(abs(fd - ad) / abs(ad))
    rel = np.array(rel)
    print(f"FD check on 64 codewords: {len(rel)} phases, {flipped}/{pairs} (codeword, phase) pairs flipped; "
          f"unflipped rel err median {np.median(rel):.2e}, 90th pct {np.percentile(rel, 90):.2e}, "
          f"max {rel.max():.2e}")
    assert len(rel) >= 10
    assert np.median(rel) < 1e-6
    assert rel.max() < 1e-3
    assert flipped <= 0.05 * pairs
