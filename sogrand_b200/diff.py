"""Differentiable decoding: torch.autograd.Function over the C ABI pair
sg_forward_device / sg_backward_device, and learning of the per-phase
extrinsic weights.

The reference scales the extrinsic information with one constant, alpha =
0.7 for every phase (SOGRAND_C/cubic_decoder_final.c:100-102).  Here the
3*Imax per-phase weights are trainable: the loss is the BCE of the final
APP against the transmitted code bits,
    loss = mean over codewords of sum_i softplus(s_i L_APP_i),  s_i = 2 c_i - 1,
or that BCE summed over the APP of every phase run (loss="phases"),
differentiated exactly on the branch of the forward pass (sorts, tested
patterns, lists, stops, early terminations held fixed).  The plain decoder
with the learned weights is then evaluated by BER.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


def _params(alpha_np, imax: int, L: int):
    import sogrand_b200 as sg

    a = np.full(sg.SG_MAX_PHASES, 0.7)
    a[: 3 * imax] = alpha_np[: 3 * imax]
    return sg.params(L=L, Imax=imax, alpha=a)


def _check_cube(llr, name="llr"):
    """The C ABI reads llr as contiguous float64 [n, 4096] device memory."""
    import torch

    if not (llr.is_cuda and llr.dtype == torch.float64 and llr.is_contiguous() and llr.dim() == 2
            and llr.shape[1] == 4096):
        raise ValueError(f"{name} must be a contiguous CUDA float64 tensor of shape [n, 4096]")


def _check_bits(code_bits, n):
    import torch

    if not (code_bits.is_cuda and code_bits.dtype == torch.uint8 and code_bits.is_contiguous()
            and tuple(code_bits.shape) == (n, 4096)):
        raise ValueError("code_bits must be a contiguous CUDA uint8 tensor of shape [n, 4096]")


def _torch_fn():
    import torch

    class DecodeBCE(torch.autograd.Function):
        @staticmethod
        def forward(ctx, alpha, llr, code_bits, imax: int, L: int, loss_mode: int):
            import sogrand_b200 as sg

            lib = _lib.load()
            _check_cube(llr)
            n = llr.shape[0]
            _check_bits(code_bits, n)
            nph = 3 * imax
            dev = llr.device
            p = _params(alpha.detach().cpu().numpy(), imax, L)
            ckpt = torch.empty((n, nph, sg.SG_CUBE), dtype=torch.float64, device=dev)
            bits = torch.empty((n, sg.SG_INFO_BYTES), dtype=torch.uint8, device=dev)
            stats = torch.empty((n, sg.STATS_DTYPE.itemsize), dtype=torch.uint8, device=dev)
            lapp = torch.empty((n, sg.SG_CUBE), dtype=torch.float64, device=dev)
            s = torch.cuda.current_stream(dev).cuda_stream
            _lib.check(lib.sg_forward_device(llr.data_ptr(), n, C.byref(p), bits.data_ptr(), lapp.data_ptr(),
                                             stats.data_ptr(), ckpt.data_ptr(), s))
            ctx.imax, ctx.want_llr, ctx.bits = imax, llr.requires_grad, bits
            if loss_mode == 0:
                sgn = code_bits.to(torch.float64) * 2.0 - 1.0
                loss = torch.nn.functional.softplus(sgn * lapp).sum(dim=1).mean()
                ctx.save_for_backward(llr, code_bits, ckpt, stats)
                ctx.p, ctx.grads = p, None
                return loss
            # every phase's APP: only the backward pass sees the phases, so
            # it runs now and the gradients are kept for backward()
            lossv, ga, gl = backward_raw(llr, code_bits, p, stats, ckpt, want_llr=llr.requires_grad, loss_mode=1)
            ctx.grads = (ga.sum(dim=0) / n, gl / n if gl is not None else None)
            return lossv.mean()

        @staticmethod
        def backward(ctx, g):
            if ctx.grads is not None:
                ga, gl = ctx.grads
                return g * ga, (g * gl if gl is not None else None), None, None, None, None
            llr, code_bits, ckpt, stats = ctx.saved_tensors
            n = llr.shape[0]
            _, ga, gl = backward_raw(llr, code_bits, ctx.p, stats, ckpt, want_llr=ctx.want_llr)
            grad_alpha = g * ga.sum(dim=0) / n
            grad_llr = g * gl / n if gl is not None else None
            return grad_alpha, grad_llr, None, None, None, None

    return DecodeBCE


_FN = None


def decode_bce(alpha, llr, code_bits, imax: int = 30, L: int = 3, loss: str = "final"):
    """Mean BCE over codewords, differentiable in alpha (float64 tensor of
    3*imax weights) and in llr (CUDA [n, 4096] float64).  code_bits: CUDA
    uint8 [n, 4096] transmitted bits.  loss: "final" -- the BCE of the final
    APP; "phases" -- the BCE of every phase's APP, summed."""
    global _FN
    if loss not in ("final", "phases"):
        raise ValueError("loss must be 'final' or 'phases'")
    if _FN is None:
        _FN = _torch_fn()
    # contiguous() keeps the autograd path to a non-contiguous llr
    return _FN.apply(alpha, llr.contiguous(), code_bits.contiguous(), imax, L, 0 if loss == "final" else 1)


def backward_raw(llr, code_bits, p, stats, ckpt, want_llr: bool = False, loss_mode: int = 0):
    """Per-codeword loss and gradients from sg_backward_device (CUDA tensors);
    loss_mode 0: BCE of the final APP, 1: summed over every phase's APP."""
    import torch

    import sogrand_b200 as sg

    _check_cube(llr)
    n = llr.shape[0]
    _check_bits(code_bits, n)
    nph = 3 * p.Imax
    dev = llr.device
    loss = torch.empty(n, dtype=torch.float64, device=dev)
    ga = torch.empty((n, nph), dtype=torch.float64, device=dev)
    gl = torch.empty((n, sg.SG_CUBE), dtype=torch.float64, device=dev) if want_llr else None
    _lib.check(_lib.load().sg_backward_device(llr.data_ptr(), n, C.byref(p), stats.data_ptr(), ckpt.data_ptr(),
                                              code_bits.data_ptr(), int(loss_mode), loss.data_ptr(), ga.data_ptr(),
                                              gl.data_ptr() if gl is not None else None,
                                              torch.cuda.current_stream(dev).cuda_stream))
    return loss, ga, gl


def forward_raw(llr, p):
    """sg_forward_device: (bits, raw stats, lapp, checkpoints)."""
    import torch

    import sogrand_b200 as sg

    _check_cube(llr)
    n = llr.shape[0]
    dev = llr.device
    ckpt = torch.empty((n, 3 * p.Imax, sg.SG_CUBE), dtype=torch.float64, device=dev)
    bits = torch.empty((n, sg.SG_INFO_BYTES), dtype=torch.uint8, device=dev)
    stats = torch.empty((n, sg.STATS_DTYPE.itemsize), dtype=torch.uint8, device=dev)
    lapp = torch.empty((n, sg.SG_CUBE), dtype=torch.float64, device=dev)
    _lib.check(_lib.load().sg_forward_device(llr.data_ptr(), n, C.byref(p), bits.data_ptr(), lapp.data_ptr(),
                                             stats.data_ptr(), ckpt.data_ptr(),
                                             torch.cuda.current_stream(dev).cuda_stream))
    return bits, stats, lapp, ckpt


def code_bits_for(info, device):
    """Transmitted code bits [n, 4096] (uint8, CUDA) of packed info blocks."""
    import torch

    import sogrand_b200 as sg

    info_np = info.cpu().numpy() if hasattr(info, "cpu") else np.asarray(info)
    return torch.from_numpy(sg.encode(info_np)).to(device)


def train_weights(steps: int = 60, batch: int = 4096, ebn0_db: float = 1.5, imax: int = 30, lr: float = 0.02,
                  seed: int = 90210, device: str = "cuda", init: float = 0.7, log=None, val_cw: int = 0,
                  val_every: int = 10, loss: str = "final"):
    """Adam on the 3*imax extrinsic weights over fresh seeded batches (each
    step a new range of the codeword stream).  With val_cw > 0 the mean BCE
    on a fixed validation batch (its own seed) is evaluated every val_every
    steps and the best weights seen are returned.  Returns (weights, history)
    where history holds the training losses and the validation points."""
    import torch

    import sogrand_b200 as sg

    alpha = torch.full((3 * imax,), init, dtype=torch.float64, device=device, requires_grad=True)
    opt = torch.optim.Adam([alpha], lr=lr)
    hist = {"train": [], "val": []}
    best = (float("inf"), alpha.detach().cpu().numpy().copy())
    if val_cw:
        vinfo, vllr = sg.gen_llr(seed + 7919, 0, val_cw, ebn0_db=ebn0_db, device=device)
        vcb = code_bits_for(vinfo, device)

    def validate(step):
        nonlocal best
        with torch.no_grad():
            v = float(decode_bce(alpha.detach(), vllr, vcb, imax, loss=loss).item())
        hist["val"].append((step, v))
        if v < best[0]:
            best = (v, alpha.detach().cpu().numpy().copy())
        if log:
            log(step, float("nan"), v)

    if val_cw:
        validate(0)
    for step in range(steps):
        info, llr = sg.gen_llr(seed, step * batch, batch, ebn0_db=ebn0_db, device=device)
        cb = code_bits_for(info, device)
        opt.zero_grad()
        lv = decode_bce(alpha, llr, cb, imax, loss=loss)
        lv.backward()
        opt.step()
        with torch.no_grad():
            alpha.clamp_(0.0, 2.0)
        hist["train"].append(float(lv.item()))
        if log:
            log(step, hist["train"][-1], None)
        if val_cw and (step + 1) % val_every == 0:
            validate(step + 1)
    if val_cw:
        return best[1], hist
    return alpha.detach().cpu().numpy(), hist
