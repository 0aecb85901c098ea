"""Multi-GPU form of the decoder: independent replicas.

Codewords are independent and the decode has no exchange step, so N GPUs
decode N disjoint ranges of one seeded codeword stream, one process per GPU,
with no collective on the data path.  Only the per-rank totals (and the max
time over ranks) are combined at the end.
"""
from __future__ import annotations


def codeword_range(rank: int, world: int, n_total: int | None = None, n_per_rank: int | None = None):
    """[first, last) codeword of this rank: either a fixed count per rank
    (weak scaling) or an even split of n_total (strong scaling)."""
    if (n_total is None) == (n_per_rank is None):
        raise ValueError("give exactly one of n_total and n_per_rank")
    if n_per_rank is not None:
        return rank * n_per_rank, (rank + 1) * n_per_rank
    base, extra = divmod(n_total, world)
    first = rank * base + min(rank, extra)
    return first, first + base + (1 if rank < extra else 0)


SUM_KEYS = ("blocks", "converged", "nonfinite", "total_ng", "total_ng_p", "bits_compared", "bit_errors",
            "block_errors")


def combine_summaries(summary: dict, device=None) -> dict:
    """Sum a decode summary over all ranks of the default process group
    (integer totals exactly; the iteration total is a multiple of 0.5)."""
    import torch
    import torch.distributed as dist

    ints = torch.tensor([int(summary[k]) for k in SUM_KEYS], dtype=torch.int64, device=device)
    it = torch.tensor([float(summary["total_iterations"])], dtype=torch.float64, device=device)
    dist.all_reduce(ints)
    dist.all_reduce(it)
    out = {k: int(v) for k, v in zip(SUM_KEYS, ints.tolist())}
    out["total_iterations"] = float(it.item())
    return out


def max_over_ranks(seconds: float, device=None) -> float:
    import torch
    import torch.distributed as dist

    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
