"""Replica sharding over 2 ranks (gloo, CPU): disjoint codeword ranges that
tile the stream, and totals combined across ranks equal one process's."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def test_ranges_tile_the_stream():
    from sogrand_b200.replicas import codeword_range

    for n, w in [(10, 3), (100000, 8), (7, 7), (3, 4)]:
        rs = [codeword_range(r, w, n_total=n) for r in range(w)]
        assert rs[0][0] == 0 and rs[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
        assert max(b - a for a, b in rs) - min(b - a for a, b in rs) <= 1
    assert codeword_range(3, 8, n_per_rank=100) == (300, 400)


def _worker(rank, world, port, out):
    import sys

    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch.distributed as dist

    import sogrand_b200 as sg
    from oracle_api import Oracle
    from sogrand_b200.replicas import codeword_range, combine_summaries, max_over_ranks

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    a, b = codeword_range(rank, world, n_total=3)
    info, llr = sg.gen_llr(11, a, b - a, ebn0_db=3.0)
    bits, stats, _ = Oracle(os.path.join(ROOT, "oracle", "libsg_oracle_twin.so")).decode(llr)
    errs = np.unpackbits(bits, axis=1) != np.unpackbits(info, axis=1)
    local = {"blocks": b - a, "converged": sum(s[3] == 1 for s in stats), "nonfinite": 0,
             "total_ng": sum(s[1] for s in stats), "total_ng_p": sum(s[2] for s in stats),
             "bits_compared": 512 * (b - a), "bit_errors": int(errs.sum()),
             "block_errors": int(errs.any(axis=1).sum()), "total_iterations": sum(s[0] for s in stats)}
    tot = combine_summaries(local)
    t = max_over_ranks(float(rank + 1))
    if rank == 0:
        out.put((tot, t))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_rank_totals_equal_single_process(oracle_paths):
    import random

    from oracle_api import Oracle
    import sogrand_b200 as sg

    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = 29500 + random.randint(0, 2000)
    mp.start_processes(_worker, args=(2, port, q), nprocs=2, join=True, start_method="spawn")
    tot, tmax = q.get()
    info, llr = sg.gen_llr(11, 0, 3, ebn0_db=3.0)
    bits, stats, _ = Oracle(oracle_paths["twin"]).decode(llr)
    assert tmax == 2.0
    assert tot["blocks"] == 3
    assert tot["total_ng"] == sum(s[1] for s in stats)
    assert tot["total_iterations"] == sum(s[0] for s in stats)
    assert tot["bit_errors"] == int((np.unpackbits(bits, axis=1) != np.unpackbits(info, axis=1)).sum())
