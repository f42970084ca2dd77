"""Multi-process sharding on CPU (gloo, world size 2).

Particles are independent; each rank integrates its shard with its global
particle ids (so it draws the same Philox stream as a single process would) and
the ranks combine the moment-weighted window sums and the weights with one
all_reduce — the only exchange the path has.  The combined ensemble mean must
equal the single-process mean.
"""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _rank_main(rank, world, port, out_path):
    import torch

    import oracle
    from stochasticphysics_b200 import provider

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    spec = provider.brown_neel_relaxation(n=96, steps=1100, oversampling=100)
    lo, hi = rank * spec.n // world, (rank + 1) * spec.n // world
    part = oracle.simulate(spec.subset(lo, hi), threads=1)
    wsum = torch.from_numpy(part["mean"] * part["weight"])  # weighted window sums of the shard
    w = torch.from_numpy(part["weight"].copy())
    dist.all_reduce(wsum)
    dist.all_reduce(w)
    if rank == 0:
        np.save(out_path, (wsum / w).numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_reproduce_the_single_process_mean(tmp_path):
    import oracle
    from stochasticphysics_b200 import provider

    out = tmp_path / "mean.npy"
    port = 29500 + (os.getpid() % 2000)
    mp.start_processes(_rank_main, args=(2, port, str(out)), nprocs=2, start_method="spawn", join=True)
    combined = np.load(out)
    spec = provider.brown_neel_relaxation(n=96, steps=1100, oversampling=100)
    full = oracle.simulate(spec)["mean"]
    np.testing.assert_allclose(combined, full, rtol=1e-12, atol=1e-14)
