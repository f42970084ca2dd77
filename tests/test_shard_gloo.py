"""Multi-process sharding on CPU (gloo, world size 2) through the library's merge.

Particles are independent; each rank integrates its shard with its global
particle ids (so it draws the same Philox stream as a single process would).
The ranks exchange each shard's moment-weighted window sums and weights (one
all_gather: the only exchange the path has) and every rank folds them with the
library's host-side merge, sp_merge_shards, which restates
MeanSimulationResult::operator+= and normalize
(Particle_Simulation/Results/MeanSimulationResult.h:63-119).  The merged
ensemble mean must equal the single-process mean.  The shards' own results come
from the oracle here (no GPU on this machine); the GPU test of the same merge
feeds it the library's shard results.
"""
import os

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp


def _rank_main(rank, world, port, out_path):
    import torch

    import oracle
    from stochasticphysics_b200 import merge_shards, provider

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        spec = provider.brown_neel_relaxation(n=96, steps=1100, oversampling=100)
        lo, hi = rank * spec.n // world, (rank + 1) * spec.n // world
        part = oracle.simulate(spec.subset(lo, hi), threads=1)
        # the shard's un-normalised sums, as sp_result.weighted_sum returns them
        mine = torch.from_numpy(np.concatenate([(part["mean"] * part["weight"]).ravel(), part["weight"]]))
        parts = [torch.empty_like(mine) for _ in range(world)]
        dist.all_gather(parts, mine)
        k, od = part["mean"].shape
        sums = [p[:k * od].numpy().reshape(k, od) for p in parts]
        weights = [p[k * od:].numpy() for p in parts]
        mean, total, weight = merge_shards(sums, weights)
        np.save(f"{out_path}.{rank}.npy", np.concatenate([mean.ravel(), weight]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_merge_to_the_single_process_mean(tmp_path):
    import oracle
    from stochasticphysics_b200 import provider

    out = tmp_path / "merged"
    port = 29500 + (os.getpid() % 2000)
    mp.start_processes(_rank_main, args=(2, port, str(out)), nprocs=2, start_method="spawn", join=True)
    spec = provider.brown_neel_relaxation(n=96, steps=1100, oversampling=100)
    full = oracle.simulate(spec)
    k, od = full["mean"].shape
    r0, r1 = np.load(f"{out}.0.npy"), np.load(f"{out}.1.npy")
    np.testing.assert_array_equal(r0, r1)  # every rank folds the shards in the same order
    np.testing.assert_allclose(r0[:k * od].reshape(k, od), full["mean"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(r0[k * od:], full["weight"], rtol=1e-13)
