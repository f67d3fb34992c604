"""Sharding over several processes (one per GPU in production), checked with
world_size 2 gloo process groups on the CPU: each rank steps its substrate
block of a microenvironment (the oracle stands in for the GPU kernels: the
test is about the host logic), and the all-gathered field equals the
unsharded run bit for bit, since no statement of the step mixes
substrates."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from biofvm_b200 import sharding as SH
from biofvm_b200 import workloads as W


def test_substrate_ranges_cover_every_substrate_once():
    for S in range(0, 12):
        for world in range(1, 6):
            blocks = [SH.substrate_range(S, world, r) for r in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == S
            assert all(a[1] == b[0] for a, b in zip(blocks, blocks[1:]))
            sizes = [b - a for a, b in blocks]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        SH.substrate_range(4, 2, 2)


def test_instance_assignment_is_balanced_and_deterministic():
    rng = np.random.default_rng(1)
    sizes = rng.integers(32 ** 3, 128 ** 3, 64) * rng.integers(1, 9, 64)
    for world in (1, 2, 4, 8):
        owner = SH.assign_instances(sizes, world)
        assert owner == SH.assign_instances(list(sizes), world)
        load = np.bincount(owner, weights=sizes, minlength=world)
        assert load.max() - load.min() <= sizes.max()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist

    from oracle import oracle as O

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        scn = W.mixed_small(shape=(9, 7, 6), S=5, n_agents=80, seed=33)
        sub = SH.shard_by_substrate(scn, world, rank)
        local = O.oracle_run(sub, 3, 7) if sub.S else np.zeros((scn.num_voxels, 0))
        full = SH.gather_substrates(local, scn.S)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), full)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_substrate_shards_gather_to_the_unsharded_field(tmp_path, world):
    from oracle import oracle as O

    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    scn = W.mixed_small(shape=(9, 7, 6), S=5, n_agents=80, seed=33)
    ref = O.oracle_run(scn, 3, 7)
    for r in range(world):
        assert np.array_equal(np.load(tmp_path / f"rank{r}.npy"), ref)
