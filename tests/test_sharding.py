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


# ---- the product path: every rank a Solver on the GPU ----

def _shard_main(rank, world, port, backend, out_dir):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group(backend, rank=rank, world_size=world)
    try:
        scn = W.mixed_small(shape=(19, 14, 11), S=5, n_agents=300, seed=35)
        shard = SH.SubstrateShard(scn, device=0)
        shard.step(scn.dt, 3)
        dev = shard.gather_device()
        np.save(os.path.join(out_dir, f"oncuda{rank}.npy"), np.array([int(dev.is_cuda)]))
        full = dev.cpu().numpy()
        blk = shard.device_block().cpu().numpy()
        shard.close()
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), full)
        np.save(os.path.join(out_dir, f"block{rank}.npy"), blk)
    finally:
        dist.destroy_process_group()


def _run_ranks(target, world, args):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, *args)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0


@pytest.mark.gpu
@pytest.mark.parametrize("world", [2, 3, 6], ids=["2", "3", "6-one-rank-empty"])
def test_solver_shards_on_the_gpu_gather_to_the_oracle(tmp_path, world):
    """Each rank (processes sharing the one GPU here; the collective runs over
    gloo) steps its substrate block with a product Solver; the gathered field
    matches the unsharded oracle run within the FP64 bar, and every rank's
    block is its columns of it.  With 6 ranks and 5 substrates one rank holds
    none and still takes part in the all-gather."""
    from oracle import oracle as O

    _run_ranks(_shard_main, world, ("gloo", str(tmp_path)))
    scn = W.mixed_small(shape=(19, 14, 11), S=5, n_agents=300, seed=35)
    ref = O.oracle_run(scn, 3, 7)
    for r in range(world):
        full = np.load(tmp_path / f"rank{r}.npy")
        assert np.all(O.max_rel_err(full, ref) <= 1e-12)
        a, b = SH.substrate_range(scn.S, world, r)
        assert np.array_equal(np.load(tmp_path / f"block{r}.npy"), full[:, a:b])


@pytest.mark.gpu
def test_device_gather_over_nccl_stays_on_the_device(tmp_path):
    """One rank over NCCL (the process group of one GPU): gather_device
    returns a CUDA tensor equal to the oracle's field."""
    from oracle import oracle as O

    _run_ranks(_shard_main, 1, ("nccl", str(tmp_path)))
    scn = W.mixed_small(shape=(19, 14, 11), S=5, n_agents=300, seed=35)
    ref = O.oracle_run(scn, 3, 7)
    assert np.load(tmp_path / "oncuda0.npy")[0] == 1
    assert np.all(O.max_rel_err(np.load(tmp_path / "rank0.npy"), ref) <= 1e-12)


def test_z_bounds_cover_every_plane_once():
    for nz in range(1, 20):
        for world in range(1, nz + 1):
            b = SH.z_bounds(nz, world)
            assert b[0] == 0 and b[-1] == nz and len(b) == world + 1
            assert all(y > x for x, y in zip(b, b[1:]))
    with pytest.raises(ValueError):
        SH.z_bounds(3, 4)


def _zslab_main(rank, world, port, backend, shape, out_dir):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group(backend, rank=rank, world_size=world)
    try:
        scn = W.mixed_small(shape=shape, S=3, n_agents=400, seed=37)
        shard = SH.ZSlabShard(scn, device=0)
        shard.step(scn.dt, 4)
        full = shard.gather()
        shard.close()
        np.save(os.path.join(out_dir, f"z{rank}.npy"), full)
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("world,shape", [(2, (13, 11, 17)), (3, (13, 11, 17)),
                                         (4, (9, 8, 5)), (2, (40, 36, 300))],
                         ids=["2", "3", "4-thin-slabs", "2-long-z"])
def test_z_slabs_join_to_the_unsplit_solve(tmp_path, world, shape):
    """One field split by z planes over ranks (processes sharing the one GPU
    here; the plane exchange runs over gloo): after 4 steps with bulk,
    agents and Dirichlet nodes, every rank's gathered field matches the
    unsplit oracle run within the FP64 bar."""
    from oracle import oracle as O

    _run_ranks(_zslab_main, world, ("gloo", shape, str(tmp_path)))
    scn = W.mixed_small(shape=shape, S=3, n_agents=400, seed=37)
    ref = O.oracle_run(scn, 4, 7)
    for r in range(world):
        got = np.load(tmp_path / f"z{r}.npy")
        assert np.all(O.max_rel_err(got, ref) <= 1e-12), O.max_rel_err(got, ref)


@pytest.mark.gpu
def test_z_slab_of_one_rank_over_nccl(tmp_path):
    """The NCCL path with one rank (the whole field is one slab)."""
    from oracle import oracle as O

    _run_ranks(_zslab_main, 1, ("nccl", (13, 11, 17), str(tmp_path)))
    scn = W.mixed_small(shape=(13, 11, 17), S=3, n_agents=400, seed=37)
    assert np.all(O.max_rel_err(np.load(tmp_path / "z0.npy"), O.oracle_run(scn, 4, 7)) <= 1e-12)


@pytest.mark.parametrize("bounds", [[0, 5, 6, 11, 17], [0, 17], [0, 1, 2, 3, 17], [0, 9, 17]])
def test_z_slab_join_algebra(bounds):
    """The join of bfvm_zslab_fixup restated in numpy on one z line: every
    slab solves its segment with the whole line's Thomas rows and zero
    carries at its ends (x'); the carries folded from the slabs' first and
    last values give x = x' + C G + X Rk, equal to the whole-line solve."""
    from oracle import oracle as O

    n, S = bounds[-1], 2
    rng = np.random.default_rng(len(bounds))
    D, decay = np.array([3.7e4, 900.0]), np.array([0.3, 0.02])
    c1, den, cx = O.oracle_thomas(n, S, 10.0, 0.01, D, decay)
    p = rng.random((n, S))
    # the reference's sequence on the whole line
    ref = p.copy()
    ref[0] /= den[0]
    for k in range(1, n):
        ref[k] = (ref[k] + c1 * ref[k - 1]) / den[k]
    for k in range(n - 2, -1, -1):
        ref[k] -= cx[k] * ref[k + 1]
    a = -cx  # forward and backward slopes (c = a except at the line end)
    c = np.where(np.arange(n)[:, None] + 1 < n, -cx, 0.0)
    R = len(bounds) - 1
    local, cst, pts = [], [], []
    for r in range(R):
        g0, g1 = bounds[r], bounds[r + 1]
        q, x = np.zeros((g1 - g0, S)), np.zeros((g1 - g0, S))
        prev = np.zeros(S)
        for k in range(g0, g1):
            prev = (p[k] + c1 * prev) / den[k]
            q[k - g0] = prev
        nxt = np.zeros(S)
        for k in range(g1 - 1, g0 - 1, -1):
            nxt = q[k - g0] + c[k] * nxt
            x[k - g0] = nxt
        A = np.cumprod(a[g0:g1], axis=0)
        G, Rk = np.zeros((g1 - g0 + 1, S)), np.ones((g1 - g0 + 1, S))
        for k in range(g1 - 1, g0 - 1, -1):
            G[k - g0] = A[k - g0] + c[k] * G[k - g0 + 1]
            Rk[k - g0] = c[k] * Rk[k - g0 + 1]
        local.append(x)
        cst.append((A[-1], G[0], Rk[0]))
        pts.append((G[:-1], Rk[:-1]))
    out = np.zeros((n, S))
    for rank in range(R):
        Q, C = np.zeros(S), []
        for r in range(R):
            C.append(Q)
            Q = cst[r][0] * Q + local[r][-1]
        X = np.zeros(S)
        for r in range(R - 1, rank, -1):
            X = local[r][0] + C[r] * cst[r][1] + cst[r][2] * X
        g0, g1 = bounds[rank], bounds[rank + 1]
        out[g0:g1] = local[rank] + C[rank] * pts[rank][0] + X * pts[rank][1]
    assert np.all(np.abs(out - ref).max(axis=0) / np.abs(ref).max(axis=0) <= 1e-13)
