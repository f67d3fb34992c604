"""Batch plane mode (BFVM_BATCH_PLANES): all steps of a group's members in
one cooperative launch, two phases per step (xy planes staged in shared
memory, their x lines given their bulk and agent updates and solved, then
their y lines; xz strips solved along z).  Every member must end where stepping it
alone ends: against the oracle, FP64 relative max-norm per substrate
<= 1e-12; against the plain single-instance path, <= 1e-10."""
import numpy as np
import pytest

from biofvm_b200 import STEP_ALL, STEP_CELLS, STEP_DIFFUSION, Batch, Solver, load_scenario
from biofvm_b200 import workloads as W
from biofvm_b200._abi import BATCH_PLANES
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL_BATCH_VS_PLAIN = 1e-10


def members(seed, count):
    """Uneven shapes (1 to 40 points per axis), 1-4 substrates, agents with
    shared voxels, bulk and Dirichlet on some members."""
    rng = np.random.default_rng(seed)
    out = []
    for b in range(count):
        shape = tuple(int(v) for v in rng.integers(1, 41, 3))
        out.append(W.mixed_small(shape=shape, S=int(rng.integers(1, 5)),
                                 n_agents=int(rng.integers(0, 300)), seed=seed * 10 + b,
                                 dirichlet=bool(b % 2), bulk=bool(b % 3)))
    return out


def run_planes(scns, steps, flags=STEP_ALL, budget=-1, calls=1):
    sols = [Solver(0) for _ in scns]
    for sv, scn in zip(sols, scns):
        load_scenario(sv, scn)
    with Batch(0) as bt:
        for sv in sols:
            bt.add(sv)
        bt.set_config((0, 0, 0), (0, 0, 0), budget)
        bt.set_mode(BATCH_PLANES)
        for _ in range(calls):
            bt.step(scns[0].dt, steps, flags)
        bt.synchronize()
        plan = bt.plan()
        out = [sv.get_densities() for sv in sols]
    for sv in sols:
        sv.close()
    return out, plan


def check_oracle(scns, got, steps, flags=STEP_ALL, what=""):
    for scn, p in zip(scns, got):
        ref = O.oracle_run(scn, steps, flags)
        err = O.max_rel_err(p, ref)
        assert np.all(err <= TOL64), (what, scn.shape, scn.S, err.max())


@pytest.mark.parametrize("budget", [-1, 0, 200_000], ids=["default-groups", "one-group",
                                                         "small-groups"])
def test_planes_match_oracle_per_member(budget):
    scns = members(seed=121, count=7)
    got, (groups, kernels) = run_planes(scns, 4, budget=budget)
    assert kernels >= groups
    if budget == 0:
        assert groups == 1
    check_oracle(scns, got, 4, what=budget)


def test_planes_one_launch_per_group():
    """Members without bulk, agents or Dirichlet nodes need no maps: the
    graph holds one memset of the work counters and one kernel per group."""
    scns = [W.mixed_small(shape=(20 + 3 * b, 17, 11 + b), S=1 + b % 3, n_agents=0, seed=390 + b,
                          dirichlet=False, bulk=False) for b in range(4)]
    got, (groups, kernels) = run_planes(scns, 7, budget=0)
    assert groups == 1 and kernels == 1
    check_oracle(scns, got, 7)


def test_planes_graph_replay_and_partial_flags():
    scns = members(seed=122, count=4)
    got, _ = run_planes(scns, 2, calls=3)
    check_oracle(scns, got, 6, what="3 calls")
    # diffusion only (plane groups); sources only (no sweep: branches)
    for flags in (STEP_DIFFUSION, STEP_CELLS | 1, STEP_DIFFUSION | STEP_CELLS):
        got, _ = run_planes(scns, 3, flags=flags)
        check_oracle(scns, got, 3, flags, what=flags)


def test_planes_split_densities_and_strips():
    """xy planes too large for one item hold a subset of the densities
    (128 x 120 x 8: one density per item; 100 x 90 x 7: two per item); xz
    planes too large for one item are cut into strips of columns
    (128 x 7 x 120 x 20: 2560 columns of 120 points, the z pairs read from
    the member's table); 128-point lines on every axis; a 128 x 128 plane of
    one density fills an item."""
    scns = [W.mixed_small(shape=(128, 120, 6), S=8, n_agents=300, seed=401),
            W.mixed_small(shape=(100, 90, 9), S=7, n_agents=200, seed=402),
            W.mixed_small(shape=(128, 7, 120), S=20, n_agents=100, seed=403),
            W.mixed_small(shape=(5, 128, 128), S=2, n_agents=100, seed=404),
            W.mixed_small(shape=(128, 128, 3), S=1, n_agents=50, seed=405)]
    got, (groups, _) = run_planes(scns, 3, budget=0)
    assert groups == 1  # every member runs in the plane kernel
    check_oracle(scns, got, 3)


def test_planes_degenerate_axes():
    """Axes of one point (n = 1 lines) and two points, odd and even sizes."""
    shapes = [(1, 17, 9), (13, 1, 8), (10, 11, 1), (1, 1, 30), (2, 2, 2), (31, 2, 1)]
    scns = [W.mixed_small(shape=sh, S=1 + k % 4, n_agents=20 * k, seed=410 + k,
                          dirichlet=bool(k % 2)) for k, sh in enumerate(shapes)]
    got, _ = run_planes(scns, 3)
    check_oracle(scns, got, 3)


def test_planes_longer_members_on_branches():
    scns = [W.mixed_small(shape=(128, 6, 5), S=2, n_agents=80, seed=93),
            W.mixed_small(shape=(140, 4, 3), S=2, n_agents=30, seed=96)]
    got, (groups, _) = run_planes(scns, 3)
    assert groups >= 2
    check_oracle(scns, got, 3)


def test_planes_see_member_changes_between_calls():
    """New agents (another count), then new Dirichlet values (same nodes)
    between calls: the maps are rebuilt from the members' lists."""
    a = W.mixed_small(shape=(12, 9, 8), S=2, n_agents=100, seed=97)
    b = W.mixed_small(shape=(12, 9, 8), S=2, n_agents=400, seed=98)
    c = W.mixed_small(shape=(7, 12, 5), S=3, n_agents=60, seed=99)
    s1, s2, r1, r2 = Solver(0), Solver(0), Solver(0), Solver(0)
    for sv, sc in ((s1, a), (s2, c), (r1, a), (r2, c)):
        load_scenario(sv, sc)
    node = int(c.dirichlet_voxels[0])
    with Batch(0) as bt:
        bt.set_mode(BATCH_PLANES)
        bt.add(s1)
        bt.add(s2)

        def both():
            bt.step(a.dt, 2)
            r1.step(a.dt, 2)
            r2.step(a.dt, 2)

        both()
        for sv in (s1, r1):
            sv.set_agents(*b.agent_arrays())
        both()
        for sv in (s2, r2):
            sv.update_dirichlet_node(node, np.full(c.S, 0.25))
        both()
        bt.synchronize()
        for s, r in ((s1, r1), (s2, r2)):
            assert np.all(O.max_rel_err(s.get_densities(), r.get_densities()) <= TOL64)
    for sv in (s1, s2, r1, r2):
        sv.close()


def test_planes_batched_workload_sample_matches_plain():
    scns = W.batched_instances(count=6, seed=100, n_min=20, n_max=96, max_agents=4000)
    got, _ = run_planes(scns, 6)
    for scn, p in zip(scns, got):
        with Solver(0) as sv:
            load_scenario(sv, scn)
            sv.step(scn.dt, 6)
            plain = sv.get_densities()
        assert np.all(O.max_rel_err(p, plain) <= TOL_BATCH_VS_PLAIN), scn.shape
    check_oracle(scns, got, 6)


def test_planes_fp32_members_run_on_branches():
    scns = members(seed=131, count=3)
    sols = [Solver(0) for _ in scns]
    for sv, scn in zip(sols, scns):
        load_scenario(sv, scn)
        sv.set_precision(32)
        sv.set_densities(scn.initial_field())
    with Batch(0) as bt:
        bt.set_mode(BATCH_PLANES)
        for sv in sols:
            bt.add(sv)
        bt.step(scns[0].dt, 3)
        bt.synchronize()
        got = [sv.get_densities() for sv in sols]
    for sv in sols:
        sv.close()
    for scn, p in zip(scns, got):
        ref = O.oracle_run(scn, 3, 7)
        assert np.all(O.max_rel_err(p, ref) <= 1e-5), scn.shape
