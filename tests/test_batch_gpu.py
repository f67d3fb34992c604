"""Many microenvironments in one batch (bfvm_batch_*): each member must end
where stepping it alone ends.  Against the oracle: FP64 relative max-norm per
substrate <= 1e-12 (the same bar as one instance); batched vs the plain
single-instance path: <= 1e-10."""
import numpy as np
import pytest

from biofvm_b200 import STEP_ALL, STEP_CELLS, STEP_DIFFUSION, Batch, BfvmError, Solver, load_scenario
from biofvm_b200 import workloads as W
from biofvm_b200._abi import BATCH_BRANCHES, BATCH_FUSED, BATCH_PERSISTENT
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL_BATCH_VS_PLAIN = 1e-10


def members(seed=71, count=6):
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


def run_batch(scns, steps, flags=STEP_ALL, config=None, tune=False, calls=1, mode=BATCH_FUSED,
              pchunk=None):
    sols = [Solver(0) for _ in scns]
    for sv, scn in zip(sols, scns):
        load_scenario(sv, scn)
    with Batch(0) as bt:
        for sv in sols:
            bt.add(sv)
        if config:
            bt.set_config(*config)
        bt.set_mode(mode)
        if pchunk:
            bt.set_persistent_chunk(pchunk)
        if tune:
            bt.tune(scns[0].dt, flags, 2)
        for _ in range(calls):
            bt.step(scns[0].dt, steps, flags)
        bt.synchronize()
        plan = bt.plan()
        out = [sv.get_densities() for sv in sols]
    for sv in sols:
        sv.close()
    return out, plan


def test_batch_matches_oracle_per_member():
    scns = members()
    got, (groups, kernels) = run_batch(scns, 3)
    assert kernels > 0
    for scn, p in zip(scns, got):
        ref = O.oracle_run(scn, 3, 7)
        assert np.all(O.max_rel_err(p, ref) <= TOL64), scn.shape


def test_batch_matches_plain_solves():
    scns = members(seed=72, count=5)
    got, _ = run_batch(scns, 4)
    for scn, p in zip(scns, got):
        with Solver(0) as sv:
            load_scenario(sv, scn)
            sv.step(scn.dt, 4)
            plain = sv.get_densities()
        assert np.all(O.max_rel_err(p, plain) <= TOL_BATCH_VS_PLAIN), scn.shape


@pytest.mark.parametrize("config", [
    ((8, 8, 8), (512, 512, 512), 0),
    ((16, 16, 16), (256, 256, 256), 0),
    ((32, 32, 32), (128, 128, 128), 0),
    ((16, 32, 8), (512, 256, 512), 1),      # every member its own group
    ((0, 0, 0), (0, 0, 0), 200_000),       # small groups
], ids=["ch8", "ch16", "ch32", "mixed-own-groups", "auto-small-groups"])
def test_batch_configs_agree(config):
    scns = members(seed=73, count=5)
    got, (groups, _) = run_batch(scns, 2, config=config)
    if config[2] == 1:
        assert groups == len(scns)
    for scn, p in zip(scns, got):
        ref = O.oracle_run(scn, 2, 7)
        assert np.all(O.max_rel_err(p, ref) <= TOL64), (config, scn.shape)


def test_graph_replay_over_several_calls():
    """The captured graph is replayed by later calls with the same plan."""
    scns = members(seed=74, count=4)
    got, _ = run_batch(scns, 2, calls=3)
    for scn, p in zip(scns, got):
        ref = O.oracle_run(scn, 6, 7)
        assert np.all(O.max_rel_err(p, ref) <= TOL64), scn.shape


def test_tuning_leaves_fields_unchanged():
    scns = members(seed=75, count=4)
    got, _ = run_batch(scns, 2, tune=True)
    for scn, p in zip(scns, got):
        ref = O.oracle_run(scn, 2, 7)
        assert np.all(O.max_rel_err(p, ref) <= TOL64), scn.shape


def test_member_changes_between_calls_are_seen():
    """set_agents on a member between batch calls: the plan is rebuilt."""
    a = W.mixed_small(shape=(10, 9, 8), S=2, n_agents=100, seed=76)
    b = W.mixed_small(shape=(10, 9, 8), S=2, n_agents=40, seed=77)
    c = W.mixed_small(shape=(7, 12, 5), S=3, n_agents=60, seed=78)
    s1, s2 = Solver(0), Solver(0)
    load_scenario(s1, a)
    load_scenario(s2, c)
    with Batch(0) as bt:
        bt.add(s1)
        bt.add(s2)
        bt.step(a.dt, 1, STEP_CELLS)
        s1.set_agents(*b.agent_arrays())
        bt.step(a.dt, 1, STEP_CELLS)
        bt.synchronize()
    got = s1.get_densities()
    lib = O.load_oracle()
    exp = a.initial_field()
    for scn in (a, b):
        v, t1, t2 = (np.ascontiguousarray(x) for x in scn.agent_arrays())
        lib.or_cells(v.size, a.S, O._d(exp), O._l(v), O._d(t1), O._d(t2))
    assert np.array_equal(got, exp)
    s1.close()
    s2.close()


def test_batch_diffusion_only_and_sources_only():
    scns = members(seed=79, count=3)
    for flags in (STEP_DIFFUSION, STEP_CELLS | 1):
        got, _ = run_batch(scns, 2, flags=flags)
        for scn, p in zip(scns, got):
            ref = O.oracle_run(scn, 2, flags)
            assert np.all(O.max_rel_err(p, ref) <= TOL64), (flags, scn.shape)


def test_batch_rejects_mixed_precision_and_non_uniform_mesh():
    with Solver(0) as a, Solver(0) as b, Batch(0) as bt:
        a.resize_space(0, 100, 0, 100, 0, 100, 10)
        b.resize_space(0, 100, 0, 100, 0, 100, 10)
        b.set_precision(32)
        bt.add(a)
        with pytest.raises(BfvmError):
            bt.add(b)
        c = Solver(0)
        c.resize_space(0, 100, 0, 100, 0, 100, 10, 20, 10)
        bt.add(c)
        with pytest.raises(BfvmError) as e:
            bt.step(0.01, 1)
        assert "uniform Cartesian" in str(e.value)
        bt.clear()
        c.close()


def test_batched_workload_small_sample_matches_plain():
    """Members drawn like the 64-instance batched workload (4 of them, 200
    steps would be slow for the oracle: 5 steps against plain solves)."""
    scns = W.batched_instances(count=4, seed=80, n_min=16, n_max=48, max_agents=3000)
    got, _ = run_batch(scns, 5)
    for scn, p in zip(scns, got):
        with Solver(0) as sv:
            load_scenario(sv, scn)
            sv.step(scn.dt, 5)
            plain = sv.get_densities()
        assert np.all(O.max_rel_err(p, plain) <= TOL_BATCH_VS_PLAIN), scn.shape


# ---- branch mode: every member's own single-instance kernels on concurrent
# graph branches ----

def plain_solves(scns, steps, flags=STEP_ALL):
    out = []
    for scn in scns:
        with Solver(0) as sv:
            load_scenario(sv, scn)
            sv.set_grid_steps(False)  # the sweep kernels, as the batch's branches
            sv.step(scn.dt, steps, flags)
            out.append(sv.get_densities())
    return out


@pytest.mark.parametrize("budget", [-1, 0, 200_000], ids=["default-groups", "one-group",
                                                         "small-groups"])
def test_branches_reproduce_plain_solves_bit_for_bit(budget):
    """The same kernels in the same order per member: identical fields."""
    scns = members(seed=81, count=6)
    got, (groups, kernels) = run_batch(scns, 3, config=((0, 0, 0), (0, 0, 0), budget),
                                       mode=BATCH_BRANCHES)
    assert kernels > 0
    if budget == 0:
        assert groups == 1
    for p, ref in zip(got, plain_solves(scns, 3)):
        assert np.array_equal(p, ref)


def test_branches_match_oracle_per_member():
    scns = members(seed=82, count=5)
    got, _ = run_batch(scns, 3, mode=BATCH_BRANCHES)
    for scn, p in zip(scns, got):
        ref = O.oracle_run(scn, 3, 7)
        assert np.all(O.max_rel_err(p, ref) <= TOL64), scn.shape


def test_branches_graph_replay_and_partial_flags():
    scns = members(seed=83, count=4)
    got, _ = run_batch(scns, 2, calls=3, mode=BATCH_BRANCHES)
    for p, ref in zip(got, plain_solves(scns, 6)):
        assert np.array_equal(p, ref)
    for flags in (STEP_DIFFUSION, STEP_CELLS | 1):
        got, _ = run_batch(scns, 2, flags=flags, mode=BATCH_BRANCHES)
        for scn, p in zip(scns, got):
            ref = O.oracle_run(scn, 2, flags)
            assert np.all(O.max_rel_err(p, ref) <= TOL64), (flags, scn.shape)


def test_branches_see_member_changes_between_calls():
    """New agents on a member between calls (another count: new device
    buffers): the graph is captured again."""
    a = W.mixed_small(shape=(10, 9, 8), S=2, n_agents=100, seed=84)
    b = W.mixed_small(shape=(10, 9, 8), S=2, n_agents=400, seed=85)
    c = W.mixed_small(shape=(7, 12, 5), S=3, n_agents=60, seed=86)
    s1, s2 = Solver(0), Solver(0)
    load_scenario(s1, a)
    load_scenario(s2, c)
    r1, r2 = Solver(0), Solver(0)
    load_scenario(r1, a)
    load_scenario(r2, c)
    for sv in (r1, r2):
        sv.set_grid_steps(False)  # the sweep kernels, as the batch's branches
    with Batch(0) as bt:
        bt.set_mode(BATCH_BRANCHES)
        bt.add(s1)
        bt.add(s2)
        bt.step(a.dt, 2)
        r1.step(a.dt, 2)
        r2.step(a.dt, 2)
        for sv in (s1, r1):
            sv.set_agents(*b.agent_arrays())
        bt.step(a.dt, 2)
        r1.step(a.dt, 2)
        r2.step(a.dt, 2)
        bt.synchronize()
        assert np.array_equal(s1.get_densities(), r1.get_densities())
        assert np.array_equal(s2.get_densities(), r2.get_densities())
    for sv in (s1, s2, r1, r2):
        sv.close()


def test_tuner_picks_a_mode_and_keeps_fields():
    scns = members(seed=87, count=4)
    sols = [Solver(0) for _ in scns]
    for sv, scn in zip(sols, scns):
        load_scenario(sv, scn)
    with Batch(0) as bt:
        for sv in sols:
            bt.add(sv)
        bt.tune(scns[0].dt, STEP_ALL, 2)
        assert bt.get_mode() in (BATCH_FUSED, BATCH_BRANCHES, BATCH_PERSISTENT)
        bt.step(scns[0].dt, 2)
        bt.synchronize()
        got = [sv.get_densities() for sv in sols]
    for sv in sols:
        sv.close()
    for scn, p in zip(scns, got):
        ref = O.oracle_run(scn, 2, 7)
        assert np.all(O.max_rel_err(p, ref) <= TOL64), scn.shape


def test_set_mode_rejects_unknown_modes():
    with Batch(0) as bt:
        with pytest.raises(BfvmError):
            bt.set_mode(7)


# ---- persistent mode: all steps of a group's members in one cooperative
# launch, phases shared by the members and separated by grid barriers ----

@pytest.mark.parametrize("pchunk", [4, 8, 16, 32, 0], ids=["ch4", "ch8", "ch16", "tiles32", "lines"])
@pytest.mark.parametrize("budget", [-1, 0, 200_000], ids=["default-groups", "one-group",
                                                         "small-groups"])
def test_persistent_matches_oracle_per_member(pchunk, budget):
    scns = members(seed=91, count=6)
    got, (groups, kernels) = run_batch(scns, 4, config=((0, 0, 0), (0, 0, 0), budget),
                                       mode=BATCH_PERSISTENT, pchunk=pchunk)
    assert kernels >= groups  # one cooperative launch per group (+ each member's maps)
    if budget == 0:
        assert groups == 1
    for scn, p in zip(scns, got):
        ref = O.oracle_run(scn, 4, 7)
        assert np.all(O.max_rel_err(p, ref) <= TOL64), (pchunk, budget, scn.shape)


def test_persistent_one_launch_per_group():
    """Members without bulk, agents or Dirichlet nodes need no maps: the
    graph holds exactly one kernel per group, whatever the step count."""
    scns = [W.mixed_small(shape=(20 + 3 * b, 17, 11 + b), S=1 + b % 3, n_agents=0, seed=190 + b,
                          dirichlet=False, bulk=False) for b in range(4)]
    got, (groups, kernels) = run_batch(scns, 7, config=((0, 0, 0), (0, 0, 0), 0),
                                       mode=BATCH_PERSISTENT)
    assert groups == 1 and kernels == 1
    for scn, p in zip(scns, got):
        ref = O.oracle_run(scn, 7, 7)
        assert np.all(O.max_rel_err(p, ref) <= TOL64), scn.shape


@pytest.mark.parametrize("pchunk", [8, 32, 0], ids=["ch8", "tiles32", "lines"])
def test_persistent_graph_replay_and_partial_flags(pchunk):
    scns = members(seed=92, count=4)
    got, _ = run_batch(scns, 2, calls=3, mode=BATCH_PERSISTENT, pchunk=pchunk)
    for scn, p in zip(scns, got):
        ref = O.oracle_run(scn, 6, 7)
        assert np.all(O.max_rel_err(p, ref) <= TOL64), scn.shape
    # diffusion only (persistent groups); sources only (no sweep: branches)
    for flags in (STEP_DIFFUSION, STEP_CELLS | 1, STEP_DIFFUSION | STEP_CELLS):
        got, _ = run_batch(scns, 3, flags=flags, mode=BATCH_PERSISTENT, pchunk=pchunk)
        for scn, p in zip(scns, got):
            ref = O.oracle_run(scn, 3, flags)
            assert np.all(O.max_rel_err(p, ref) <= TOL64), (flags, scn.shape)


def test_persistent_lines_of_128_points_and_longer_members_on_branches():
    """A member with 128-point lines runs in the persistent kernel (16 chunks
    of 8); one with a 140-point axis cannot and runs on a branch."""
    scns = [W.mixed_small(shape=(128, 6, 5), S=2, n_agents=80, seed=93),
            W.mixed_small(shape=(5, 128, 7), S=1, n_agents=50, seed=94),
            W.mixed_small(shape=(6, 5, 128), S=3, n_agents=50, seed=95),
            W.mixed_small(shape=(140, 4, 3), S=2, n_agents=30, seed=96)]
    for pchunk in (8, 16, 32, 0):
        got, (groups, _) = run_batch(scns, 3, mode=BATCH_PERSISTENT, pchunk=pchunk)
        assert groups >= 2  # the 140-point member is in a group of its own kind
        for scn, p in zip(scns, got):
            ref = O.oracle_run(scn, 3, 7)
            assert np.all(O.max_rel_err(p, ref) <= TOL64), (pchunk, scn.shape)


def test_persistent_sees_member_changes_between_calls():
    """New agents (another count), then new Dirichlet values (same nodes)
    between calls: the maps are rebuilt from the members' lists every call."""
    a = W.mixed_small(shape=(12, 9, 8), S=2, n_agents=100, seed=97)
    b = W.mixed_small(shape=(12, 9, 8), S=2, n_agents=400, seed=98)
    c = W.mixed_small(shape=(7, 12, 5), S=3, n_agents=60, seed=99)
    s1, s2 = Solver(0), Solver(0)
    load_scenario(s1, a)
    load_scenario(s2, c)
    r1, r2 = Solver(0), Solver(0)
    load_scenario(r1, a)
    load_scenario(r2, c)
    new_val = np.full(c.S, 0.25)
    node = int(c.dirichlet_voxels[0])
    with Batch(0) as bt:
        bt.set_mode(BATCH_PERSISTENT)
        bt.add(s1)
        bt.add(s2)
        bt.step(a.dt, 2)
        r1.step(a.dt, 2)
        r2.step(a.dt, 2)
        for sv in (s1, r1):
            sv.set_agents(*b.agent_arrays())
        bt.step(a.dt, 2)
        r1.step(a.dt, 2)
        r2.step(a.dt, 2)
        for sv in (s2, r2):
            sv.update_dirichlet_node(node, new_val)
        bt.step(a.dt, 2)
        r1.step(a.dt, 2)
        r2.step(a.dt, 2)
        bt.synchronize()
        for s, r in ((s1, r1), (s2, r2)):
            assert np.all(O.max_rel_err(s.get_densities(), r.get_densities()) <= TOL64)
    for sv in (s1, s2, r1, r2):
        sv.close()


@pytest.mark.parametrize("pchunk", [8, 32, 0], ids=["ch8", "tiles32", "lines"])
def test_persistent_batched_workload_sample_matches_plain(pchunk):
    scns = W.batched_instances(count=5, seed=100, n_min=20, n_max=64, max_agents=4000)
    got, _ = run_batch(scns, 6, mode=BATCH_PERSISTENT, pchunk=pchunk)
    for scn, p in zip(scns, got):
        with Solver(0) as sv:
            load_scenario(sv, scn)
            sv.step(scn.dt, 6)
            plain = sv.get_densities()
        assert np.all(O.max_rel_err(p, plain) <= TOL_BATCH_VS_PLAIN), scn.shape
        ref = O.oracle_run(scn, 6, 7)
        assert np.all(O.max_rel_err(p, ref) <= TOL64), scn.shape


def test_persistent_fp32_members_run_on_branches():
    """FP32 members cannot run in the FP64 persistent kernel: the batch runs
    them on branches, within the FP32 bar against the FP64 oracle."""
    scns = members(seed=101, count=3)
    sols = [Solver(0) for _ in scns]
    for sv, scn in zip(sols, scns):
        load_scenario(sv, scn)
        sv.set_precision(32)
        sv.set_densities(scn.initial_field())
    with Batch(0) as bt:
        bt.set_mode(BATCH_PERSISTENT)
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


@pytest.mark.parametrize("pchunk", [32, 8])
def test_persistent_many_densities(pchunk):
    """Members with 12 and 20 densities: the tile form stages chunk tables of
    more than 48 KB in shared memory (the kernel's limit is raised while the
    batch is planned); every form matches the oracle."""
    scns = [W.mixed_small(shape=(70, 40, 33), S=12, n_agents=200, seed=301),
            W.mixed_small(shape=(128, 21, 17), S=20, n_agents=100, seed=302),
            W.mixed_small(shape=(20, 31, 90), S=3, n_agents=50, seed=303)]
    got, _ = run_batch(scns, 3, mode=BATCH_PERSISTENT, pchunk=pchunk)
    for scn, p in zip(scns, got):
        ref = O.oracle_run(scn, 3, 7)
        assert np.all(O.max_rel_err(p, ref) <= TOL64), (pchunk, scn.shape, scn.S)


def test_persistent_chunk_setter_rejects_other_lengths():
    with Batch(0) as bt:
        with pytest.raises(BfvmError):
            bt.set_persistent_chunk(12)
        bt.set_persistent_chunk(16)
        assert bt.get_persistent_chunk() == 16
        bt.set_persistent_chunk(0)
        assert bt.get_persistent_chunk() == 0
