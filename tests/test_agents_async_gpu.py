"""The asynchronous agent exchange (bfvm_set_agents_async,
bfvm_get_agent_densities_async, bfvm_wait_transfers) against the synchronous
calls: the same agents each step give bit-identical agent densities and
fields, whatever the overlap of the copies with the steps."""
import numpy as np
import pytest
import torch

from biofvm_b200 import STEP_ALL, Solver, load_scenario
from biofvm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def pinned(a, keep):
    t = torch.empty(a.shape, dtype=torch.from_numpy(a[:0]).dtype, pin_memory=True)
    keep.append(t)
    v = t.numpy()
    v[...] = a
    return v


def agent_steps(scn, steps, seed):
    """Per step: agents that moved (new voxels), changed their rates, and a
    changing count (one step with none)."""
    rng = np.random.default_rng(seed)
    vox, t1, t2 = scn.agent_arrays()
    out = []
    for k in range(steps):
        A = 0 if k == 2 else int(rng.integers(len(vox) // 2, len(vox) + 1))
        v = rng.integers(0, scn.num_voxels, size=A).astype(np.int64)
        f = rng.uniform(0.5, 1.5, size=(A, scn.S))
        a = t1[:A] * f
        b = 1.0 + (t2[:A] - 1.0) * f
        out.append((v, np.ascontiguousarray(a), np.ascontiguousarray(b)))
    return out


SHAPES = [
    ((24, 20, 16), 3),  # whole steps in one cooperative launch
    ((96, 80, 72), 2),  # the sweep kernels
]


@pytest.mark.parametrize("shape,S", SHAPES)
def test_async_exchange_matches_the_synchronous_calls(shape, S):
    scn = W.mixed_small(shape=shape, S=S, n_agents=600, seed=71)
    steps = 6
    agents = agent_steps(scn, steps, 72)

    with Solver(0) as sv:
        load_scenario(sv, scn)
        want = []
        for v, a, b in agents:
            sv.set_agents(v, a, b)
            sv.step(scn.dt, 1, STEP_ALL)
            o = np.empty((len(v), S))
            sv.get_agent_densities(o)
            want.append(o)
        want_p = sv.get_densities()

    keep = []
    with Solver(0) as sv:
        load_scenario(sv, scn)
        host = [tuple(pinned(x, keep) for x in ag) for ag in agents]
        got = [pinned(np.full((len(ag[0]), S), np.nan), keep) for ag in agents]
        for (v, a, b), o in zip(host, got):
            sv.set_agents_async(v, a, b)
            sv.step(scn.dt, 1, STEP_ALL)
            sv.get_agent_densities_async(o)
        sv.wait_transfers()
        got_p = sv.get_densities()

    for k in range(steps):
        assert np.array_equal(got[k], want[k]), k
    assert np.array_equal(got_p, want_p)


def test_async_and_synchronous_calls_mix():
    scn = W.mixed_small(shape=(40, 36, 30), S=2, n_agents=400, seed=73)
    (v0, a0, b0), (v1, a1, b1), _, (v2, a2, b2) = agent_steps(scn, 4, 74)

    def run(calls):
        keep = []
        with Solver(0) as sv:
            load_scenario(sv, scn)
            outs = []
            for c in calls:
                outs.extend(c(sv, keep) or [])
            sv.synchronize()
            return [np.array(o) for o in outs], sv.get_densities()

    def sync_set(v, a, b):
        return lambda sv, keep: sv.set_agents(v, a, b)

    def async_set(v, a, b):
        return lambda sv, keep: sv.set_agents_async(
            pinned(v, keep), pinned(a, keep), pinned(b, keep))

    def step(sv, keep):
        sv.step(scn.dt, 1, STEP_ALL)

    def sync_get(n):
        def f(sv, keep):
            o = np.empty((n, scn.S))
            sv.get_agent_densities(o)
            return [o]
        return f

    def async_get(n):
        def f(sv, keep):
            return [sv.get_agent_densities_async(pinned(np.zeros((n, scn.S)), keep))]
        return f

    n1, n2 = len(v1), len(v2)
    want, want_p = run([sync_set(v1, a1, b1), step, sync_get(n1), sync_set(v2, a2, b2), step,
                        sync_get(n2)])
    sequences = [
        # two uploads before a step (the first never used)
        [async_set(v0, a0, b0), async_set(v1, a1, b1), step, async_get(n1),
         async_set(v2, a2, b2), step, sync_get(n2)],
        # a synchronous set replacing an asynchronous one
        [async_set(v0, a0, b0), sync_set(v1, a1, b1), step, async_get(n1),
         async_set(v2, a2, b2), step, async_get(n2)],
        # an asynchronous read followed by a synchronous one of the same step
        [sync_set(v1, a1, b1), step, async_get(n1), sync_get(n1), sync_set(v2, a2, b2), step,
         sync_get(n2)],
    ]
    for calls in sequences:
        got, got_p = run(calls)
        assert len(got) in (2, 3)
        for g in got[:-1]:
            assert np.array_equal(g, want[0])
        assert np.array_equal(got[-1], want[1])
        assert np.array_equal(got_p, want_p)


def test_wait_without_transfers_and_an_empty_upload():
    scn = W.mixed_small(shape=(12, 10, 8), S=1, n_agents=50, seed=76)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.wait_transfers()
        sv.set_agents_async(np.zeros(0, np.int64), np.zeros((0, 1)), np.zeros((0, 1)))
        sv.step(scn.dt, 1, STEP_ALL)
        out = sv.get_agent_densities_async(np.zeros((0, 1)))
        sv.wait_transfers()
        assert out.shape == (0, 1)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.set_agents(np.zeros(0, np.int64), np.zeros((0, 1)), np.zeros((0, 1)))
        sv.step(scn.dt, 1, STEP_ALL)
        p = sv.get_densities()
    with Solver(0) as sv2:
        load_scenario(sv2, scn)
        sv2.set_agents_async(np.zeros(0, np.int64), np.zeros((0, 1)), np.zeros((0, 1)))
        sv2.step(scn.dt, 1, STEP_ALL)
        assert np.array_equal(sv2.get_densities(), p)
