"""The GPU adjoint (bfvm_adjoint_forward/backward) against the FP64
tangent-linear model of the oracle and against central finite differences of
the GPU forward.  Tolerances: adjoint . v vs tangent-linear dLoss <= 1e-9
relative (both exact derivatives of the same discrete map in FP64); vs
central differences (h = 1e-6 relative perturbation) <= 1e-6."""
import numpy as np
import pytest

from biofvm_b200 import BfvmError
from biofvm_b200 import workloads as W
from biofvm_b200.adjoint import AdjointProblem, loss_difference, transport
from oracle import tangent_linear as TL

pytestmark = pytest.mark.gpu


def params(scn):
    return (np.array(scn.agent_secretion, float), np.array(scn.agent_uptake, float),
            np.array(scn.D, float), np.array(scn.decay, float))


def direction(scn, seed):
    rng = np.random.default_rng(seed)
    sec, upt, D, decay = params(scn)
    return (sec * rng.standard_normal(sec.shape), upt * rng.standard_normal(upt.shape),
            D * rng.standard_normal(D.shape), decay * rng.standard_normal(decay.shape))


def dot(g, v):
    return (np.sum(g["secretion"] * v[0]) + np.sum(g["uptake"] * v[1]) + np.sum(g["D"] * v[2])
            + np.sum(g["decay"] * v[3]))


CASES = {
    # shape, S, agents, steps, checkpoint interval, flags
    "all-parts": ((9, 7, 6), 2, 60, 5, 2, 7),
    "one-segment": ((6, 8, 5), 3, 30, 4, 10, 7),
    "diffusion-only": ((8, 6, 7), 2, 0, 4, 3, 4),
    "sources-only": ((5, 6, 4), 2, 50, 3, 2, 3),
    "thin-axes": ((12, 1, 3), 1, 20, 6, 4, 7),
}


@pytest.mark.parametrize("name", list(CASES))
def test_adjoint_matches_tangent_linear(name):
    shape, S, A, steps, k, flags = CASES[name]
    scn = W.mixed_small(shape=shape, S=S, n_agents=A, seed=sum(shape) + S)
    th = params(scn)
    v = direction(scn, 3)
    target = np.random.default_rng(4).uniform(0, 2, (scn.num_voxels, S))
    prob = AdjointProblem(scn, steps, checkpoint_every=k, flags=flags)
    try:
        p = prob.forward(*th)
        g = prob.backward(p - target)
    finally:
        prob.close()
    pt, pd = TL.tangent_run(scn, steps, flags, *th, *v)
    dL = np.sum((pt - target) * pd)
    adj = dot(g, v)
    assert abs(adj - dL) <= 1e-9 * abs(dL), (adj, dL)


def test_adjoint_matches_central_differences_on_the_gpu():
    scn = W.mixed_small(shape=(10, 8, 6), S=2, n_agents=80, seed=21)
    th = params(scn)
    v = direction(scn, 5)
    target = np.random.default_rng(6).uniform(0, 2, (scn.num_voxels, scn.S))
    prob = AdjointProblem(scn, 6, checkpoint_every=4)
    try:
        p = prob.forward(*th)
        g = prob.backward(p - target)
        h = 1e-6
        pp = prob.run(*[a + h * b for a, b in zip(th, v)])
        pm = prob.run(*[a - h * b for a, b in zip(th, v)])
    finally:
        prob.close()
    fd = loss_difference(pp, pm, target) / (2 * h)
    adj = dot(g, v)
    assert abs(adj - fd) <= 1e-6 * abs(fd), (adj, fd)


def test_adjoint_of_the_initial_field():
    scn = W.mixed_small(shape=(7, 6, 5), S=2, n_agents=30, seed=22)
    th = params(scn)
    zero = [np.zeros_like(x) for x in th]
    rng = np.random.default_rng(7)
    dp0 = rng.standard_normal((scn.num_voxels, scn.S))
    target = rng.uniform(0, 2, (scn.num_voxels, scn.S))
    prob = AdjointProblem(scn, 4, checkpoint_every=3)
    try:
        p = prob.forward(*th)
        g = prob.backward(p - target, want_p0=True)
    finally:
        prob.close()
    pt, pd = TL.tangent_run(scn, 4, 7, *th, *zero, dp0=dp0)
    dL = np.sum((pt - target) * pd)
    assert abs(np.sum(g["p0"] * dp0) - dL) <= 1e-9 * abs(dL)


def test_torch_autograd_wrapper():
    import torch

    scn = W.mixed_small(shape=(8, 7, 5), S=2, n_agents=40, seed=23)
    th = params(scn)
    target = np.random.default_rng(8).uniform(0, 2, (scn.num_voxels, scn.S))
    prob = AdjointProblem(scn, 3, checkpoint_every=2)
    try:
        ts = [torch.tensor(x, dtype=torch.float64, device="cuda", requires_grad=True) for x in th]
        out = transport(prob, *ts)
        loss = 0.5 * ((out - torch.tensor(target, device="cuda")) ** 2).sum()
        loss.backward()
        p = prob.forward(*th)
        g = prob.backward(p - target)
    finally:
        prob.close()
    for t, key in zip(ts, ("secretion", "uptake", "D", "decay")):
        np.testing.assert_allclose(t.grad.cpu().numpy(), g[key], rtol=1e-12, atol=0)


def test_backward_refuses_a_changed_solver():
    scn = W.mixed_small(shape=(6, 5, 4), S=1, n_agents=10, seed=24)
    prob = AdjointProblem(scn, 2, checkpoint_every=1)
    try:
        p = prob.forward(*params(scn))
        prob.solver.set_agents(*W.mixed_small(shape=(6, 5, 4), S=1, n_agents=3,
                                               seed=25).agent_arrays())
        with pytest.raises(BfvmError):
            prob.backward(p)
    finally:
        prob.close()
