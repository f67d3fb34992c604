"""The FP64 tangent-linear model (oracle/tangent_linear.py) that checks the
GPU adjoint, pinned on the CPU: its primal is the oracle's field bit for bit,
and its directional derivatives agree with central finite differences."""
import numpy as np
import pytest

from biofvm_b200 import workloads as W
from oracle import oracle as O
from oracle import tangent_linear as TL


def scenario():
    return W.mixed_small(shape=(7, 6, 5), S=2, n_agents=40, seed=91)


def params(scn):
    return (np.array(scn.agent_secretion, float), np.array(scn.agent_uptake, float),
            np.array(scn.D, float), np.array(scn.decay, float))


def direction(scn, seed):
    rng = np.random.default_rng(seed)
    sec, upt, D, decay = params(scn)
    return (sec * rng.standard_normal(sec.shape), upt * rng.standard_normal(upt.shape),
            D * rng.standard_normal(D.shape), decay * rng.standard_normal(decay.shape))


def test_primal_is_the_oracle_field():
    scn = scenario()
    zero = [np.zeros_like(x) for x in params(scn)]
    p, _ = TL.tangent_run(scn, 4, 7, *params(scn), *zero)
    assert np.array_equal(p, O.oracle_run(scn, 4, 7))


@pytest.mark.parametrize("flags", [7, 4, 3])
def test_tangent_matches_central_differences(flags):
    scn = scenario()
    th = params(scn)
    v = direction(scn, 5)
    zero = [np.zeros_like(x) for x in th]
    rng = np.random.default_rng(6)
    target = rng.uniform(0, 2, (scn.num_voxels, scn.S))

    def loss(t):
        p, _ = TL.tangent_run(scn, 4, flags, *t, *zero)
        return 0.5 * np.sum((p - target) ** 2)

    p, pd = TL.tangent_run(scn, 4, flags, *th, *v)
    dL = np.sum((p - target) * pd)
    h = 1e-6
    lp = loss([a + h * b for a, b in zip(th, v)])
    lm = loss([a - h * b for a, b in zip(th, v)])
    fd = (lp - lm) / (2 * h)
    assert abs(fd - dL) <= 1e-6 * abs(dL), (fd, dL)
