"""The oracle (plain-C restatement) pinned against the reference: the golden
fixtures made by the unmodified reference, and the compiled reference itself
where oracle/_ref is built.  CPU only."""
import numpy as np
import pytest

from biofvm_b200 import workloads as W
from cases import CASES, input_fingerprint, sha
from conftest import load_golden
from oracle import oracle as O

REF = O.reference_available("core2")


def _check_against_golden(p, g):
    assert tuple(g["shape"]) == p.shape
    if "p" in g:
        # bit-exact: the oracle follows the reference statement by statement
        assert np.array_equal(p, g["p"])
    else:
        assert np.array_equal(p.ravel()[g["sample_idx"]], g["sample_val"])
    assert sha(p) == str(g["sha"])


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_matches_reference_golden(name):
    build, flags, steps, _ = CASES[name]
    scn = build()
    g = load_golden(name)
    assert input_fingerprint(scn) == str(g["fingerprint"]), "scenario builder changed"
    assert int(g["flags"]) == flags and int(g["steps"]) == steps
    if scn.num_agents:
        vox, _, _ = scn.agent_arrays()
        assert np.array_equal(vox, g["agent_voxels"])
        ovox, _, _ = O.oracle_agent_arrays(scn)
        assert np.array_equal(ovox, g["agent_voxels"])
    p = O.oracle_run(scn, steps, flags)
    _check_against_golden(p, g)


@pytest.mark.skipif(not REF, reason="compiled reference (oracle/_ref) not built")
@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_oracle_matches_live_reference(seed):
    rng = np.random.default_rng(seed)
    shape = tuple(int(v) for v in rng.integers(1, 14, 3))
    S = int(rng.integers(1, 5))
    scn = W.mixed_small(shape=shape, S=S, n_agents=int(rng.integers(0, 200)), seed=seed,
                        dirichlet=bool(seed % 2))
    for flags in (1, 2, 4, 7):
        a = O.oracle_run(scn, 3, flags)
        b = O.reference_run(scn, 3, flags)
        assert np.array_equal(a, b), (shape, S, flags)


@pytest.mark.skipif(not REF, reason="compiled reference (oracle/_ref) not built")
def test_reference_individual_calls_match_oracle():
    """apply_dirichlet_conditions and the single simulate_* calls, one by one."""
    scn = W.mixed_small(shape=(9, 8, 7), S=2, n_agents=120, seed=31)
    with O.Reference(scn) as ref:
        ref.apply_dirichlet()
        exp = scn.initial_field()
        O.load_oracle()
        lib = O.load_oracle()
        dv = np.ascontiguousarray(scn.dirichlet_voxels, np.int64)
        dval = np.ascontiguousarray(scn.dirichlet_values)
        lib.or_apply_dirichlet(scn.S, O._d(exp), dv.size, O._l(dv), O._d(dval))
        assert np.array_equal(ref.densities(), exp)


def test_convergence_known_answer():
    """Convergence test 1 of the reference: the 1-D cosine decays as
    exp(-D pi^2 t / L0^2).  The LOD/implicit error is O(dt) + O(dx^2):
    refining dt by 4 and dx by 2 cuts the error by about 4."""
    errs = []
    for dt, dx in ((0.004, 40.0), (0.001, 20.0)):
        scn = W.convergence_1d(dt=dt, t_max=0.2, dx=dx)
        p = O.oracle_run(scn, flags=4)
        exact = W.convergence_1d_exact(scn)
        errs.append(np.abs(p[:, 0] - exact).max())
    assert errs[0] < 2e-2
    assert 3.0 < errs[0] / errs[1] < 5.0, errs


def test_mass_balance_without_sources():
    """Neumann boundaries, no sources: each implicit sweep keeps the total of a
    substrate and divides it by (1 + dt*decay/3), so one step scales it by
    (1 + dt*decay/3)^-3."""
    scn = W.mixed_small(shape=(16, 12, 10), S=3, n_agents=0, seed=4, dirichlet=False,
                        bulk=False)
    p0 = scn.initial_field()
    p1 = O.oracle_run(scn, 1, 4)
    c2 = scn.dt * scn.decay / 3.0
    np.testing.assert_allclose(p1.sum(0), p0.sum(0) / (1 + c2) ** 3, rtol=1e-13)


@pytest.mark.skipif(not REF, reason="compiled reference (oracle/_ref) not built")
@pytest.mark.parametrize("shape", [(17, 13, 1), (9, 11, 3), (1, 6, 1)])
def test_lod2d_oracle_matches_reference(shape):
    """diffusion_decay_solver__constant_coefficients_LOD_2D: the z = 0 plane,
    decay split in halves, Dirichlet before each sweep."""
    scn = W.mixed_small(shape=shape, S=2, n_agents=0, seed=sum(shape), bulk=False)
    a = O.oracle_lod2d_run(scn, 3)
    with O.Reference(scn) as ref:
        ref.set_solver(2)
        ref.run(3, 4)
        b = ref.densities()
    assert np.array_equal(a, b)


@pytest.mark.skipif(not REF, reason="compiled reference (oracle/_ref) not built")
def test_gradients_match_reference():
    """compute_all_gradient_vectors (every scenario here uses dx = 10: the
    reference keeps the first 2*dx it sees in static variables)."""
    scn = W.mixed_small(shape=(9, 7, 6), S=3, n_agents=50, seed=5)
    with O.Reference(scn) as ref:
        ref.run(2, 7)  # the reference takes its index jumps from the LOD_3D setup
        p = ref.densities()
        g = ref.gradients()
    assert np.array_equal(O.oracle_gradients(p, scn.shape, scn.mesh.dx), g)
