"""Parity of the CUDA path (through the C ABI) with the reference.

Tolerances: FP64 relative max-norm error per substrate
<= 1e-12 against the oracle/reference; the per-voxel kernels (bulk, cells,
Dirichlet) are bit-exact; FP32 sweeps <= 1e-5.
"""
import numpy as np
import pytest

from biofvm_b200 import STEP_ALL, STEP_BULK, STEP_CELLS, STEP_DIFFUSION, Solver, load_scenario
from biofvm_b200 import workloads as W
from biofvm_b200._abi import FP32_FP64MATH, PATH_AUTO, PATH_DIRECT, PATH_GENERIC, PATH_TMA, BfvmError
from cases import CASES, sha
from conftest import load_golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-5


def rel_err(a, b):
    return O.max_rel_err(a, b)


def run_gpu(scn, steps, flags, fused=True, precision=64, path=PATH_AUTO):
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.set_kernel_path(path)
        if precision != 64:
            sv.set_precision(precision)
        if fused:
            sv.step(scn.dt, steps, flags)
        else:
            for _ in range(steps):
                if flags & STEP_BULK:
                    sv.simulate_bulk_sources_and_sinks(scn.dt)
                if flags & STEP_CELLS:
                    sv.simulate_cell_sources_and_sinks(scn.dt)
                if flags & STEP_DIFFUSION:
                    sv.simulate_diffusion_decay(scn.dt)
        return sv.get_densities()


PATHS = [PATH_AUTO, PATH_TMA, PATH_DIRECT, PATH_GENERIC]
PATH_IDS = ["auto", "tma", "direct", "generic"]


@pytest.mark.parametrize("path", PATHS, ids=PATH_IDS)
@pytest.mark.parametrize("fused", [True, False], ids=["fused", "per_call"])
@pytest.mark.parametrize("name", list(CASES))
def test_golden_cases(name, fused, path):
    build, flags, steps, _ = CASES[name]
    scn = build()
    g = load_golden(name)
    p = run_gpu(scn, steps, flags, fused, path=path)
    assert p.shape == tuple(g["shape"])
    if not flags & STEP_DIFFUSION:
        # per-voxel updates only: same IEEE operations in the same order
        assert sha(p) == str(g["sha"])
        return
    if "p" in g:
        ref = g["p"]
    else:
        ref = O.oracle_run(scn, steps, flags)
        assert sha(ref) == str(g["sha"])
    err = rel_err(p, ref)
    assert np.all(err <= TOL64), err
    assert np.all(np.isfinite(p))


def test_bulk_with_shared_coefficient_rows_is_exact():
    """A bulk region with one rate vector (the sphere of the headline
    workload) runs the kernel that shares coefficient rows between voxels:
    bulk steps alone must equal the oracle's bit for bit, and so must a
    region where every voxel has its own rates (the per-voxel kernel)."""
    scn = W.lod_cube(24, 3, 0, steps=3, seed=101, bulk_radius=80.0, name="bulk_rows")
    assert len(scn.bulk_voxels) > 100
    assert np.array_equal(run_gpu(scn, 3, STEP_BULK), O.oracle_run(scn, 3, STEP_BULK))
    build, _, _, _ = CASES["small_bulk_only"]
    scn2 = build()
    assert np.array_equal(run_gpu(scn2, 3, STEP_BULK), O.oracle_run(scn2, 3, STEP_BULK))


def test_dirichlet_alone_is_exact():
    scn = W.mixed_small(shape=(10, 9, 8), S=3, n_agents=0, seed=41)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.apply_dirichlet_conditions()
        got = sv.get_densities()
    exp = scn.initial_field()
    for v, x in zip(scn.dirichlet_voxels, scn.dirichlet_values):
        exp[v] = x
    assert np.array_equal(got, exp)


def test_dirichlet_update_and_remove():
    """update_dirichlet_node changes the first matching node; remove takes the
    node out of both lists (the reference's remove pops the value list twice,
    BioFVM_microenvironment.cpp:186-187; here the lists stay consistent)."""
    scn = W.mixed_small(shape=(8, 8, 8), S=2, n_agents=0, seed=42, dirichlet=False, bulk=False)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.add_dirichlet_node(5, [1.0, 2.0])
        sv.add_dirichlet_node(77, [3.0, 4.0])
        sv.add_dirichlet_node(300, [5.0, 6.0])
        sv.update_dirichlet_node(77, [7.0, 8.0])
        sv.remove_dirichlet_node(5)
        sv.update_dirichlet_node(400, [9.0, 9.5])  # not present: added
        sv.apply_dirichlet_conditions()
        got = sv.get_densities()
    exp = scn.initial_field()
    exp[77] = [7.0, 8.0]
    exp[300] = [5.0, 6.0]
    exp[400] = [9.0, 9.5]
    assert np.array_equal(got, exp)


def test_voxel_and_agent_access():
    scn = W.mixed_small(shape=(11, 7, 5), S=2, n_agents=50, seed=43)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        vox = np.array([0, 3, 384, 3], np.int64)
        np.testing.assert_array_equal(sv.get_voxel_densities(vox), scn.p0[vox])
        sv.set_voxel_densities([1, 2], [[10.0, 11.0], [12.0, 13.0]])
        p = sv.get_densities()
        assert np.array_equal(p[1:3], [[10.0, 11.0], [12.0, 13.0]])
        out = np.empty((scn.num_agents, scn.S))
        sv.get_agent_densities(out)
        v, _, _ = scn.agent_arrays()
        assert np.array_equal(out, p[v])


def test_bad_arguments_are_reported():
    with Solver(0) as sv:
        sv.resize_space(0, 100, 0, 100, 0, 100, 10)
        with pytest.raises(BfvmError) as e:
            sv.set_agents([1000], [[0.0]], [[1.0]])
        assert "outside" in str(e.value)
        with pytest.raises(BfvmError):
            sv.add_dirichlet_node(-1, [1.0])


def test_non_uniform_mesh_is_rejected_like_the_reference():
    with Solver(0) as sv:
        sv.resize_space(0, 100, 0, 100, 0, 100, 10, 20, 10)
        with pytest.raises(BfvmError) as e:
            sv.simulate_diffusion_decay(0.01)
        assert "uniform Cartesian" in str(e.value)


def test_add_density_keeps_existing_values():
    scn = W.mixed_small(shape=(6, 5, 4), S=2, n_agents=0, seed=44, dirichlet=False, bulk=False)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.add_density(1e3, 0.1)
        p = sv.get_densities()
    assert p.shape == (scn.num_voxels, 3)
    assert np.array_equal(p[:, :2], scn.p0) and np.all(p[:, 2] == 0)


def test_stale_thomas_setup_matches_reference_and_can_be_reset():
    """The reference computes its Thomas coefficients once, from the first
    dt (BioFVM_solvers.cpp:87,172); a later dt only changes bulk/cells."""
    scn = W.mixed_small(shape=(10, 8, 6), S=2, n_agents=0, seed=45, dirichlet=False, bulk=False)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.simulate_diffusion_decay(0.01)
        sv.simulate_diffusion_decay(0.05)  # coefficients still those of dt=0.01
        stale = sv.get_densities()
        sv.set_densities(scn.p0)
        sv.reset_diffusion_setup()
        sv.simulate_diffusion_decay(0.05)
        fresh = sv.get_densities()
    exp = O.oracle_run(scn, 2, 4)
    assert np.all(rel_err(stale, exp) <= TOL64)
    scn5 = W.mixed_small(shape=(10, 8, 6), S=2, n_agents=0, seed=45, dirichlet=False,
                         bulk=False)
    scn5.dt = 0.05
    exp5 = O.oracle_run(scn5, 1, 4)
    assert np.all(rel_err(fresh, exp5) <= TOL64)


def test_plain_50_against_reference_golden():
    """The 50^3 workload end to end (100 fused steps), checked against the
    unmodified reference's output digest through the oracle."""
    scn = W.plain_50()
    p = run_gpu(scn, 100, 7)
    g = load_golden("plain_50")
    ref = O.oracle_run(scn, 100, 7)
    assert sha(ref) == str(g["sha"])
    assert np.all(rel_err(p, ref) <= TOL64)


@pytest.mark.parametrize("path", PATHS, ids=PATH_IDS)
def test_fp32_sweeps_error_bound(path):
    scn = W.lod_cube(48, 4, 2000, steps=20, seed=5, bulk_radius=150.0, name="lod_48")
    ref = O.oracle_run(scn, 20, 7)
    p32 = run_gpu(scn, 20, 7, precision=32, path=path)
    err = rel_err(p32, ref)
    assert np.all(err <= TOL32), err


@pytest.mark.parametrize("path", PATHS, ids=PATH_IDS)
def test_fp32_field_with_fp64_sweeps(path):
    """BFVM_FP32_FP64MATH: only the stored field is rounded to FP32 (once per
    sweep and source update), so after 20 steps the error stays within a few
    hundred FP32 units in the last place (<= 1e-6 relative)."""
    scn = W.lod_cube(48, 4, 2000, steps=20, seed=5, bulk_radius=150.0, name="lod_48")
    ref = O.oracle_run(scn, 20, 7)
    got = run_gpu(scn, 20, 7, precision=FP32_FP64MATH, path=path)
    err = rel_err(got, ref)
    assert np.all(err <= 1e-6), err


@pytest.mark.parametrize("shape,S", [((7, 5, 3), 1), ((13, 11, 9), 3), ((40, 33, 21), 2)])
def test_layouts_without_tma_alignment(shape, S):
    """Row or plane strides that are not 16-byte multiples fall back to the
    register kernel for that axis; mixed paths in one step must agree."""
    scn = W.mixed_small(shape=shape, S=S, n_agents=100, seed=sum(shape))
    ref = O.oracle_run(scn, 3, 7)
    p = run_gpu(scn, 3, 7)
    assert np.all(rel_err(p, ref) <= TOL64)


def test_long_lines_multiple_boxes():
    """Lines longer than one 256-row tensor box (two boxes per tile)."""
    scn = W.mixed_small(shape=(20, 300, 12), S=2, n_agents=200, seed=77)
    ref = O.oracle_run(scn, 2, 7)
    for path in PATHS:
        p = run_gpu(scn, 2, 7, path=path)
        assert np.all(rel_err(p, ref) <= TOL64), path


@pytest.mark.parametrize("shape", [(1024, 2, 3), (3, 1024, 2), (2, 3, 1024)],
                         ids=["x", "y", "z"])
def test_longest_lines(shape):
    """Lines of 1024 points, the longest an axis may have (32 chunks of 32
    points), on every kernel path."""
    scn = W.mixed_small(shape=shape, S=2, n_agents=200, seed=sum(shape) + 1)
    ref = O.oracle_run(scn, 2, 7)
    for path in PATHS:
        p = run_gpu(scn, 2, 7, path=path)
        assert np.all(rel_err(p, ref) <= TOL64), path


@pytest.mark.parametrize("shape,S,kind", [((96, 20, 12), 4, PATH_TMA), ((160, 12, 10), 5, PATH_TMA),
                                          ((96, 20, 12), 1, 0), ((64, 20, 12), 6, 0)],
                         ids=["rows96x4", "rows160x5", "register_S1", "register_n64"])
def test_default_x_kernel(shape, S, kind):
    """Untuned, x sweeps with the row kernel at 32-point chunks when there are
    at least 4 densities and rows of at least 96 points, else with the
    register kernel; either way the step matches the oracle, fused and per
    call."""
    scn = W.mixed_small(shape=shape, S=S, n_agents=300, seed=sum(shape) + S)
    ref = O.oracle_run(scn, 3, 7)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        assert sv.get_sweep_kernel(0) == kind
        if kind:
            assert sv.get_sweep_config(0)[0] == 32
    for fused in (True, False):
        p = run_gpu(scn, 3, 7, fused=fused)
        assert np.all(rel_err(p, ref) <= TOL64), fused


def test_default_x_kernel_follows_added_densities():
    """Densities added after the mesh (the usual driver order) move x to the
    row kernel once there are 4; the step still matches the oracle."""
    scn = W.mixed_small(shape=(128, 10, 8), S=4, n_agents=100, seed=5, dirichlet=False,
                        bulk=False)
    ref = O.oracle_run(scn, 2, 7)
    m = scn.mesh
    with Solver(0) as sv:
        sv.resize_densities(1)
        sv.resize_space(m.x0, m.x1, m.y0, m.y1, m.z0, m.z1, m.dx, m.dy, m.dz)
        assert sv.get_sweep_kernel(0) == 0
        for _ in range(3):
            sv.add_density(0.0, 0.0)
        assert sv.get_sweep_kernel(0) == PATH_TMA
        sv.set_coefficients(scn.D, scn.decay)
        sv.set_densities(scn.p0)
        v, t1, t2 = scn.agent_arrays()
        sv.set_agents(v, t1, t2)
        sv.step(scn.dt, 2, 7)
        p = sv.get_densities()
    assert np.all(rel_err(p, ref) <= TOL64)


LONG_SHAPES = [(2048, 3, 2), (3, 2048, 2), (2, 3, 2048), (4100, 2, 3), (2, 4100, 2),
               (3, 2, 4100), (1025, 5, 4)]


@pytest.mark.parametrize("shape", LONG_SHAPES, ids=["x2048", "y2048", "z2048", "x4100", "y4100",
                                                    "z4100", "x1025"])
@pytest.mark.parametrize("fused", [True, False], ids=["fused", "per_call"])
def test_lines_longer_than_1024_points(shape, fused):
    """Axes past the chunked kernels' 1024 points run one thread per column
    with the reference's own operation sequence: the whole step (bulk,
    agents, Dirichlet nodes) against the oracle."""
    scn = W.mixed_small(shape=shape, S=2, n_agents=300, seed=sum(shape) + 3)
    ref = O.oracle_run(scn, 3, 7)
    p = run_gpu(scn, 3, 7, fused)
    assert np.all(rel_err(p, ref) <= TOL64), rel_err(p, ref)


def test_long_lines_fp32_and_slabs():
    """An FP32 field on a 2048-point axis (FP64 arithmetic along it), and the
    x and y sweeps by slabs of planes with a long x axis."""
    scn = W.mixed_small(shape=(2048, 4, 6), S=3, n_agents=100, seed=41)
    ref = O.oracle_run(scn, 3, 7)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.set_precision(32)
        sv.set_densities(scn.initial_field())
        sv.step(scn.dt, 3)
        assert np.all(rel_err(sv.get_densities(), ref) <= TOL32)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.set_slab_planes(2)
        sv.step(scn.dt, 3)
        assert np.all(rel_err(sv.get_densities(), ref) <= TOL64)


def test_lod2d_plane_of_2048_squared():
    """diffusion_decay_solver__constant_coefficients_LOD_2D on a 2048 x 2048
    plane with Dirichlet nodes: both axes run the long-line kernel, which
    follows the reference's operation sequence, so the plane equals the
    oracle's bit for bit."""
    scn = W.mixed_small(shape=(2048, 2048, 1), S=2, n_agents=0, seed=2048, bulk=False)
    ref = O.oracle_lod2d_run(scn, 2)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        for _ in range(2):
            sv.simulate_diffusion_decay_2d(scn.dt)
        p = sv.get_densities()
    assert np.array_equal(p, ref)


def test_long_lines_tuner_and_adjoint_limits():
    """The sweep tuner leaves a long axis to its one kernel; the adjoint
    refuses lines past 1024 points."""
    scn = W.mixed_small(shape=(1500, 6, 5), S=2, n_agents=50, seed=43)
    ref = O.oracle_run(scn, 2, 7)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.tune_sweeps(scn.dt, 1)
        sv.step(scn.dt, 2)
        assert np.all(rel_err(sv.get_densities(), ref) <= TOL64)
        from biofvm_b200._abi import call
        with pytest.raises(BfvmError) as e:
            call("bfvm_adjoint_forward", sv.handle, scn.dt, 2, 7, 1)
        assert "1024 points" in str(e.value)


@pytest.mark.slow
def test_lod_256_full_size_two_steps():
    """The full 256^3 x 10 workload with 100k agents: two fused steps against
    the oracle, then the exact per-substrate balance of a diffusion-only step."""
    scn = W.lod_256(steps=2)
    p = run_gpu(scn, 2, 7)
    ref = O.oracle_run(scn, 2, 7)
    err = rel_err(p, ref)
    assert np.all(err <= TOL64), err
    # balance: Neumann boundaries, no sources -> total / (1 + dt*decay/3)^3
    with Solver(0) as sv:
        load_scenario(sv, scn)
        rng = np.random.default_rng(0)
        p0 = rng.random((scn.num_voxels, scn.S))
        sv.set_densities(p0)
        sv.step(scn.dt, 1, STEP_DIFFUSION)
        p1 = sv.get_densities()
    c2 = scn.dt * scn.decay / 3.0
    np.testing.assert_allclose(p1.sum(0), p0.sum(0) / (1 + c2) ** 3, rtol=1e-12)


@pytest.mark.parametrize("chunk", [8, 16, 32])
@pytest.mark.parametrize("path", PATHS, ids=PATH_IDS)
def test_chunk_lengths(chunk, path):
    """Every chunk length on every path (the segment lists and the chunk
    tables are rebuilt for it)."""
    scn = W.mixed_small(shape=(40, 36, 30), S=3, n_agents=300, seed=91)
    ref = O.oracle_run(scn, 2, 7)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.set_kernel_path(path)
        for ax in range(3):
            sv.set_sweep_config(ax, chunk, 16 if chunk == 8 else 32)
        sv.step(scn.dt, 2)
        p = sv.get_densities()
    assert np.all(rel_err(p, ref) <= TOL64)


@pytest.mark.parametrize("path", PATHS, ids=PATH_IDS)
@pytest.mark.parametrize("name", ["mixed_full", "mixed_odd", "plain_50"])
def test_sources_fused_into_the_x_sweep(name, path):
    """Bulk and cell updates in the x sweep's prologue give the same field as
    the separate source kernels."""
    build, flags, steps, _ = CASES[name]
    scn = build()
    steps = min(steps, 10)
    ref = O.oracle_run(scn, steps, flags)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.set_kernel_path(path)
        sv.set_fuse_sources(True)
        sv.step(scn.dt, steps, flags)
        p = sv.get_densities()
    assert np.all(rel_err(p, ref) <= TOL64)


@pytest.mark.parametrize("path", PATHS, ids=PATH_IDS)
@pytest.mark.parametrize("shape", [(17, 13, 1), (9, 11, 3), (64, 48, 1)])
def test_lod2d(shape, path):
    """diffusion_decay_solver__constant_coefficients_LOD_2D on the GPU: the
    z = 0 plane only, decay split in halves, Dirichlet before each sweep."""
    scn = W.mixed_small(shape=shape, S=2, n_agents=0, seed=sum(shape), bulk=False)
    ref = O.oracle_lod2d_run(scn, 3)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.set_kernel_path(path)
        for _ in range(3):
            sv.simulate_diffusion_decay_2d(scn.dt)
        p = sv.get_densities()
    assert np.all(rel_err(p, ref) <= TOL64)


X_LINE_CASES = [
    # more densities x chunks per row than the row kernel's tiles hold
    # (S * chunks > 512), so the x sweep runs on the line kernel; Dirichlet
    # nodes before and after it
    ((520, 6, 4), 32, False),  # 17 chunks of 32 points: 8-density tiles
    ((400, 5, 3), 48, False),  # 13 chunks: 16-density tiles
    ((600, 8, 1), 32, True),   # LOD_2D plane
]


@pytest.mark.parametrize("shape,S,two_d", X_LINE_CASES)
def test_x_sweep_on_the_line_kernel(shape, S, two_d):
    scn = W.mixed_small(shape=shape, S=S, n_agents=40, seed=sum(shape) + S, bulk=True)
    steps = 2
    ref = O.oracle_lod2d_run(scn, steps) if two_d else O.oracle_run(scn, steps, STEP_ALL)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.set_kernel_path(PATH_TMA)
        if two_d:
            for _ in range(steps):
                sv.simulate_diffusion_decay_2d(scn.dt)
        else:
            sv.step(scn.dt, steps, STEP_ALL)
        p = sv.get_densities()
    assert np.all(rel_err(p, ref) <= TOL64)


def test_line_sweeps_after_a_resize_that_keeps_the_allocation():
    """The y and z sweeps' tensor maps follow the mesh: a smaller mesh in the
    same device allocation, then a LOD_2D step and 3-D steps on one solver,
    match fresh solvers."""
    big = W.mixed_small(shape=(40, 36, 30), S=2, n_agents=0, seed=81, bulk=False)
    small = W.mixed_small(shape=(24, 20, 16), S=2, n_agents=30, seed=82)
    with Solver(0) as sv:
        sv.set_kernel_path(PATH_TMA)
        load_scenario(sv, big)
        sv.step(big.dt, 2, STEP_ALL)
        load_scenario(sv, small)
        sv.step(small.dt, 3, STEP_ALL)
        p = sv.get_densities()
    ref = O.oracle_run(small, 3, STEP_ALL)
    assert np.all(rel_err(p, ref) <= TOL64)
    with Solver(0) as sv:
        sv.set_kernel_path(PATH_TMA)
        load_scenario(sv, small)
        sv.simulate_diffusion_decay_2d(small.dt)
        sv.step(small.dt, 2, STEP_ALL)
        p = sv.get_densities()
    with Solver(0) as sv:
        sv.set_kernel_path(PATH_GENERIC)
        load_scenario(sv, small)
        sv.simulate_diffusion_decay_2d(small.dt)
        sv.step(small.dt, 2, STEP_ALL)
        q = sv.get_densities()
    assert np.all(rel_err(p, q) <= TOL64)


def test_agents_sharing_voxels_keep_list_order():
    """Hundreds of agents in a handful of voxels: the implicit per-agent update
    does not commute, so only the reference's list order reproduces it
    (bit-exact, cells step alone)."""
    scn = W.mixed_small(shape=(3, 2, 2), S=3, n_agents=700, seed=61, dirichlet=False,
                        bulk=False)
    ref = O.oracle_run(scn, 2, STEP_CELLS)
    for fused in (True, False):
        assert np.array_equal(run_gpu(scn, 2, STEP_CELLS, fused=fused), ref)


def test_agents_replaced_between_steps():
    """set_agents replaces the whole list (more, fewer, none)."""
    a = W.mixed_small(shape=(12, 9, 7), S=2, n_agents=400, seed=62)
    b = W.mixed_small(shape=(12, 9, 7), S=2, n_agents=90, seed=63)
    with Solver(0) as sv:
        load_scenario(sv, a)
        sv.step(a.dt, 1, STEP_CELLS)
        sv.set_agents(*b.agent_arrays())
        sv.step(a.dt, 1, STEP_CELLS)
        sv.set_agents(np.zeros(0, np.int64), np.zeros((0, 2)), np.zeros((0, 2)))
        sv.step(a.dt, 1, STEP_CELLS)
        got = sv.get_densities()
    lib = O.load_oracle()
    exp = a.initial_field()
    for scn in (a, b):
        v, t1, t2 = (np.ascontiguousarray(x) for x in scn.agent_arrays())
        lib.or_cells(v.size, a.S, O._d(exp), O._l(v), O._d(t1), O._d(t2))
    assert np.array_equal(got, exp)


def test_add_density_after_agents_gives_identity_update():
    """add_density widens every agent's constants with temp1 = 0, temp2 = 1
    (secretion and uptake of a new density start at zero)."""
    scn = W.mixed_small(shape=(8, 6, 5), S=2, n_agents=120, seed=64, dirichlet=False,
                        bulk=False)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.add_density(1e3, 0.1)
        sv.set_voxel_densities(np.arange(scn.num_voxels), np.c_[scn.p0, np.full(scn.num_voxels, 2.5)])
        sv.step(scn.dt, 2, STEP_CELLS)
        got = sv.get_densities()
    ref = O.oracle_run(scn, 2, STEP_CELLS)
    assert np.array_equal(got[:, :2], ref) and np.all(got[:, 2] == 2.5)


@pytest.mark.parametrize("precision", [64, 32])
def test_gradients_bit_exact_on_the_device_field(precision):
    """Central differences of the device field, bit for bit as the reference's
    compute_all_gradient_vectors computes them on the same field; the
    components at axis ends keep their earlier values across calls."""
    scn = W.mixed_small(shape=(11, 9, 1), S=2, n_agents=40, seed=66)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        if precision != 64:
            sv.set_precision(precision)
        sv.step(scn.dt, 2)
        sv.compute_all_gradient_vectors()
        g1 = sv.get_gradient_vectors()
        p1 = sv.get_densities()
        sv.step(scn.dt, 1)
        sv.compute_all_gradient_vectors()
        g2 = sv.get_gradient_vectors()
        p2 = sv.get_densities()
    e1 = O.oracle_gradients(p1, scn.shape, scn.mesh.dx)
    assert np.array_equal(g1, e1)
    assert np.array_equal(g2, O.oracle_gradients(p2, scn.shape, scn.mesh.dx, g=e1))
    assert np.all(g2[:, :, 2] == 0)  # nz = 1: no z neighbours anywhere


@pytest.mark.parametrize("shape", [(24, 20, 16), (70, 33, 9)])
def test_sweep_tuner_keeps_the_field_and_the_results(shape):
    """bfvm_tune_sweeps times every kernel of every axis on the solver's own
    field: the field must come back unchanged, and steps with the chosen
    kernels must still match the oracle."""
    scn = W.mixed_small(shape=shape, S=3, n_agents=300, seed=sum(shape))
    with Solver(0) as sv:
        load_scenario(sv, scn)
        before = sv.get_densities()
        chosen = sv.tune_sweeps(scn.dt, 2)
        assert np.array_equal(sv.get_densities(), before)
        assert len(chosen) == 3
        sv.step(scn.dt, 3)
        got = sv.get_densities()
    assert np.all(rel_err(got, O.oracle_run(scn, 3, 7)) <= TOL64), chosen


@pytest.mark.parametrize("shape,S", [((256, 12, 9), 10), ((128, 10, 6), 8), ((224, 7, 5), 10),
                                     ((128, 12, 7), 4), ((256, 6, 5), 16)])
def test_row_kernel_builds_for_one_density_count(shape, S):
    """The x row kernel compiled for exactly S densities (constant offsets
    along the rows), with interleaved and with planar chunk tables: the same
    arithmetic as the general build, so bit-identical results, and within
    the oracle bar; the plan reports the build it runs."""
    scn = W.mixed_small(shape=shape, S=S, n_agents=500, seed=sum(shape) + 3 * S)
    ref = O.oracle_run(scn, 3, 7)
    got = {}
    for build in (0, 1, 2):
        with Solver(0) as sv:
            load_scenario(sv, scn)
            sv.set_kernel_path(PATH_TMA)
            sv.set_sweep_config(0, 32, 16, 1)
            sv.set_row_build(build)
            sv.step(scn.dt, 3)
            assert sv.get_row_build() == (build, build)
            got[build] = sv.get_densities()
        assert np.all(rel_err(got[build], ref) <= TOL64), build
    assert np.array_equal(got[1], got[0]) and np.array_equal(got[2], got[0])


def test_row_build_falls_back_where_it_does_not_apply():
    """Builds 1 and 2 exist for 4, 8, 10 and 16 densities only: with 6
    densities the general build runs (effective 0) and the sweep still meets
    the oracle; a solver starts with build 2 requested."""
    scn = W.mixed_small(shape=(128, 9, 5), S=6, n_agents=300, seed=77)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        assert sv.get_row_build()[0] == 2
        sv.set_kernel_path(PATH_TMA)
        sv.set_sweep_config(0, 32, 16, 1)
        sv.set_row_build(2)
        sv.step(scn.dt, 3)
        assert sv.get_row_build() == (2, 0)
        got = sv.get_densities()
        with pytest.raises(BfvmError):
            sv.set_row_build(3)
    assert np.all(rel_err(got, O.oracle_run(scn, 3, 7)) <= TOL64)


@pytest.mark.parametrize("shape,S", [((256, 12, 9), 10), ((160, 20, 7), 4), ((96, 9, 5), 7)])
def test_row_kernel_with_three_stage_ring(shape, S):
    """The x row kernel with a ring of three tiles (and whole warps per
    chunk) against the oracle, next to the two-tile ring, and compiled for
    two blocks per SM at 32-point chunks."""
    scn = W.mixed_small(shape=shape, S=S, n_agents=500, seed=sum(shape) + S)
    ref = O.oracle_run(scn, 3, 7)
    for stages, minb in ((2, 1), (3, 1), (2, 2)):
        with Solver(0) as sv:
            load_scenario(sv, scn)
            sv.set_kernel_path(PATH_TMA)
            if minb == 2:
                sv.set_sweep_config(0, 32, 16, 2)
            sv.set_row_stages(stages)
            sv.step(scn.dt, 3)
            assert sv.get_sweep_config(0)[3] == stages
            assert np.all(rel_err(sv.get_densities(), ref) <= TOL64), (stages, minb)


# ---- x and y sweeps by slabs of z planes (bfvm_set_slab_planes) ----

def _run_slabs(scn, steps, planes, path=PATH_AUTO, flags=7, precision=64):
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.set_kernel_path(path)
        if precision != 64:
            sv.set_precision(precision)
        sv.set_slab_planes(planes)
        assert sv.get_slab_planes() == planes
        sv.set_grid_steps(False)  # whole-axis runs use the sweep kernels too
        sv.step(scn.dt, steps, flags)
        return sv.get_densities()


@pytest.mark.parametrize("path", [PATH_AUTO, PATH_TMA, PATH_GENERIC], ids=["auto", "tma", "generic"])
@pytest.mark.parametrize("planes", [1, 2, 3, 7, 29])
def test_slabs_reproduce_whole_axis_sweeps(planes, path):
    """The same kernels on every line, only in another order: identical
    fields (Dirichlet nodes, bulk and agents included; 30 planes, so the last
    slab is partial for most thicknesses)."""
    scn = W.mixed_small(shape=(33, 21, 30), S=3, n_agents=400, seed=95)
    whole = _run_slabs(scn, 3, 0, path)
    got = _run_slabs(scn, 3, planes, path)
    assert np.array_equal(got, whole)
    assert np.all(rel_err(got, O.oracle_run(scn, 3, 7)) <= TOL64)


@pytest.mark.parametrize("planes", [2, 5])
def test_slabs_on_the_direct_path_and_fp32(planes):
    """Slabs through the direct kernel, and in FP32: the same fields as the
    whole-axis sweeps."""
    scn = W.mixed_small(shape=(40, 24, 17), S=2, n_agents=200, seed=96)
    got = _run_slabs(scn, 3, planes, PATH_DIRECT)
    assert np.array_equal(got, _run_slabs(scn, 3, 0, PATH_DIRECT))
    assert np.all(rel_err(got, O.oracle_run(scn, 3, 7)) <= TOL64)
    got32 = _run_slabs(scn, 3, planes, PATH_AUTO, precision=32)
    whole32 = _run_slabs(scn, 3, 0, PATH_AUTO, precision=32)
    assert np.array_equal(got32, whole32)


def test_slabs_leave_lod2d_alone_and_reject_negative():
    scn = W.mixed_small(shape=(17, 13, 1), S=2, n_agents=0, seed=97, bulk=False)
    ref = O.oracle_lod2d_run(scn, 3)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.set_slab_planes(1)
        for _ in range(3):
            sv.simulate_diffusion_decay_2d(scn.dt)
        assert np.all(rel_err(sv.get_densities(), ref) <= TOL64)
        with pytest.raises(BfvmError):
            sv.set_slab_planes(-1)


def test_tuner_picks_a_slab_thickness():
    scn = W.mixed_small(shape=(48, 40, 64), S=4, n_agents=500, seed=98)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        before = sv.get_densities()
        sv.tune_sweeps(scn.dt, 2)
        assert np.array_equal(sv.get_densities(), before)
        k = sv.get_slab_planes()
        assert k in (0, 2, 4, 8, 16, 32)
        sv.step(scn.dt, 3)
        got = sv.get_densities()
    assert np.all(rel_err(got, O.oracle_run(scn, 3, 7)) <= TOL64), k


# ---- error path of the bounded waits (no GPU fault involved) ----

def test_bounded_wait_gives_up_and_the_device_stays_usable():
    """A kernel waits, with the sweeps' bounded wait, on a barrier that
    nothing completes: it must give up after the limit, report it through the
    status word, and leave the context usable for a normal step."""
    from biofvm_b200.solver import selftest_bounded_wait

    gave_up, ms = selftest_bounded_wait(0, 3_000_000)  # 3 ms
    assert gave_up
    assert 2.5 <= ms < 1000.0, ms
    scn = W.mixed_small(shape=(20, 18, 16), S=2, n_agents=100, seed=99)
    assert np.all(rel_err(run_gpu(scn, 2, 7, path=PATH_TMA), O.oracle_run(scn, 2, 7)) <= TOL64)
    with pytest.raises(BfvmError):
        selftest_bounded_wait(0, 10)  # below the 1 us floor


# ---- host threads, one solver each ----

_THREADS_CHILD = r"""
import sys, threading
sys.path.insert(0, sys.argv[1])
import numpy as np
from biofvm_b200 import Solver, load_scenario
from biofvm_b200 import workloads as W
from biofvm_b200._abi import PATH_AUTO, PATH_TMA
scns = [W.mixed_small(shape=(30 + 4 * i, 24, 20), S=2, n_agents=150, seed=200 + i) for i in range(4)]
out = [None] * 4
errs = []
go = threading.Barrier(4)
def work(i):
    try:
        with Solver(0) as sv:
            load_scenario(sv, scns[i])
            sv.set_kernel_path(PATH_TMA if i % 2 else PATH_AUTO)
            go.wait()
            sv.step(scns[i].dt, 3)
            out[i] = sv.get_densities()
    except Exception as e:
        errs.append(repr(e))
ts = [threading.Thread(target=work, args=(i,)) for i in range(4)]
[t.start() for t in ts]
[t.join() for t in ts]
assert not errs, errs
np.savez(sys.argv[2], *out)
"""


def test_host_threads_each_with_a_solver(tmp_path):
    """Four host threads, each with its own solver, step at the same time
    from a fresh process (so the library's first-use caches are filled
    concurrently); every field must match the oracle."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = tmp_path / "fields.npz"
    r = subprocess.run([sys.executable, "-c", _THREADS_CHILD, root, str(out)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    got = np.load(out)
    for i in range(4):
        scn = W.mixed_small(shape=(30 + 4 * i, 24, 20), S=2, n_agents=150, seed=200 + i)
        assert np.all(rel_err(got[f"arr_{i}"], O.oracle_run(scn, 3, 7)) <= TOL64), i


# ---- whole steps of a small field in one thread-block cluster ----

@pytest.mark.parametrize("case", [
    dict(shape=(50, 50, 50), S=1, n_agents=1000, dirichlet=True, bulk=False),
    dict(shape=(33, 17, 9), S=4, n_agents=400, dirichlet=True, bulk=True),
    dict(shape=(40, 40, 40), S=3, n_agents=2000, dirichlet=False, bulk=True),
    dict(shape=(7, 1, 5), S=2, n_agents=50, dirichlet=True, bulk=True),
    dict(shape=(64, 3, 64), S=2, n_agents=100, dirichlet=True, bulk=True),
], ids=["50cube", "odd", "40cube-S3", "thin", "64-lines"])
def test_cluster_steps_equal_the_reference_bit_for_bit(case):
    """bfvm_step on a field that fits a cluster runs every step in one
    launch, with the reference's own operation sequence: the field must equal
    the oracle's (the reference restated in C) exactly."""
    scn = W.mixed_small(seed=sum(case["shape"]) + case["S"], **case)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.set_cluster_steps(True)
        assert sv.get_cluster_steps() > 0
        sv.step(scn.dt, 4)
        p = sv.get_densities()
    assert np.array_equal(p, O.oracle_run(scn, 4, 7))


def test_cluster_steps_agree_with_the_sweep_kernels_and_can_be_turned_off():
    scn = W.plain_50(steps=10)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.set_cluster_steps(True)
        blocks = sv.get_cluster_steps()
        assert blocks in (1, 2, 4, 8)
        sv.step(scn.dt, 10)
        a = sv.get_densities()
        sv.set_densities(scn.initial_field())
        sv.set_cluster_steps(False)
        assert sv.get_cluster_steps() == 0
        sv.step(scn.dt, 10)
        b = sv.get_densities()
        sv.set_cluster_steps(True)
        sv.set_kernel_path(PATH_TMA)
        assert sv.get_cluster_steps() == 0  # only under the AUTO path
    assert np.all(rel_err(a, b) <= TOL64)


def test_cluster_steps_not_used_for_large_fields():
    with Solver(0) as sv:
        sv.set_cluster_steps(True)
        sv.resize_densities(2)
        sv.resize_space(0, 650, 0, 640, 0, 640, 10)  # 65 points along x
        assert sv.get_cluster_steps() == 0
        sv.resize_space(0, 640, 0, 640, 0, 640, 10)  # 64^3 x 2: 4 MB
        assert sv.get_cluster_steps() == 0
        sv.resize_space(0, 400, 0, 400, 0, 400, 10)  # 40^3 x 2: 1 MB
        assert sv.get_cluster_steps() > 0


GRID_CASES = [
    dict(shape=(50, 50, 50), S=1, n_agents=1000, dirichlet=True, bulk=True),
    dict(shape=(23, 17, 31), S=3, n_agents=400, dirichlet=True, bulk=True),
    dict(shape=(40, 40, 40), S=5, n_agents=2000, dirichlet=True, bulk=True),
    dict(shape=(64, 3, 64), S=2, n_agents=100, dirichlet=True, bulk=True),
    dict(shape=(1, 64, 2), S=4, n_agents=50, dirichlet=False, bulk=True),
]
GRID_IDS = ["50cube", "odd", "40cube-S5", "thin", "one-point-x"]


@pytest.mark.parametrize("case", GRID_CASES, ids=GRID_IDS)
def test_grid_steps_match_the_oracle_and_the_sweep_kernels(case):
    """bfvm_step on a small FP64 field runs every step in one cooperative
    launch (chunked lines per tile, Dirichlet values applied as chunks load,
    sources in a phase of their own):
    within 1e-12 of the oracle and of the sweep kernels, agents sharing
    voxels included."""
    scn = W.mixed_small(seed=sum(case["shape"]) + 3 * case["S"], **case)
    ref = O.oracle_run(scn, 4, 7)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        assert sv.get_grid_steps() > 0  # the default for a field this small
        sv.step(scn.dt, 4)
        a = sv.get_densities()
        sv.set_densities(scn.initial_field())
        sv.set_grid_steps(False)
        assert sv.get_grid_steps() == 0
        sv.step(scn.dt, 4)
        b = sv.get_densities()
    assert np.all(rel_err(a, ref) <= TOL64)
    assert np.all(rel_err(a, b) <= TOL64)


@pytest.mark.parametrize("flags", [STEP_DIFFUSION, STEP_BULK | STEP_DIFFUSION,
                                   STEP_CELLS | STEP_DIFFUSION],
                         ids=["diffusion", "bulk+diffusion", "cells+diffusion"])
def test_grid_steps_with_some_parts_of_the_step(flags):
    scn = W.mixed_small(shape=(30, 20, 10), S=2, n_agents=300, seed=91)
    ref = O.oracle_run(scn, 3, flags)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.set_grid_steps(True)
        assert sv.get_grid_steps() > 0
        sv.step(scn.dt, 3, flags)
        p = sv.get_densities()
    assert np.all(rel_err(p, ref) <= TOL64)


def test_grid_steps_follow_changes_between_calls():
    """Agents, bulk rates and Dirichlet nodes changed between bfvm_step calls
    are seen by the next cooperative launch (its voxel maps are rebuilt per
    call)."""
    scn = W.mixed_small(shape=(24, 20, 16), S=2, n_agents=200, seed=92)
    scn2 = W.mixed_small(shape=(24, 20, 16), S=2, n_agents=300, seed=93)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.set_grid_steps(True)
        assert sv.get_grid_steps() > 0
        sv.step(scn.dt, 2)
        mid = sv.get_densities()
        v, t1, t2 = scn2.agent_arrays()
        sv.set_agents(v, t1, t2)
        sv.set_bulk_rates_sparse(scn2.bulk_voxels, scn2.bulk_supply, scn2.bulk_target,
                                 scn2.bulk_uptake)
        sv.step(scn.dt, 2)
        p = sv.get_densities()
    scn2.p0 = mid
    scn2.dirichlet_voxels, scn2.dirichlet_values = scn.dirichlet_voxels, scn.dirichlet_values
    scn2.D, scn2.decay = scn.D, scn.decay
    assert np.all(rel_err(p, O.oracle_run(scn2, 2, 7)) <= TOL64)


def test_grid_steps_eligibility():
    with Solver(0) as sv:
        sv.resize_densities(1)
        sv.resize_space(0, 500, 0, 500, 0, 500, 10)  # 50^3 x 1 (fits a cluster)
        assert sv.get_grid_steps() > 0  # on by default
        sv.set_cluster_steps(True)  # the bit-exact cluster mode comes first
        assert sv.get_cluster_steps() > 0 and sv.get_grid_steps() == 0
        sv.set_cluster_steps(False)
        sv.resize_densities(2)
        sv.set_kernel_path(PATH_TMA)  # only under the AUTO path
        assert sv.get_grid_steps() == 0
        sv.set_kernel_path(PATH_AUTO)
        sv.set_precision(32)  # FP64 only
        assert sv.get_grid_steps() == 0
        sv.set_precision(64)
        sv.resize_space(0, 650, 0, 640, 0, 640, 10)  # 65 points along x
        assert sv.get_grid_steps() == 0
        sv.resize_densities(3)
        sv.resize_space(0, 640, 0, 640, 0, 640, 10)  # 64^3 x 3 > 2^19
        assert sv.get_grid_steps() == 0
        sv.resize_densities(2)
        sv.resize_space(0, 640, 0, 640, 0, 640, 10)  # 64^3 x 2 = 2^19
        assert sv.get_grid_steps() > 0
        sv.set_grid_steps(False)
        assert sv.get_grid_steps() == 0


def test_add_density_after_the_setup_matches_a_fresh_solver():
    """After a step (Thomas setup done), add_density rebuilds the tables for
    the new count: stepping on equals a solver that had every density from
    the start (bit for bit, same kernels)."""
    scn = W.mixed_small(shape=(20, 18, 16), S=2, n_agents=0, seed=46, dirichlet=False,
                        bulk=False)
    D3, l3 = 3e4, 0.2
    with Solver(0) as a, Solver(0) as b:
        load_scenario(a, scn)
        a.step(scn.dt, 2)
        a.add_density(D3, l3)
        p = a.get_densities()
        p[:, 2] = np.linspace(0.0, 1.0, p.shape[0])
        a.set_densities(p)
        b.resize_densities(3)
        m = scn.mesh
        b.resize_space(m.x0, m.x1, m.y0, m.y1, m.z0, m.z1, m.dx, m.dy, m.dz)
        b.set_coefficients(np.append(scn.D, D3), np.append(scn.decay, l3))
        b.set_densities(p)
        for sv in (a, b):
            sv.set_cluster_steps(False)
            sv.step(scn.dt, 3)
        assert np.array_equal(a.get_densities(), b.get_densities())
