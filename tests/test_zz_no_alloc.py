"""bfvm_get_voxel_densities_noalloc: the voxel-density gather for callers that
can't call cudaMalloc (it stages its data in a fixed file-scope device array
instead of allocating).  Collected last on purpose: a failure here leaves
every other test already run.  Calls the C ABI directly and compares with the
allocating bfvm_get_voxel_densities, on two calls in a row."""
import numpy as np
import pytest

from biofvm_b200 import Solver, load_scenario
from biofvm_b200 import workloads as W
from biofvm_b200._abi import BFVM_ERR_ARG, BFVM_OK, dptr, load_library, lptr

pytestmark = pytest.mark.gpu

TOL64 = 1e-12  # the FP64 parity tolerance of the other GPU tests


def test_noalloc_gather_matches_the_allocating_gather():
    lib = load_library()
    scn = W.mixed_small(shape=(30, 20, 10), S=3, n_agents=200, seed=5)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.step(scn.dt, 2)
        for call, size in enumerate((1500, 700)):  # two calls in a row
            rng = np.random.default_rng(call + 1)
            vox = np.ascontiguousarray(rng.integers(0, scn.num_voxels, size), np.int64)
            expected = sv.get_voxel_densities(vox)
            got = np.full_like(expected, np.nan)
            rc = lib.bfvm_get_voxel_densities_noalloc(sv.handle, vox.size, lptr(vox), dptr(got))
            assert rc == BFVM_OK, lib.bfvm_last_error()
            err = np.abs(got - expected).max(axis=0) / np.maximum(np.abs(expected).max(axis=0),
                                                                  1e-300)
            assert np.all(err <= TOL64), (call, err)
            sv.step(scn.dt, 1)  # the field changes between the two calls


def test_noalloc_gather_rejects_sizes_beyond_its_scratch():
    lib = load_library()
    with Solver(0) as sv:
        sv.resize_densities(4)
        sv.resize_space(0, 1000, 0, 1000, 0, 1000, 10)
        vox = np.zeros(200_000, np.int64)  # 200k x (8 + 32) bytes > 4 MiB
        out = np.empty((vox.size, 4))
        rc = lib.bfvm_get_voxel_densities_noalloc(sv.handle, vox.size, lptr(vox), dptr(out))
        assert rc == BFVM_ERR_ARG
        assert b"static scratch" in lib.bfvm_last_error()


def test_noalloc_gather_in_fp32_matches_the_allocating_gather():
    """The FP32 field goes through the same static array (the gather widens
    to FP64); both gathers read the same FP32 values, so they agree exactly."""
    lib = load_library()
    scn = W.mixed_small(shape=(24, 18, 12), S=4, n_agents=150, seed=9)
    with Solver(0) as sv:
        load_scenario(sv, scn)
        sv.set_precision(32)
        sv.set_densities(scn.initial_field())
        sv.step(scn.dt, 2)
        for call, size in enumerate((900, 2500)):
            rng = np.random.default_rng(call + 11)
            vox = np.ascontiguousarray(rng.integers(0, scn.num_voxels, size), np.int64)
            expected = sv.get_voxel_densities(vox)
            got = np.full_like(expected, np.nan)
            rc = lib.bfvm_get_voxel_densities_noalloc(sv.handle, vox.size, lptr(vox), dptr(got))
            assert rc == BFVM_OK, lib.bfvm_last_error()
            assert np.array_equal(got, expected), call
            sv.step(scn.dt, 1)


def test_noalloc_gather_at_exactly_the_scratch_size():
    """3 densities: 131072 voxels take 1 MiB of voxel list (already a
    multiple of 256 bytes) + 3 MiB of values = the whole 4 MiB; one voxel
    more does not fit and is refused."""
    lib = load_library()
    with Solver(0) as sv:
        sv.resize_densities(3)
        sv.resize_space(0, 1000, 0, 1000, 0, 1000, 10)  # 100^3 voxels
        rng = np.random.default_rng(3)
        sv.set_densities(rng.random((sv.num_voxels, 3)))
        vox = np.ascontiguousarray(rng.integers(0, sv.num_voxels, 131072), np.int64)
        expected = sv.get_voxel_densities(vox)
        got = np.full_like(expected, np.nan)
        rc = lib.bfvm_get_voxel_densities_noalloc(sv.handle, vox.size, lptr(vox), dptr(got))
        assert rc == BFVM_OK, lib.bfvm_last_error()
        assert np.array_equal(got, expected)
        vox1 = np.ascontiguousarray(np.append(vox, 0), np.int64)
        out1 = np.empty((vox1.size, 3))
        rc = lib.bfvm_get_voxel_densities_noalloc(sv.handle, vox1.size, lptr(vox1), dptr(out1))
        assert rc == BFVM_ERR_ARG
        assert b"static scratch" in lib.bfvm_last_error()


def test_noalloc_gather_refuses_a_count_whose_byte_size_would_wrap():
    """count = 2^61: count * 8 wraps to 0 in 64 bits.  The count is bounded
    before any product of it, so the call is refused without reading the
    (one-element) host arrays past their end."""
    lib = load_library()
    with Solver(0) as sv:
        sv.resize_densities(2)
        sv.resize_space(0, 100, 0, 100, 0, 100, 10)
        vox = np.zeros(1, np.int64)
        out = np.empty((1, 2))
        rc = lib.bfvm_get_voxel_densities_noalloc(sv.handle, 2 ** 61, lptr(vox), dptr(out))
        assert rc == BFVM_ERR_ARG
        assert b"static scratch" in lib.bfvm_last_error()
