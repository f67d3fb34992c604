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
