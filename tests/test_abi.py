"""The C-ABI library: it loads, exports exactly what include/bfvm.h declares,
and its error path works without a GPU (no compute call is made here)."""
import ctypes
import os
import re

import numpy as np
import pytest

from biofvm_b200 import _abi
from biofvm_b200.mesh import CartesianMesh, agent_constants, nodes_from_spacing
from oracle import oracle as O

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "bfvm.h")).read()
    return sorted(set(re.findall(r"BFVM_API\s+[\w\s\*]*?\b(bfvm_\w+)\s*\(", text)))


def exported_symbols(path):
    import subprocess

    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_library_exports_every_declared_symbol():
    lib = _abi.load_library()
    names = header_symbols()
    assert len(names) >= 35
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_abi.SIGNATURES), "bindings and header disagree"
    exported = {s for s in exported_symbols(_abi.LIB_PATH) if s.startswith("bfvm_")}
    assert exported == set(names)


def test_error_path_without_device():
    lib = _abi.load_library()
    assert lib.bfvm_version() >= 100
    # a null handle is rejected before any device work
    rc = lib.bfvm_synchronize(None)
    assert rc == _abi.BFVM_ERR_ARG
    assert b"null solver handle" in lib.bfvm_last_error()
    rc = lib.bfvm_create(None, 0)
    assert rc == _abi.BFVM_ERR_ARG


@pytest.mark.parametrize("box,d", [((0, 1000), 20.0), ((-500, 500), 30.0), ((0, 2560), 10.0),
                                   ((0.5, 7.25), 0.33), ((-3, 3), 2.0)])
def test_node_counts_match_oracle(box, d):
    lib = O.load_oracle()
    assert nodes_from_spacing(box[0], box[1], d) == lib.or_nodes_from_spacing(box[0], box[1], d)


def test_nearest_voxel_and_agent_constants_match_oracle():
    rng = np.random.default_rng(0)
    m = CartesianMesh(-100.0, 230.0, 0.0, 90.0, -5.0, 45.0, 10.0, 10.0, 10.0)
    pts = np.column_stack([rng.uniform(-120, 250, 500), rng.uniform(-10, 100, 500),
                           rng.uniform(-10, 60, 500)])
    got = m.nearest_voxel_index(pts)
    lib = O.load_oracle()
    box = np.array([m.x0, m.y0, m.z0])
    exp = [lib.or_nearest_voxel(O._d(box), m.dx, m.dy, m.dz, m.nx, m.ny, m.nz, *map(float, p))
           for p in pts]
    assert np.array_equal(got, np.array(exp))
    S = 3
    sec, sat, up = (rng.uniform(0, 5, (40, S)) for _ in range(3))
    vol = rng.uniform(100, 5000, 40)
    t1, t2 = agent_constants(0.01, vol, m.dV, sec, sat, up)
    for a in range(40):
        r1, r2 = np.empty(S), np.empty(S)
        lib.or_agent_constants(S, 0.01, float(vol[a]), m.dV, O._d(np.ascontiguousarray(sec[a])),
                               O._d(np.ascontiguousarray(sat[a])),
                               O._d(np.ascontiguousarray(up[a])), O._d(r1), O._d(r2))
        assert np.array_equal(t1[a], r1) and np.array_equal(t2[a], r2)


@pytest.mark.skipif(not O.reference_available(), reason="compiled reference not built")
def test_mesh_matches_reference():
    from biofvm_b200 import workloads as W

    for shape in ((5, 6, 7), (1, 9, 2), (40, 3, 3)):
        scn = W.mixed_small(shape=shape, S=2, n_agents=0, seed=1, dx=7.5)
        with O.Reference(scn) as ref:
            nxyz, geom = ref.mesh_info()
        assert nxyz[:3] == scn.mesh.shape
        assert geom[3] == scn.mesh.dV
        assert nxyz[4] == int(scn.mesh.uniform)
