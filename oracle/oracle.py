"""Test infrastructure only: Python drivers of the two CPU checkers.

* ``oracle_*`` call liboracle.so, the plain-C restatement of the reference's
  transport step (bfvm_oracle.c; single thread, no FMA).
* ``reference_*`` call oracle/_ref/libbiofvm_ref*.so, the UNMODIFIED BioFVM
  sources compiled by oracle/Makefile, through the harness in ref_capi.cpp.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only to check or to time the reference; the product never does.
"""
from __future__ import annotations

import ctypes
import os
import time
from ctypes import POINTER, c_double, c_int, c_int64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_LIBS = {"core2": os.path.join(REF_DIR, "libbiofvm_ref.so"),
            "v3": os.path.join(REF_DIR, "libbiofvm_ref_v3.so")}

_DP = POINTER(c_double)
_LP = POINTER(c_int64)
_IP = POINTER(c_int)

_oracle = None
_refs: dict[str, ctypes.CDLL] = {}


def _d(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_DP)


def _l(a):
    if a is None:
        return None
    assert a.dtype == np.int64 and a.flags.c_contiguous
    return a.ctypes.data_as(_LP)


def load_oracle() -> ctypes.CDLL:
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_LIB):
            raise ImportError(f"{ORACLE_LIB} missing: run `make -C oracle oracle`")
        lib = ctypes.CDLL(ORACLE_LIB)
        lib.or_nodes_from_spacing.restype = c_int
        lib.or_nodes_from_spacing.argtypes = [c_double, c_double, c_double]
        lib.or_nearest_voxel.restype = c_int64
        lib.or_nearest_voxel.argtypes = [_DP, c_double, c_double, c_double, c_int, c_int, c_int,
                                         c_double, c_double, c_double]
        lib.or_thomas_setup.restype = None
        lib.or_thomas_setup.argtypes = [c_int, c_int, c_double, c_double, _DP, _DP, _DP, _DP, _DP]
        lib.or_thomas_setup_2d.restype = None
        lib.or_thomas_setup_2d.argtypes = [c_int, c_int, c_double, c_double, _DP, _DP, _DP, _DP,
                                           _DP]
        lib.or_lod2d.restype = None
        lib.or_lod2d.argtypes = [c_int, c_int, c_int, _DP, _DP, _DP, _DP, _DP, _DP, c_int, _LP,
                                 _DP]
        lib.or_apply_dirichlet.restype = None
        lib.or_apply_dirichlet.argtypes = [c_int, _DP, c_int, _LP, _DP]
        lib.or_lod3d.restype = None
        lib.or_lod3d.argtypes = [c_int, c_int, c_int, c_int, _DP, _DP, _DP, _DP, _DP, _DP, _DP,
                                 _DP, c_int, _LP, _DP]
        lib.or_bulk.restype = None
        lib.or_bulk.argtypes = [c_int64, c_int, _DP, _DP, _DP, _DP, c_double]
        lib.or_agent_constants.restype = None
        lib.or_agent_constants.argtypes = [c_int, c_double, c_double, c_double, _DP, _DP, _DP,
                                           _DP, _DP]
        lib.or_cells.restype = None
        lib.or_cells.argtypes = [c_int64, c_int, _DP, _LP, _DP, _DP]
        lib.or_gradients.restype = None
        lib.or_gradients.argtypes = [c_int, c_int, c_int, c_int, _DP, c_double, c_double,
                                     c_double, _DP]
        lib.or_run.restype = None
        lib.or_run.argtypes = [c_int, c_int, c_int, c_int, c_double, c_double, c_int, c_int, _DP,
                               _DP, _DP, _DP, _DP, _DP, c_int64, _LP, _DP, _DP, c_int, _LP, _DP]
        _oracle = lib
    return _oracle


def reference_available(variant: str = "core2") -> bool:
    return os.path.exists(REF_LIBS[variant])


def load_reference(variant: str = "core2") -> ctypes.CDLL:
    if variant not in _refs:
        path = REF_LIBS[variant]
        if not os.path.exists(path):
            raise ImportError(f"{path} missing: run `make -C oracle ref` where the reference "
                              "sources are present")
        lib = ctypes.CDLL(path)
        V = c_void_p
        sig = {
            "refh_create": (V, [c_int]),
            "refh_destroy": (None, [V]),
            "refh_set_threads": (None, [V, c_int, c_int]),
            "refh_resize_space": (None, [V] + [c_double] * 9),
            "refh_resize_space_nodes": (None, [V] + [c_double] * 6 + [c_int] * 3),
            "refh_mesh_info": (None, [V, _IP, _DP]),
            "refh_set_coefficients": (None, [V, _DP, _DP]),
            "refh_set_densities": (None, [V, _DP]),
            "refh_get_densities": (None, [V, _DP]),
            "refh_set_bulk": (None, [V, _DP, _DP, _DP]),
            "refh_add_dirichlet": (None, [V, c_int, _DP]),
            "refh_update_dirichlet": (None, [V, c_int, _DP]),
            "refh_add_agent": (c_int, [V] + [c_double] * 4 + [_DP, _DP, _DP, c_double]),
            "refh_set_solver": (None, [V, c_int]),
            "refh_step_bulk": (None, [V, c_double]),
            "refh_step_cells": (None, [V, c_double]),
            "refh_step_diffusion": (None, [V, c_double]),
            "refh_apply_dirichlet": (None, [V]),
            "refh_run": (c_double, [V, c_double, c_int, c_int]),
            "refh_num_threads": (c_int, []),
            "refh_gradients": (None, [V, _DP]),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _refs[variant] = lib
    return _refs[variant]


# ---------------------------------------------------------------------------
# oracle (C restatement)

def oracle_thomas(n: int, S: int, dx: float, dt: float, D, decay):
    lib = load_oracle()
    D = np.ascontiguousarray(D, np.float64)
    decay = np.ascontiguousarray(decay, np.float64)
    c1 = np.empty(S)
    den = np.empty((n, S))
    cx = np.empty((n, S))
    lib.or_thomas_setup(n, S, dx, dt, _d(D), _d(decay), _d(c1), _d(den), _d(cx))
    return c1, den, cx


def oracle_lod2d_run(scn, steps: int) -> np.ndarray:
    """steps of the 2-D LOD solver on the z = 0 plane (diffusion only)."""
    lib = load_oracle()
    m = scn.mesh
    S = scn.S
    p = np.ascontiguousarray(scn.initial_field(), np.float64).copy()
    D = np.ascontiguousarray(scn.D, np.float64)
    dec = np.ascontiguousarray(scn.decay, np.float64)
    c1 = np.empty(S)
    dnx, cxx = np.empty((m.nx, S)), np.empty((m.nx, S))
    dny, cxy = np.empty((m.ny, S)), np.empty((m.ny, S))
    lib.or_thomas_setup_2d(m.nx, S, m.dx, scn.dt, _d(D), _d(dec), _d(c1), _d(dnx), _d(cxx))
    lib.or_thomas_setup_2d(m.ny, S, m.dx, scn.dt, _d(D), _d(dec), _d(c1), _d(dny), _d(cxy))
    if scn.dirichlet_voxels is not None and len(scn.dirichlet_voxels):
        dv = np.ascontiguousarray(scn.dirichlet_voxels, np.int64)
        dval = np.ascontiguousarray(scn.dirichlet_values, np.float64)
    else:
        dv, dval = np.zeros(0, np.int64), np.zeros((0, S))
    for _ in range(steps):
        lib.or_lod2d(m.nx, m.ny, S, _d(p), _d(c1), _d(dnx), _d(cxx), _d(dny), _d(cxy), dv.size,
                     _l(dv), _d(dval))
    return p


def oracle_agent_arrays(scn):
    """(voxel, temp1, temp2) through the oracle's own restatement."""
    lib = load_oracle()
    m = scn.mesh
    A, S = scn.num_agents, scn.S
    box = np.array([m.x0, m.y0, m.z0])
    vox = np.empty(A, np.int64)
    t1 = np.empty((A, S))
    t2 = np.empty((A, S))
    for a in range(A):
        x, y, z = (float(v) for v in scn.agent_pos[a])
        vox[a] = lib.or_nearest_voxel(_d(box), m.dx, m.dy, m.dz, m.nx, m.ny, m.nz, x, y, z)
        sec = np.ascontiguousarray(scn.agent_secretion[a])
        sat = np.ascontiguousarray(scn.agent_saturation[a])
        up = np.ascontiguousarray(scn.agent_uptake[a])
        r1 = np.empty(S)
        r2 = np.empty(S)
        lib.or_agent_constants(S, scn.dt, float(scn.agent_volume[a]), m.dV, _d(sec), _d(sat),
                               _d(up), _d(r1), _d(r2))
        t1[a] = r1
        t2[a] = r2
    return vox, t1, t2


def oracle_run(scn, steps: int | None = None, flags: int = 7, p0=None) -> np.ndarray:
    """Runs the scenario through the C restatement; returns [N, S]."""
    lib = load_oracle()
    m = scn.mesh
    steps = scn.steps if steps is None else steps
    p = np.ascontiguousarray(scn.initial_field() if p0 is None else p0, np.float64).copy()
    supply, target, uptake = scn.dense_bulk()
    if scn.num_agents:
        vox, t1, t2 = oracle_agent_arrays(scn)
    else:
        vox, t1, t2 = np.zeros(0, np.int64), np.zeros((0, scn.S)), np.zeros((0, scn.S))
    if scn.dirichlet_voxels is not None and len(scn.dirichlet_voxels):
        dv = np.ascontiguousarray(scn.dirichlet_voxels, np.int64)
        dval = np.ascontiguousarray(scn.dirichlet_values, np.float64)
    else:
        dv, dval = np.zeros(0, np.int64), np.zeros((0, scn.S))
    lib.or_run(m.nx, m.ny, m.nz, scn.S, m.dx, scn.dt, steps, flags, _d(p),
               _d(np.ascontiguousarray(scn.D, np.float64)),
               _d(np.ascontiguousarray(scn.decay, np.float64)), _d(supply), _d(target),
               _d(uptake), vox.size, _l(vox), _d(t1), _d(t2), dv.size, _l(dv), _d(dval))
    return p


# ---------------------------------------------------------------------------
# the compiled reference

class Reference:
    """One reference Microenvironment built from a Scenario, the way the
    reference's example drivers build one."""

    def __init__(self, scn, variant: str = "core2", threads: int = 1,
                 cells_single_thread: bool = True):
        self.lib = load_reference(variant)
        self.scn = scn
        lib = self.lib
        m = scn.mesh
        self.h = lib.refh_create(scn.S)
        lib.refh_set_threads(self.h, threads, 1 if cells_single_thread else 0)
        lib.refh_resize_space(self.h, m.x0, m.x1, m.y0, m.y1, m.z0, m.z1, m.dx, m.dy, m.dz)
        lib.refh_set_coefficients(self.h, _d(np.ascontiguousarray(scn.D, np.float64)),
                                  _d(np.ascontiguousarray(scn.decay, np.float64)))
        if scn.p0 is not None:
            lib.refh_set_densities(self.h, _d(np.ascontiguousarray(scn.p0, np.float64)))
        supply, target, uptake = scn.dense_bulk()
        if supply is not None or target is not None or uptake is not None:
            lib.refh_set_bulk(self.h, _d(supply), _d(target), _d(uptake))
        if scn.dirichlet_voxels is not None:
            for v, x in zip(scn.dirichlet_voxels, scn.dirichlet_values):
                lib.refh_add_dirichlet(self.h, int(v), _d(np.ascontiguousarray(x, np.float64)))
        self.agent_voxels = np.zeros(scn.num_agents, np.int64)
        for a in range(scn.num_agents):
            x, y, z = (float(v) for v in scn.agent_pos[a])
            self.agent_voxels[a] = lib.refh_add_agent(
                self.h, x, y, z, float(scn.agent_volume[a]),
                _d(np.ascontiguousarray(scn.agent_secretion[a], np.float64)),
                _d(np.ascontiguousarray(scn.agent_saturation[a], np.float64)),
                _d(np.ascontiguousarray(scn.agent_uptake[a], np.float64)), scn.dt)

    def set_solver(self, dims: int):
        self.lib.refh_set_solver(self.h, dims)

    def mesh_info(self):
        nxyz = (c_int * 5)()
        geom = (c_double * 10)()
        self.lib.refh_mesh_info(self.h, nxyz, geom)
        return tuple(nxyz), tuple(geom)

    def run(self, steps: int, flags: int = 7, dt: float | None = None) -> float:
        """Steps bulk -> cells -> diffusion; returns wall seconds (steady_clock)."""
        return self.lib.refh_run(self.h, self.scn.dt if dt is None else dt, steps, flags)

    def step_bulk(self, dt=None):
        self.lib.refh_step_bulk(self.h, self.scn.dt if dt is None else dt)

    def step_cells(self, dt=None):
        self.lib.refh_step_cells(self.h, self.scn.dt if dt is None else dt)

    def step_diffusion(self, dt=None):
        self.lib.refh_step_diffusion(self.h, self.scn.dt if dt is None else dt)

    def apply_dirichlet(self):
        self.lib.refh_apply_dirichlet(self.h)

    def gradients(self) -> np.ndarray:
        """compute_all_gradient_vectors, then every gradient_vector(n): [N, S, 3]."""
        out = np.zeros((self.scn.num_voxels, self.scn.S, 3))
        self.lib.refh_gradients(self.h, _d(out))
        return out

    def densities(self) -> np.ndarray:
        out = np.empty((self.scn.num_voxels, self.scn.S))
        self.lib.refh_get_densities(self.h, _d(out))
        return out

    def close(self):
        if self.h:
            self.lib.refh_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def reference_run(scn, steps: int | None = None, flags: int = 7, variant: str = "core2",
                  threads: int = 1) -> np.ndarray:
    with Reference(scn, variant, threads) as r:
        r.run(scn.steps if steps is None else steps, flags)
        return r.densities()


def max_rel_err(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per-substrate relative max-norm error: max|a-b| / max|b| (columns)."""
    a = np.asarray(a).reshape(b.shape)
    den = np.maximum(np.abs(b).max(axis=0), 1e-300)
    return np.abs(a - b).max(axis=0) / den


def wall(f, *args, **kw):
    t0 = time.perf_counter()
    out = f(*args, **kw)
    return out, time.perf_counter() - t0


def oracle_gradients(p: np.ndarray, shape, dx: float, dy: float | None = None,
                     dz: float | None = None, g: np.ndarray | None = None) -> np.ndarray:
    """compute_all_gradient_vectors on the field p [N, S]: [N, S, 3] (entries at
    axis ends keep g's values, zero by default)."""
    lib = load_oracle()
    nx, ny, nz = shape
    p = np.ascontiguousarray(p, np.float64)
    S = p.shape[1]
    out = np.zeros((p.shape[0], S, 3)) if g is None else np.array(g, np.float64, copy=True)
    lib.or_gradients(nx, ny, nz, S, _d(p), dx, dx if dy is None else dy,
                     dx if dz is None else dz, _d(out))
    return out
