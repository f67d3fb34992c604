"""Test infrastructure only (the oracle): an FP64 tangent-linear model of the
transport step, to check the GPU adjoint.

For a direction v in parameter space (per-agent secretion and uptake rates,
per-substrate diffusion coefficients and decay rates) it propagates the
forward-mode derivative pdot alongside the field p through n steps of
bulk -> cells -> LOD_3D, statement for statement as the reference computes p:

* bulk (BioFVM_microenvironment.cpp:603-609): p1 = (p0 + dt S T)/((U+S) dt + 1),
  pdot1 = pdot0 / ((U+S) dt + 1)  (bulk rates are not differentiated);
* cells, agents in list order (BioFVM_basic_agent.cpp:234-235):
  x' = (x + t1)/t2,  xdot' = (xdot + t1dot)/t2 - x' t2dot/t2, with
  t1dot = secdot * sat * c and t2dot = c secdot + c uptdot (:139-147);
* Dirichlet before each sweep (BioFVM_solvers.cpp:177,207,241): pdot = 0 there;
* each axis solve y = A^-1 x with A = (1 + c2) I + c1 L (L the Neumann
  Laplacian along the axis, BioFVM_solvers.cpp:105-142):
  ydot = A^-1 (xdot - c1dot L y - c2dot y),  c1dot = dt Ddot/dx^2,
  c2dot = dt decaydot/3.  A^-1 is applied with the reference's Thomas
  factors (or_thomas_setup) and its elimination order (:186-200).

The primal p follows the same statements, so it reproduces the oracle's
field.  dLoss = sum((p_T - target) * pdot_T) for Loss = 1/2 |p_T - target|^2.
"""
from __future__ import annotations

import numpy as np

from . import oracle as O


def thomas_factors(n: int, S: int, dx: float, dt: float, D, decay):
    lib = O.load_oracle()
    c1 = np.zeros(S)
    den = np.zeros((n, S))
    cx = np.zeros((n, S))
    D = np.ascontiguousarray(D, np.float64)
    decay = np.ascontiguousarray(decay, np.float64)
    lib.or_thomas_setup(n, S, dx, dt, O._d(D), O._d(decay), O._d(c1), O._d(den), O._d(cx))
    return c1, den, cx


def _solve(arr, c1, den, cx):
    """In place on arr [n, ..., S]: the reference's Thomas elimination."""
    n = arr.shape[0]
    arr[0] /= den[0]
    for i in range(1, n):
        arr[i] += c1 * arr[i - 1]
        arr[i] /= den[i]
    for i in range(n - 2, -1, -1):
        arr[i] -= cx[i] * arr[i + 1]


def _laplacian(arr):
    """Neumann Laplacian along axis 0 of arr [n, ..., S]."""
    out = np.zeros_like(arr)
    n = arr.shape[0]
    if n > 1:
        out[:-1] += arr[:-1] - arr[1:]
        out[1:] += arr[1:] - arr[:-1]
    return out


def tangent_run(scn, nsteps: int, flags: int, secretion, uptake, D, decay, dsec, dupt, dD,
                ddecay, p0=None, dp0=None):
    """(p_T, pdot_T) as [N, S] arrays."""
    nx, ny, nz = scn.shape
    S, dt, dx = scn.S, scn.dt, scn.mesh.dx
    N = nx * ny * nz
    p = (scn.initial_field() if p0 is None else np.array(p0, np.float64)).reshape(nz, ny, nx, S)
    pd = np.zeros_like(p) if dp0 is None else np.array(dp0, np.float64).reshape(nz, ny, nx, S)
    factors = [thomas_factors(n, S, dx, dt, D, decay) for n in (nx, ny, nz)]
    c1dot = dt * np.asarray(dD, np.float64) / dx / dx
    c2dot = dt * np.asarray(ddecay, np.float64) / 3.0
    pf, pdf = p.reshape(N, S), pd.reshape(N, S)

    bulk = scn.bulk_voxels is not None and len(scn.bulk_voxels) > 0
    if bulk:
        bv = np.asarray(scn.bulk_voxels, np.int64)
        st = scn.bulk_target * scn.bulk_supply
        su = scn.bulk_uptake + scn.bulk_supply
        bden = su * dt + 1.0
    A = scn.num_agents
    if A:
        from biofvm_b200.mesh import agent_constants

        vox, _, _ = scn.agent_arrays()
        vol = np.asarray(scn.agent_volume, np.float64).reshape(-1, 1)
        c = dt * vol / scn.mesh.dV
        sat = np.asarray(scn.agent_saturation, np.float64)
        t1, t2 = agent_constants(dt, scn.agent_volume, scn.mesh.dV,
                                 np.asarray(secretion, np.float64), sat,
                                 np.asarray(uptake, np.float64))
        t1d = np.asarray(dsec, np.float64) * sat * c
        t2d = c * np.asarray(dsec, np.float64) + c * np.asarray(dupt, np.float64)
    dirichlet = scn.dirichlet_voxels is not None and len(scn.dirichlet_voxels) > 0

    def apply_dirichlet():
        if dirichlet:
            for v, val in zip(scn.dirichlet_voxels, scn.dirichlet_values):
                pf[v] = val
                pdf[v] = 0.0

    for _ in range(nsteps):
        if flags & 1 and bulk:
            pf[bv] = (pf[bv] + dt * st) / bden
            pdf[bv] = pdf[bv] / bden
        if flags & 2 and A:
            for a in range(A):
                v = vox[a]
                x_new = (pf[v] + t1[a]) / t2[a]
                pdf[v] = (pdf[v] + t1d[a]) / t2[a] - x_new * t2d[a] / t2[a]
                pf[v] = x_new
        if not flags & 4:
            continue
        for ax, spatial in ((0, 2), (1, 1), (2, 0)):
            apply_dirichlet()
            c1, den, cx = factors[ax]
            y = np.moveaxis(p, spatial, 0)
            yd = np.moveaxis(pd, spatial, 0)
            _solve(y, c1, den, cx)
            yd -= c1dot * _laplacian(y) + c2dot * y
            _solve(yd, c1, den, cx)
    return pf.copy(), pdf.copy()
