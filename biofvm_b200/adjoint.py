"""The transport path as a differentiable function (reverse mode on the GPU).

``AdjointProblem(scn, nsteps)`` holds one device-resident microenvironment
set up from a workload scenario.  ``forward(secretion, uptake, D, decay)``
runs ``nsteps`` steps from the scenario's initial field with those
parameters (per-agent secretion and uptake rates [A, S], per-substrate
diffusion coefficients and decay rates [S]) and records checkpoints;
``backward(seed)`` returns dLoss/d(parameter) for seed = dLoss/d(final
field), through bfvm_adjoint_backward.  ``transport(...)`` wraps the pair in
a ``torch.autograd.Function``.

The agent constants follow Basic_Agent::set_internal_uptake_constants
(BioFVM_basic_agent.cpp:114-148): with c = dt V / V_voxel,
temp1 = secretion * saturation * c and temp2 = 1 + c secretion + c uptake, so
d/dsecretion = saturation c dtemp1 + c dtemp2 and d/duptake = c dtemp2.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import call, dptr
from .mesh import agent_constants
from .solver import Solver, load_scenario


class AdjointProblem:
    def __init__(self, scn, nsteps: int, checkpoint_every: int = 20,
                 flags: int = _abi.STEP_ALL, device: int = 0):
        self.scn = scn
        self.nsteps = int(nsteps)
        self.k = int(checkpoint_every)
        self.flags = int(flags)
        self.solver = Solver(device)
        load_scenario(self.solver, scn)
        self.p0 = scn.initial_field()
        if scn.num_agents:
            self.vox, _, _ = scn.agent_arrays()
            vol = np.asarray(scn.agent_volume, np.float64).reshape(-1, 1)
            self.saturation = np.asarray(scn.agent_saturation, np.float64)
        else:
            self.vox = np.zeros(0, np.int64)
            vol = np.zeros((0, 1))
            self.saturation = np.zeros((0, scn.S))
        self.c = scn.dt * vol / scn.mesh.dV

    def close(self) -> None:
        self.solver.close()

    def set_parameters(self, secretion, uptake, D, decay) -> None:
        scn, sv = self.scn, self.solver
        sv.set_coefficients(np.asarray(D, np.float64), np.asarray(decay, np.float64))
        sv.reset_diffusion_setup()
        if scn.num_agents:
            t1, t2 = agent_constants(scn.dt, scn.agent_volume, scn.mesh.dV,
                                     np.asarray(secretion, np.float64), self.saturation,
                                     np.asarray(uptake, np.float64))
            sv.set_agents(self.vox, t1, t2)
        sv.set_densities(self.p0)

    def run(self, secretion, uptake, D, decay) -> np.ndarray:
        """Forward only (no checkpoints)."""
        self.set_parameters(secretion, uptake, D, decay)
        self.solver.step(self.scn.dt, self.nsteps, self.flags)
        return self.solver.get_densities()

    def forward(self, secretion, uptake, D, decay) -> np.ndarray:
        self.set_parameters(secretion, uptake, D, decay)
        call("bfvm_adjoint_forward", self.solver.handle, self.scn.dt, self.nsteps, self.flags,
             self.k)
        return self.solver.get_densities()

    def backward(self, seed: np.ndarray, want_p0: bool = False) -> dict:
        scn = self.scn
        S, A, N = scn.S, scn.num_agents, scn.num_voxels
        seed = np.ascontiguousarray(seed, np.float64).reshape(N, S)
        gD = np.zeros(S)
        gdecay = np.zeros(S)
        gt1 = np.zeros((A, S))
        gt2 = np.zeros((A, S))
        gp0 = np.zeros((N, S)) if want_p0 else None
        call("bfvm_adjoint_backward", self.solver.handle,
             ctypes.c_void_p(seed.ctypes.data), 0, dptr(gD), dptr(gdecay),
             dptr(gt1) if A else None, dptr(gt2) if A else None,
             dptr(gp0) if want_p0 else None)
        out = {"D": gD, "decay": gdecay, "temp1": gt1, "temp2": gt2,
               "secretion": gt1 * self.saturation * self.c + gt2 * self.c,
               "uptake": gt2 * self.c}
        if want_p0:
            out["p0"] = gp0
        return out


def loss_difference(p_plus: np.ndarray, p_minus: np.ndarray, target: np.ndarray) -> float:
    """L(p+) - L(p-) for L(p) = 1/2 |p - target|^2, summed as
    1/2 sum((p+ - p-)(p+ + p- - 2 target)): the two losses are never formed,
    so the difference keeps its digits (central finite differences)."""
    return 0.5 * float(np.sum((p_plus - p_minus) * (p_plus + p_minus - 2.0 * target)))


def transport(problem: AdjointProblem, secretion, uptake, D, decay):
    """torch.autograd entry: the final field [N, S] (float64, on the inputs'
    device) as a differentiable function of the four parameter tensors."""
    import torch

    class _Transport(torch.autograd.Function):
        @staticmethod
        def forward(ctx, sec, upt, d, lam):
            out = problem.forward(sec.detach().cpu().numpy(), upt.detach().cpu().numpy(),
                                  d.detach().cpu().numpy(), lam.detach().cpu().numpy())
            return torch.from_numpy(out).to(sec.device)

        @staticmethod
        def backward(ctx, grad_out):
            g = problem.backward(grad_out.detach().cpu().numpy())
            dev = grad_out.device
            return (torch.from_numpy(g["secretion"]).to(dev),
                    torch.from_numpy(g["uptake"]).to(dev),
                    torch.from_numpy(g["D"]).to(dev),
                    torch.from_numpy(g["decay"]).to(dev))

    return _Transport.apply(secretion, uptake, D, decay)
