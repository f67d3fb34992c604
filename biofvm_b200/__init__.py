"""biofvm_b200: BioFVM's per-step transport path on NVIDIA B200 (sm_100a).

The compute lives in libbfvm.so (hand-written CUDA, C ABI in include/bfvm.h);
this package holds the Python view of that ABI, the host-side mesh geometry
and the seeded synthetic workloads.  There is no CPU fallback: without the
built library, importing the solver raises.
"""
from . import mesh, workloads
from ._abi import BfvmError, FP32, FP64, STEP_ALL, STEP_BULK, STEP_CELLS, STEP_DIFFUSION
from .batch import Batch
from .solver import Solver, load_scenario

__all__ = ["Batch", "Solver", "load_scenario", "mesh", "workloads", "BfvmError", "FP32", "FP64",
           "STEP_ALL", "STEP_BULK", "STEP_CELLS", "STEP_DIFFUSION"]
