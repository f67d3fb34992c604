"""Regenerates tests/golden/*.npz by running the UNMODIFIED BioFVM reference,
compiled from its own sources by oracle/Makefile (oracle/_ref/), on the seeded
cases of cases.py.  Needs the reference sources (only present where the
fixtures are made):

    make -C oracle && python tests/golden/make_golden.py

Each fixture holds the case's input fingerprint, the agents' voxel indices as
the reference assigned them, and the densities after the run: the whole
array, or its SHA-256 plus sampled values for the larger cases.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

from cases import CASES, input_fingerprint, sample_index, sha  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main() -> None:
    out_dir = os.path.dirname(os.path.abspath(__file__))
    for name, (build, flags, steps, store) in CASES.items():
        scn = build()
        with O.Reference(scn, "core2", threads=1) as ref:
            ref.run(steps, flags)
            p = ref.densities()
            vox = ref.agent_voxels.copy()
        rec = {"fingerprint": np.array(input_fingerprint(scn)), "flags": np.array(flags),
               "steps": np.array(steps), "agent_voxels": vox, "sha": np.array(sha(p)),
               "shape": np.array(p.shape)}
        if store == "full":
            rec["p"] = p
        else:
            idx = sample_index(p.size)
            rec["sample_idx"] = idx
            rec["sample_val"] = p.ravel()[idx]
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), **rec)
        print(f"{name}: {p.shape} sha={rec['sha']}")


if __name__ == "__main__":
    main()
