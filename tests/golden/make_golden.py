"""Regenerate the golden fixtures from the reference itself.

Runs oracle/_ref/ipg_ref_harness (the reference sources compiled unmodified
against the project's FFTW/GSL subset, see oracle/Makefile) on small seeded
inputs and stores inputs and outputs as compressed .npz files next to this
script. The reference has no tests or golden vectors of its own, so these
fixtures are what pins the oracle and the CUDA path.

    make -C oracle ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parent.parent))

from refcase import run_harness  # noqa: E402
from ipglasma_b200.synthetic import gaussian_blobs  # noqa: E402

CASES = [
    # name, N, L fm, Ny, seed, maxtime fm
    ("blobs_n16", 16, 2.0, 2, 3, 0.2),
    ("blobs_n32", 32, 3.75, 3, 1, 0.2),
]


def main() -> None:
    for name, N, L, Ny, seed, maxtime in CASES:
        A, B = gaussian_blobs(N, L, 2.0, 1.5)
        with tempfile.TemporaryDirectory() as tmp:
            full = run_harness(Path(tmp) / "full", A, B, N, L, Ny, 2.0, 0.2, seed, maxtime,
                               write_outputs=5)
            steps = run_harness(Path(tmp) / "steps", A, B, N, L, Ny, 2.0, 0.2, seed, maxtime,
                                mode="steps", steps=4)
            assert full.meta["newton_restart_draws"] == 0, "case needs Newton restarts"
            xa, xb = full.xi()
            meta = {k: v for k, v in full.meta.items() if k != "stdout"}
            meta.update(case=name, g=2.0, m=0.2, seed=seed, maxtime=maxtime,
                        steps_mode_steps=4)
            hydro = (Path(tmp) / "full" / "epsilon-u-Hydro-TauHydro-0.dat").read_text()
            tmunu = sorted((Path(tmp) / "full").glob("Tmunu-t*-0.dat"))[0]
            np.savez_compressed(
                HERE / f"{name}.npz",
                g2muA=A, g2muB=B, xiA=xa, xiB=xb,
                VA=full.mats("VA.bin"), VB=full.mats("VB.bin"),
                tau0_Ux=full.mats("tau0_Ux.bin"), tau0_Uy=full.mats("tau0_Uy.bin"),
                tau0_pi=full.mats("tau0_pi.bin"), obs=full.observables(),
                final_Ux=full.mats("final_Ux.bin"), final_E1=full.mats("final_E1.bin"),
                final_pi=full.mats("final_pi.bin"),
                steps_Ux=steps.mats("steps_Ux.bin"), steps_E2=steps.mats("steps_E2.bin"),
                steps_phi=steps.mats("steps_phi.bin"), steps_pi=steps.mats("steps_pi.bin"),
                meta=json.dumps(meta), hydro_file=hydro, tmunu_file=tmunu.read_text(),
                tmunu_name=tmunu.name)
            print("wrote", name, meta["eccentricity2"], meta["gauss_violation"])


if __name__ == "__main__":
    main()
