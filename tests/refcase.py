"""Helpers that run the reference harness (oracle/_ref) and load its dumps.

Test infrastructure: only tests, the smoke check and the CPU-baseline leg of
bench.py use this module.
"""
from __future__ import annotations

import json
import os
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
REF = ROOT / "oracle" / "_ref"
HARNESS = REF / "ipg_ref_harness"
HARNESS_OFAST = REF / "ipg_ref_harness_ofast"


@dataclass
class RefRun:
    out: Path
    N: int
    meta: dict

    def mats(self, name: str) -> np.ndarray:
        a = np.fromfile(self.out / name, dtype="<f8")
        return a.reshape(self.N * self.N, 9, 2).view(np.complex128)[..., 0].reshape(-1, 3, 3)

    def xi(self) -> tuple[np.ndarray, np.ndarray]:
        return (np.fromfile(self.out / "xiA.bin", dtype="<f8"),
                np.fromfile(self.out / "xiB.bin", dtype="<f8"))

    def observables(self) -> np.ndarray:
        """(25, N*N): eps, u(4), T(10), pi(10)."""
        a = np.fromfile(self.out / "obs.bin", dtype="<f8")
        return a.reshape(self.N * self.N, 25).T.copy()


def run_harness(out: Path, g2mu2A, g2mu2B, N: int, L: float, Ny: int,
                g: float, m: float, seed: int, maxtime: float,
                mode: str = "full", steps: int = 0, write_outputs: int = 0,
                size_output: int = 0, L_output: float = 0.0, dtau: float = -1.0,
                threads: int = 1, binary: Path = HARNESS,
                timeout: float = 3600, dumps: bool = True, extra=()) -> RefRun:
    if not binary.exists():
        raise FileNotFoundError(f"{binary} missing: run `make -C oracle`")
    out = Path(out)
    out.mkdir(parents=True, exist_ok=True)
    g2 = out / "g2mu.bin"
    np.concatenate([np.asarray(g2mu2A, dtype="<f8").ravel(),
                    np.asarray(g2mu2B, dtype="<f8").ravel()]).tofile(g2)
    cmd = [str(binary), "--g2mu", str(g2), "--out", str(out), "--N", str(N),
           "--L", repr(L), "--Ny", str(Ny), "--g", repr(g), "--m", repr(m),
           "--seed", str(seed), "--maxtime", repr(maxtime), "--mode", mode,
           "--steps", str(steps), "--write-outputs", str(write_outputs),
           "--size-output", str(size_output or N),
           "--L-output", repr(L_output or L), "--dtau", repr(dtau),
           "--dumps", "1" if dumps else "0", *extra]
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    res = subprocess.run(cmd, capture_output=True, text=True, env=env,
                         timeout=timeout)
    if res.returncode != 0:
        raise RuntimeError(f"harness failed: {res.stderr[-2000:]}")
    meta = json.loads((out / "harness.json").read_text())
    meta["stdout"] = res.stdout
    for line in res.stdout.splitlines():
        if line.startswith("Gauss violation="):
            meta["gauss_violation"] = float(line.split("=")[1])
    return RefRun(out, N, meta)


def rel_err(a: np.ndarray, b: np.ndarray, scale: float | None = None) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    s = scale if scale is not None else max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / s)
