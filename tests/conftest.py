import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


def _ensure_oracle(target: str, path: Path) -> None:
    if path.exists():
        return
    # the oracle's Makefile knows where the reference sources are;
    # IPG_REF_SRC overrides it
    src = [f"REF_SRC={os.environ['IPG_REF_SRC']}"] if os.environ.get("IPG_REF_SRC") else []
    make = ["make", "-s", "-C", str(ROOT / "oracle")]
    if target == "ref" and subprocess.run(make + ["have-ref", *src],
                                          capture_output=True).returncode != 0:
        pytest.skip(f"{path} not built and the reference sources are absent")
    subprocess.run(make + [target, *src], check=True, capture_output=True)


@pytest.fixture(scope="session")
def oracle_port():
    import oracle_port as op
    _ensure_oracle("port", op.LIB)
    return op


@pytest.fixture(scope="session")
def ref_harness():
    import refcase
    _ensure_oracle("ref", refcase.HARNESS)
    return refcase


@pytest.fixture(scope="session")
def golden():
    import json

    import numpy as np

    def load(name: str):
        d = dict(np.load(ROOT / "tests" / "golden" / f"{name}.npz"))
        d["meta"] = json.loads(str(d["meta"]))
        return d

    return load
