"""The GPU writer's number formatter (ipglasma_b200/csrc/fmt.cuh), compiled
here as plain C++, prints every value exactly as std::to_chars with
precision 6 (printf "%.6g", the host writers' format): random doubles over
and beyond its range, exact ties, decade and rounding boundaries, ints."""
import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_formatter_matches_to_chars(tmp_path):
    exe = tmp_path / "fmt_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe),
                    str(HERE / "native" / "fmt_check.cpp")], check=True)
    res = subprocess.run([str(exe), "300000"], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    assert " mismatches 0 " in res.stdout, res.stdout
