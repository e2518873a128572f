"""Input-file handling of the drop-in executable (no GPU: these cases end
before the first device call).

The reference reads keys with Setup::StringFind (Setup.cpp:24-71): a missing
input file ends the program with "The input file named <f> is absent.
Exiting.", a missing key with "<key> not found in <f>" and "Create a complete
input file.", both with exit status 1. A file without the EndOfFile marker
makes the reference's search loop forever once it looks for a key that is
not there; the executable here stops at the end of the file and reports the
missing key in the same words instead.
"""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
EXE = ROOT / "ipglasma_b200" / "ipglasma_b200"

KEYS = """size 32
L 6.0
Nc 3
Ny 3
g 2.0
m 0.2
UVdamp 0.
maxtime 0.2
"""


def run(tmp_path, text, name="input"):
    if not EXE.exists():
        pytest.skip("executable not built")
    if text is not None:
        (tmp_path / name).write_text(text)
    return subprocess.run([str(EXE), name], cwd=tmp_path, capture_output=True, text=True,
                          timeout=60)


def test_missing_input_file(tmp_path):
    res = run(tmp_path, None, "nonexistent_input")
    assert res.returncode == 1
    assert "The input file named nonexistent_input is absent. Exiting." in res.stderr


def test_missing_key(tmp_path):
    res = run(tmp_path, KEYS + "EndOfFile\n")
    assert res.returncode == 1
    assert "writeOutputs not found in input" in res.stderr
    assert "Create a complete input file." in res.stdout


def test_missing_end_of_file_marker_does_not_hang(tmp_path):
    res = run(tmp_path, KEYS)
    assert res.returncode == 1
    assert "writeOutputs not found in input" in res.stderr


def test_keys_after_end_of_file_are_not_read(tmp_path):
    """Everything after EndOfFile is ignored, as in the reference."""
    text = KEYS.replace("maxtime 0.2\n", "EndOfFile\nmaxtime 0.2\n")
    res = run(tmp_path, text)
    assert res.returncode == 1
    assert "maxtime not found in input" in res.stderr
