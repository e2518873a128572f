"""The C-ABI library loads and exports every entry point include/*.h declares;
argument validation works without a GPU."""
import ctypes as ct
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w \*]*?\b(ipg_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("ipg_create", "ipg_destroy", "ipg_set_g2mu", "ipg_set_noise",
                 "ipg_init_fields", "ipg_run", "ipg_evolve", "ipg_get_observables"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from ipglasma_b200 import build

    lib_path = build.build_library()
    lib = ct.CDLL(str(lib_path))
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.parametrize("field,value", [("size", 100), ("size", 4), ("Nc", 2), ("Ny", 0),
                                         ("L", -1.0), ("maxtime", 0.0), ("precision", 7)])
def test_bad_config_rejected_before_device_use(field, value):
    import ipglasma_b200 as ipg

    cfg = ipg.Config(size=32, L=4.0, Ny=2)
    setattr(cfg, field, value)
    with pytest.raises(ipg.IPGError) as e:
        ipg.Event(cfg)
    assert e.value.status == 1  # IPG_ERR_BAD_CONFIG


def test_time_grid_follows_reference_rule():
    """dtau = maxtime / ((int(10 maxtime / a) + 1) a) and itmax = int(maxtime/(a dtau)+0.1)
    (main.cpp:531-534, Evolution.cpp:396); checked on the host side of ipg_create,
    which validates before any device call."""
    for N, L, maxtime, steps in ((256, 30.0, 0.4, 35), (512, 40.0, 0.6, 77)):
        a = L / N
        it = int(10 * maxtime / a) + 1
        dtau = maxtime / (it * a)
        assert int(maxtime / (a * dtau) + 0.1) == steps
