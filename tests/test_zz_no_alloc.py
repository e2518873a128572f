"""ipg_wilson_lines_noalloc: the allocation-free Wilson-line entry point.

It exists for callers that cannot allocate device memory (code inside another
framework's memory pool, hosts that forbid allocation after start-up). It
keeps its scratch in one fixed device array, so two things are checked here
beyond the result itself: two calls in a row give the same answer (the array
keeps the previous call's contents, which must not leak into the next call),
and sizes beyond the array's limit are rejected before any device work.

The expected values come from the regular entry point (ipg_init_fields) on
the same inputs. This file sorts last so that a run stopping at the first
failure has already run every other test.
"""
import ctypes as ct
import json
from pathlib import Path

import numpy as np
import pytest

import ipglasma_b200 as ipg

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent


def _noalloc():
    lib = ipg.lib()
    fn = lib.ipg_wilson_lines_noalloc
    fn.restype = ct.c_int
    fn.argtypes = [ct.c_int, ct.c_int, ct.c_double, ct.c_double, ct.c_double, ct.c_double,
                   ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]
    return fn


def test_noalloc_matches_regular_entry_point_twice():
    import torch

    g = dict(np.load(ROOT / "tests" / "golden" / "blobs_n32.npz"))
    m = json.loads(str(g["meta"]))
    N, Ny = m["N"], m["Ny"]
    cfg = ipg.Config(size=N, L=m["L"], Ny=Ny, g=m["g"], m=m["m"], maxtime=m["maxtime"])
    with ipg.Event(cfg) as ev:
        ev.set_g2mu(g["g2muA"], g["g2muB"])
        ev.set_noise(g["xiA"], g["xiB"])
        ev.init_fields()
        expect = {"A": ev.get_field(ipg.VA), "B": ev.get_field(ipg.VB)}

    fn = _noalloc()
    dev = torch.device("cuda:0")
    out = torch.empty(N * N * 18, dtype=torch.float64, device=dev)
    # two calls in a row per nucleus, alternating, so each call starts from
    # the other nucleus's leftovers in the shared scratch array
    for rep in range(2):
        for nuc in ("A", "B"):
            d_g2 = torch.tensor(g[f"g2mu{nuc}"], dtype=torch.float64, device=dev)
            d_xi = torch.tensor(g[f"xi{nuc}"], dtype=torch.float64, device=dev)
            out.fill_(np.nan)
            torch.cuda.synchronize()
            st = fn(N, Ny, m["L"], m["g"], m["m"], 0.0, d_g2.data_ptr(), d_xi.data_ptr(),
                    out.data_ptr(), None)
            torch.cuda.synchronize()
            assert st == 0
            V = out.cpu().numpy().view(np.complex128).reshape(N * N, 3, 3)
            assert np.abs(V - expect[nuc]).max() < 1e-12, (rep, nuc)
            assert np.abs(V - g[f"V{nuc}"]).max() < 1e-12, (rep, nuc)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    fn = _noalloc()
    small = torch.zeros(16, dtype=torch.float64, device="cuda:0")
    p = small.data_ptr()
    for N in (512, 1024, 100):
        assert fn(N, 2, 10.0, 2.0, 0.2, 0.0, p, p, p, None) == 1  # IPG_ERR_BAD_CONFIG
    assert fn(32, 0, 10.0, 2.0, 0.2, 0.0, p, p, p, None) == 1
