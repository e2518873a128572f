"""IP-Sat colour-charge maps (ipg_set_nuclei_ipsat) against the reference's
own Init::setColorChargeDensity (Init.cpp:753-1676), driven by the harness
with the same nucleon positions and the same Q_s^2(T, y) table.

The table here is synthetic, in the layout of the reference's
qs2Adj_vs_Tp_vs_Y_200.in (Init.cpp:441-480: records "y T Q_s^2", 44
rapidities 0.25 apart per T, 200 T values increasing): Q_s^2 grows with T
and y like a saturation scale. Both sides read the same file, so the test
pins the algorithm (thickness sums, distance cut, table interpolation, the
fluctuating-x fixed point, wounding, event averages), not the table.

The reference's fixed point for nucleus A starts from the rapidity that
nucleus B ended on at the previous cell its thread handled; the harness runs
on one thread, the order the library reproduces. Bounds: T_A, T_B 1e-12 of
their maximum; g^2 mu^2 1e-12 relative where nonzero, and nonzero at the same
cells; N_part, N_coll exact; the averages 1e-10 relative (summation order).
"""
import json
import subprocess

import numpy as np
import pytest

import ipglasma_b200 as ipg

pytestmark = pytest.mark.gpu

NY, NT, DY = 44, 200, 0.25


def synthetic_table():
    T = 1e-4 * (9.44 / 1e-4) ** (np.arange(NT) / (NT - 1))
    y = DY * np.arange(NY)
    qs2 = 2.2 * T[:, None] ** 0.92 * np.exp(0.28 * y[None, :]) * (1 + 0.05 * np.sin(3 * y))[None, :]
    return T, qs2


def write_table(path, T, qs2):
    with open(path, "w") as f:
        for it in range(NT):
            for iy in range(NY):
                f.write(f"{DY * iy:.17g} {T[it]:.17g} {qs2[it, iy]:.17g}\n")


CASES = {
    # N, L, nucleus, b, roots, fluctuating x
    "PbPb_fluct": (256, 30.0, "Pb", 4.0, 5020.0, 1),
    "AuAu_fixed_x": (128, 24.0, "Au", 7.0, 200.0, 0),
    # sqrt(s) = 10 GeV puts the fixed point's rapidity below zero, where the
    # reference carries Q_s from cell to cell (the single-threaded pass)
    "OO_negative_y": (128, 12.0, "O", 1.0, 10.0, 1),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_ipsat_maps_match_reference(case, ref_harness, tmp_path):
    from ipglasma_b200.synthetic import nucleus_spec, sample_nucleus

    N, L, nuc, b, roots, fluct = CASES[case]
    rng = np.random.Generator(np.random.PCG64(77))
    A = sample_nucleus(rng, nucleus_spec(nuc))
    B = sample_nucleus(rng, nucleus_spec(nuc))
    T, qs2 = synthetic_table()
    table = tmp_path / "qs2_table.in"
    write_table(table, T, qs2)
    T, qs2 = ipg.read_qs_table(table, NY)  # the values both sides read
    nucf = tmp_path / "nucleons.bin"
    np.concatenate([[len(A), len(B)], A[:, :2].ravel(), B[:, :2].ravel()]).astype("<f8").tofile(nucf)
    out = tmp_path / "ref"
    cmd = [str(ref_harness.HARNESS), "--mode", "ipsat", "--nucleons", str(nucf), "--table",
           str(table), "--out", str(out), "--N", str(N), "--L", repr(L), "--g", "2.0",
           "--b", repr(b), "--roots", repr(roots), "--fluct", str(fluct)]
    res = subprocess.run(cmd, capture_output=True, text=True, env={"OMP_NUM_THREADS": "1"},
                         timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    meta = json.loads((out / "harness.json").read_text())
    ref = np.fromfile(out / "ipsat.bin", dtype="<f8").reshape(4, N * N)
    with ipg.Event(ipg.Config(size=N, L=L, Ny=2, maxtime=0.1)) as ev:
        rep = ev.set_nuclei_ipsat(A, B, b, (T, qs2), roots=roots, use_fluctuating_x=bool(fluct))
        th = ev.thickness()
        g2 = ev.g2mu()
    for k in range(2):
        assert np.abs(th[k] - ref[k]).max() <= 1e-12 * ref[k].max(), k
        r, o = ref[2 + k], g2[k]
        assert np.array_equal(r > 0, o > 0), (k, int((r > 0).sum()), int((o > 0).sum()))
        m = r > 0
        assert m.sum() > 0
        rel = np.abs(o[m] - r[m]) / r[m]
        assert rel.max() < 1e-12, (k, rel.max())
    assert rep["Npart"] == meta["Npart"] and rep["Ncoll"] == meta["Ncoll"]
    for key in ("Tpp", "average_Qs", "average_Qs_avg", "average_Qs_min"):
        assert abs(rep[key] - meta[key]) <= 1e-10 * abs(meta[key]), key
    if case == "OO_negative_y":
        assert rep["flags"] & 8  # the sequential pass ran
    print("IPSAT " + json.dumps(dict(case=case, report=rep, reference=meta)))
