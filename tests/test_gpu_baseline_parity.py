"""FP64 CUDA path vs the reference at the benchmark configurations.

The reference harness (the reference's own sources, compiled by oracle/Makefile)
runs the whole event on the host cores; the CUDA path is fed the same g^2 mu^2
maps and the same unit normals (the MT19937-64 stream the reference drew,
dumped by the harness), so both sides compute the same event.

  - Au+Au 256^2, L = 30 fm, b = 2 fm, Ny = 50, seeded Woods-Saxon nuclei,
    g^2 mu ~ sqrt(T_A), tau up to 0.4 fm (35 steps);
  - Pb+Pb 512^2, L = 40 fm, b = 6 fm, Ny = 50, tau up to 0.6 fm (77 steps).

Bounds (with the reference's own spread beside it: its -O2
and -Ofast builds differ at the Au+Au 256^2 event by 8.1e-11 in e on cells
above 1% of the maximum, 8.7e-10 above 0.1%, 7.4e-11 in eps_2, 3.5e-12 of the
maximum in T^{mu nu}, and 9e-9 in the tau = 0 links, where Newton stops at
sum |F| < 1e-6 after different iterations):
  - e per cell: 1e-10 relative on cells above 1% of max e, 1e-9 above 0.1%;
  - eps_2: 1e-10 relative; T^{mu nu}: 1e-11 of the component's maximum;
  - Wilson lines 1e-12; tau = 0 links 1e-7 (the Newton stopping spread);
  - Gauss-law violation and max |U^dag U - 1| are reported for both sides;
    Gauss is printed by the reference with 6 digits (1e-5 relative), the
    unitarity drift of the Taylor-2 link update agrees to 1e-12 absolute.
The harness runs with all host threads; its Newton restarts would draw from
one shared random stream across threads (Init.cpp:3448,3461), so the test
asserts that neither side restarted any link.
"""
import json
import os

import numpy as np
import pytest

import ipglasma_b200 as ipg

pytestmark = pytest.mark.gpu

CASES = {
    "AuAu256": dict(N=256, L=30.0, nucleus="Au", b=2.0, Ny=50, maxtime=0.4, seed=1000,
                    itmax=35),
    "PbPb512": dict(N=512, L=40.0, nucleus="Pb", b=6.0, Ny=50, maxtime=0.6, seed=1001,
                    itmax=77),
}


def unitarity(U: np.ndarray) -> float:
    d = np.einsum("nji,njk->nik", U.conj(), U) - np.eye(3)
    return float(np.abs(d).max())


def compare(case: str, ref_harness, tmp_path_factory):
    from ipglasma_b200.synthetic import make_event

    p = CASES[case]
    N, L, Ny = p["N"], p["L"], p["Ny"]
    A, B, _, _ = make_event(N, L, p["nucleus"], p["b"], seed=p["seed"])
    out = tmp_path_factory.mktemp(case)
    ref = ref_harness.run_harness(out, A, B, N, L, Ny, 2.0, 0.2, p["seed"], p["maxtime"],
                                  threads=os.cpu_count() or 1)
    assert ref.meta["itmax"] == p["itmax"]
    assert ref.meta["newton_restart_draws"] == 0
    xa, xb = ref.xi()
    cfg = ipg.Config(size=N, L=L, Ny=Ny, g=2.0, m=0.2, maxtime=p["maxtime"])
    with ipg.Event(cfg) as ev:
        ev.set_g2mu(A, B)
        ev.set_noise(xa, xb)
        rep = ev.init_fields()
        assert rep.newton_failed == 0 and rep.newton_restarted == 0
        err = {"VA": float(np.abs(ev.get_field(ipg.VA) - ref.mats("VA.bin")).max()),
               "VB": float(np.abs(ev.get_field(ipg.VB) - ref.mats("VB.bin")).max()),
               "tau0_Ux": float(np.abs(ev.get_field(ipg.UX) - ref.mats("tau0_Ux.bin")).max()),
               "tau0_Uy": float(np.abs(ev.get_field(ipg.UY) - ref.mats("tau0_Uy.bin")).max())}
        res = ev.run()
        eps, u4, _, T10 = ev.observables()
    obs = ref.observables()
    e = obs[0]
    for frac in (1e-2, 1e-3):
        m = e > frac * e.max()
        err[f"e_above_{frac:g}_max"] = float(np.max(np.abs(eps[m] - e[m]) / e[m]))
        err[f"cells_above_{frac:g}_max"] = int(m.sum())
    m = e > 1e-2 * e.max()
    err["u"] = float(np.abs(u4[:, m] - obs[1:5][:, m]).max())
    err["T10_of_max"] = max(float(np.abs(T10[k] - obs[5 + k]).max() / np.abs(obs[5 + k]).max())
                            for k in range(10))
    err["eps2_rel"] = abs(res.eccentricity[1] / ref.meta["eccentricity2"] - 1)
    ref_unit = max(unitarity(ref.mats("final_Ux.bin")), unitarity(ref.mats("final_Uy.bin")))
    report = dict(case=case, N=N, Ny=Ny, itmax=res.itmax, errors=err,
                  gauss_violation={"cuda": res.gauss_violation,
                                   "reference": ref.meta["gauss_violation"]},
                  unitarity_max={"cuda": res.unitarity_max, "reference": ref_unit},
                  eps2={"cuda": res.eccentricity[1], "reference": ref.meta["eccentricity2"]},
                  reference_s={k: v for k, v in ref.meta.items() if k.startswith("t_")},
                  reference_threads=os.cpu_count())
    print("PARITY " + json.dumps(report))
    assert res.itmax == p["itmax"]
    assert err["VA"] < 1e-12 and err["VB"] < 1e-12
    assert err["tau0_Ux"] < 1e-7 and err["tau0_Uy"] < 1e-7
    assert err["e_above_0.01_max"] < 1e-10
    assert err["e_above_0.001_max"] < 1e-9
    assert err["T10_of_max"] < 1e-11
    assert err["eps2_rel"] < 1e-10
    assert err["u"] < 1e-8
    assert abs(res.gauss_violation - ref.meta["gauss_violation"]) <= \
        1e-5 * ref.meta["gauss_violation"] + 1e-18
    assert abs(res.unitarity_max - ref_unit) < 1e-12
    return xa, xb, A, B, res, eps


@pytest.fixture(scope="module")
def auau256(ref_harness, tmp_path_factory):
    return compare("AuAu256", ref_harness, tmp_path_factory)


def test_AuAu256_Ny50_matches_reference(auau256):
    """The 256^2 Au+Au event, every stage and observable against the reference."""
    assert auau256 is not None


def test_PbPb512_Ny50_matches_reference(ref_harness, tmp_path_factory):
    """The 512^2 Pb+Pb event (77 steps) against the reference."""
    compare("PbPb512", ref_harness, tmp_path_factory)


def test_fp32_form_error_at_AuAu256(auau256):
    """The FP32 bulk form on the same 256^2 Au+Au event, against the FP64 form
    (which the tests above pin to the reference). E_T and eps_2 meet the
    1e-5 target (measured: a few 1e-6). The per-cell e error is the known
    miss of that target: its rms sits at a few 1e-5 (cells above 1% of the
    maximum) because the FP32 state itself, rounded once at tau = 0, already
    moves e by that much in this chaotic evolution; bounded here at 1e-4."""
    xa, xb, A, B, r64, e64 = auau256
    p = CASES["AuAu256"]
    cfg = ipg.Config(size=p["N"], L=p["L"], Ny=p["Ny"], g=2.0, m=0.2, maxtime=p["maxtime"],
                     precision=ipg.FP32)
    with ipg.Event(cfg) as ev:
        ev.set_g2mu(A, B)
        ev.set_noise(xa, xb)
        ev.init_fields()
        r32 = ev.run()
        e32 = ev.observables()[0]
    hot = e64 > 1e-2 * e64.max()
    rel = np.abs(e32[hot] - e64[hot]) / e64[hot]
    err = dict(E_T=abs(r32.E_T / r64.E_T - 1),
               eps2=abs(r32.eccentricity[1] / r64.eccentricity[1] - 1),
               e_rms=float(np.sqrt(np.mean(rel ** 2))), e_max=float(rel.max()),
               unitarity_fp32=r32.unitarity_max)
    print("FP32 " + json.dumps(err))
    assert err["E_T"] < 1e-5
    assert err["eps2"] < 1e-5
    assert err["e_rms"] < 1e-4
    assert r32.unitarity_max < 1e-6
    assert r32.gauss_violation <= r64.gauss_violation + 1e-10
