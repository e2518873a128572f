"""CUDA path vs the reference (live harness and golden fixtures) on the GPU.

Tolerances, and why:
  - Wilson lines, tau=0 links and fields, leapfrog steps: 1e-12 absolute on
    O(1) matrices (measured 1e-15 .. 1e-14: only libm vs CUDA transcendentals
    and FMA contraction differ).
  - T^{mu nu}: 1e-11 relative to the largest component (measured ~7e-13).
  - e(x,y) per cell: 1e-10 relative where e > 1e-2 max e, and 1e-9 where
    e > 1e-3 max e. In the weak-field cells the reference itself moves by
    1.3e-10 between its -O2 and -Ofast (finite-math off) builds, because
    T^tautau there is a difference of O(1) numbers (3 - Re tr U_plaq).
  - epsilon_2: 1e-10 relative; Gauss-law violation: the reference prints 6
    significant digits, so 1e-5 relative.
"""
import numpy as np
import pytest

import ipglasma_b200 as ipg

pytestmark = pytest.mark.gpu

FIELDS = [("Ux", ipg.UX), ("Uy", ipg.UY), ("E1", ipg.E1), ("E2", ipg.E2),
          ("phi", ipg.PHI), ("pi", ipg.PI)]


def event_from(golden_case: dict, precision=ipg.FP64) -> ipg.Event:
    m = golden_case["meta"]
    cfg = ipg.Config(size=m["N"], L=m["L"], Ny=m["Ny"], g=m["g"], m=m["m"],
                     maxtime=m["maxtime"], precision=precision)
    ev = ipg.Event(cfg)
    ev.set_g2mu(golden_case["g2muA"], golden_case["g2muB"])
    ev.set_noise(golden_case["xiA"], golden_case["xiB"])
    return ev


def check_observables(ev, obs, meta, result):
    eps, u4, pi10, T10 = ev.observables()
    for k in range(10):
        scale = np.abs(obs[5 + k]).max()
        assert np.abs(T10[k] - obs[5 + k]).max() <= 1e-11 * scale, k
    e = obs[0]
    for frac, tol in ((1e-2, 1e-10), (1e-3, 1e-9)):
        mask = e > frac * e.max()
        assert np.max(np.abs(eps[mask] - e[mask]) / e[mask]) < tol, frac
    mask = e > 1e-2 * e.max()
    assert np.abs(u4[:, mask] - obs[1:5][:, mask]).max() < 1e-8
    assert abs(result.eccentricity[1] - meta["eccentricity2"]) < 1e-10 * meta["eccentricity2"]
    assert abs(result.gauss_violation - meta["gauss_violation"]) <= 1e-5 * meta["gauss_violation"]


@pytest.mark.parametrize("case", ["blobs_n16", "blobs_n32"])
def test_stages_match_golden(golden, case):
    g = golden(case)
    with event_from(g) as ev:
        rep = ev.init_fields()
        assert rep.newton_failed == 0 and rep.newton_restarted == 0
        assert np.abs(ev.get_field(ipg.VA) - g["VA"]).max() < 1e-12
        assert np.abs(ev.get_field(ipg.VB) - g["VB"]).max() < 1e-12
        assert np.abs(ev.get_field(ipg.UX) - g["tau0_Ux"]).max() < 1e-12
        assert np.abs(ev.get_field(ipg.UY) - g["tau0_Uy"]).max() < 1e-12
        assert np.abs(ev.get_field(ipg.PI) - g["tau0_pi"]).max() < 1e-12 * np.abs(g["tau0_pi"]).max()
        res = ev.run()
        assert res.itmax == g["meta"]["itmax"]
        check_observables(ev, g["obs"], g["meta"], res)
        assert np.abs(ev.get_field(ipg.UX) - g["final_Ux"]).max() < 1e-12
        assert np.abs(ev.get_field(ipg.E1) - g["final_E1"]).max() < 1e-12 * np.abs(g["final_E1"]).max()


def test_leapfrog_steps_from_reference_state(golden):
    """Evolution only: start from the reference's tau=0 state."""
    g = golden("blobs_n16")
    m = g["meta"]
    cfg = ipg.Config(size=m["N"], L=m["L"], Ny=m["Ny"], g=m["g"], m=m["m"], maxtime=m["maxtime"])
    with ipg.Event(cfg) as ev:
        zero = np.zeros_like(g["tau0_Ux"])
        ev.set_field(ipg.UX, g["tau0_Ux"])
        ev.set_field(ipg.UY, g["tau0_Uy"])
        ev.set_field(ipg.PI, g["tau0_pi"])
        for f in (ipg.E1, ipg.E2, ipg.PHI):
            ev.set_field(f, zero)
        ev.mark_initialized()
        ev.evolve(m["steps_mode_steps"])
        for name, which in (("Ux", ipg.UX), ("E2", ipg.E2), ("phi", ipg.PHI), ("pi", ipg.PI)):
            ref = g[f"steps_{name}"]
            assert np.abs(ev.get_field(which) - ref).max() < 1e-12 * max(1.0, np.abs(ref).max()), name


def test_live_reference_event(ref_harness, tmp_path):
    """A fresh case (not in the fixtures) run through the reference on this box."""
    from ipglasma_b200.synthetic import gaussian_blobs

    N, L, Ny, seed, maxtime = 64, 7.5, 4, 1, 0.2
    A, B = gaussian_blobs(N, L, 2.0, 1.5)
    ref = ref_harness.run_harness(tmp_path / "ref", A, B, N, L, Ny, 2.0, 0.2, seed, maxtime)
    assert ref.meta["newton_restart_draws"] == 0
    xa, xb = ref.xi()
    cfg = ipg.Config(size=N, L=L, Ny=Ny, g=2.0, m=0.2, maxtime=maxtime)
    with ipg.Event(cfg) as ev:
        ev.set_g2mu(A, B)
        ev.set_noise(xa, xb)
        ev.init_fields()
        assert np.abs(ev.get_field(ipg.UX) - ref.mats("tau0_Ux.bin")).max() < 1e-12
        res = ev.run()
        check_observables(ev, ref.observables(), dict(ref.meta, eccentricity2=ref.meta["eccentricity2"]), res)


def test_oracle_port_agrees_on_gpu_box(oracle_port, golden):
    """The C restatement gives the same answer on the GPU box's host cores."""
    g = golden("blobs_n16")
    m = g["meta"]
    r = oracle_port.run_event(m["N"], m["Ny"], m["L"], m["g"], m["m"], 0.0, m["maxtime"],
                              g["g2muA"], g["g2muB"], g["xiA"], g["xiB"])
    with event_from(g) as ev:
        ev.init_fields()
        res = ev.run()
        eps, _, _, T10 = ev.observables()
    assert np.abs(T10 - r["T10"]).max() <= 1e-11 * np.abs(r["T10"]).max()
    assert abs(res.eccentricity[1] - r["ecc2"]) < 1e-10 * r["ecc2"]


def test_device_noise_is_deterministic_and_gaussian():
    from ipglasma_b200.synthetic import gaussian_blobs

    N, L, Ny = 64, 7.5, 4
    A, B = gaussian_blobs(N, L)
    outs = []
    for _ in range(2):
        with ipg.Event(ipg.Config(size=N, L=L, Ny=Ny, maxtime=0.1, seed=99)) as ev:
            ev.set_g2mu(A, B)
            ev.use_device_noise()
            ev.init_fields()
            outs.append(ev.get_field(ipg.VA))
    assert np.array_equal(outs[0], outs[1])
    V = outs[0]
    assert np.abs(np.einsum("nij,nkj->nik", V, V.conj()) - np.eye(3)).max() < 1e-12


def test_full_size_invariants_fp64():
    """Size-independent properties at the Pb+Pb 512^2 workload: Gauss law holds,
    links stay unitary to the Taylor-2 drift, T^tautau >= 0 in the bulk, the
    Landau frame is found in the interaction region, energy is finite."""
    from ipglasma_b200.synthetic import make_event

    N, L = 512, 40.0
    A, B, _, _ = make_event(N, L, "Pb", 6.0, seed=11)
    with ipg.Event(ipg.Config(size=N, L=L, Ny=50, maxtime=0.6, seed=5)) as ev:
        ev.set_g2mu(A, B)
        ev.use_device_noise()
        rep = ev.init_fields()
        assert rep.newton_failed == 0
        res = ev.run()
        eps, u4, _, T10 = ev.observables()
    assert res.itmax == 77
    assert res.gauss_violation < 1e-6
    assert res.unitarity_max < 1e-5
    assert np.isfinite(res.E_T) and res.E_T > 0
    hot = T10[0] > 1e-2 * T10[0].max()
    assert np.all(eps[hot] > 0)
    # u is a unit time-like vector: u^tau^2 - u_x^2 - u_y^2 - tau^2 u_eta^2 = 1
    tau = res.tau_final
    norm = u4[0] ** 2 - u4[1] ** 2 - u4[2] ** 2 - tau * tau * u4[3] ** 2
    assert np.abs(norm[hot] - 1).max() < 1e-8


def test_fp32_form_error_against_fp64():
    """The FP32 bulk form against the plain FP64 form on the same event
    (same noise, same FP64 initial conditions). Bounds, from the 512^2 Pb+Pb
    measurements (E_T 4e-6, eps2 1e-6 to 6e-6, e rms 5e-5) with margin for a
    smaller lattice: E_T and eps2 to 1e-4, e per cell (cells above 1% of the
    maximum) to 1e-3 rms, Gauss law and unitarity at FP32 rounding."""
    from ipglasma_b200.synthetic import make_event

    # O+O in a 10 fm box: the nuclei fit, so the clamped edges see no field
    N, L = 128, 10.0
    A, B, _, _ = make_event(N, L, "O", 1.0, seed=3)
    out = {}
    for prec in (ipg.FP64, ipg.FP32):
        with ipg.Event(ipg.Config(size=N, L=L, Ny=10, maxtime=0.4, seed=9,
                                  precision=prec)) as ev:
            ev.set_g2mu(A, B)
            ev.use_device_noise()
            ev.init_fields()
            res = ev.run()
            out[prec] = (res, ev.observables()[0])
    (r64, e64), (r32, e32) = out[ipg.FP64], out[ipg.FP32]
    assert abs(r32.E_T / r64.E_T - 1) < 1e-4
    assert abs(r32.eccentricity[1] / r64.eccentricity[1] - 1) < 1e-4
    hot = e64 > 1e-2 * e64.max()
    rel = np.abs(e32[hot] - e64[hot]) / e64[hot]
    assert np.sqrt(np.mean(rel ** 2)) < 1e-3
    # FP32 adds no Gauss-law violation beyond the FP64 form's plus rounding
    assert r32.gauss_violation <= r64.gauss_violation + 1e-10
    assert r32.unitarity_max < 1e-6


def test_g2mu_from_nucleons_matches_host_map():
    """ipg_set_nuclei builds on the device the same g2mu maps as the host
    generator (separable Gaussian thickness, Q_s ~ sqrt(T) scaling)."""
    from ipglasma_b200.synthetic import make_event

    N, L = 128, 20.0
    A, B, nA, nB = make_event(N, L, "Pb", 4.0, seed=7)  # positions already shifted
    with ipg.Event(ipg.Config(size=N, L=L, Ny=2, maxtime=0.1)) as ev:
        ev.set_nuclei(nA, nB, b=0.0)
        g = ev.g2mu()
    for dev, host in ((g[0], A), (g[1], B)):
        assert np.abs(dev - host).max() <= 1e-12 * host.max()


_DUMP = r'''
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
import ipglasma_b200 as ipg
from ipglasma_b200.synthetic import make_event
out = {}
for prec, tag in ((ipg.FP64, "d"), (ipg.FP32, "s")):
    for N, L in ((64, 20.0), (128, 24.0)):
        gA, gB, _, _ = make_event(N, L, "Pb", 4.0, 7)
        cfg = ipg.Config(size=N, L=L, Ny=12, maxtime=0.2, precision=prec, seed=5)
        with ipg.Event(cfg) as ev:
            ev.set_g2mu(gA, gB); ev.use_device_noise(); ev.init_fields(); ev.run()
            for name, f in (("ux", ipg.UX), ("uy", ipg.UY), ("e1", ipg.E1), ("e2", ipg.E2),
                            ("phi", ipg.PHI), ("pi", ipg.PI)):
                out[f"{tag}{name}{N}"] = ev.get_field(f)
np.savez(sys.argv[2], **out)
'''


def test_tile_kernels_match_plain_load_kernels_bit_for_bit(tmp_path):
    """The TMA-staged tile kernels (default) and the plain-load kernels
    (IPG_FP32_KERNEL=pair, IPG_FP64_KERNEL=site) run the same per-site code,
    so whole events agree to the bit in both forms, edge tiles included."""
    import os
    import subprocess
    import sys
    from pathlib import Path
    root = str(Path(__file__).resolve().parent.parent)
    script = tmp_path / "dump.py"
    script.write_text(_DUMP)
    runs = {}
    for tag, env in (("tile", {}), ("plain", {"IPG_FP32_KERNEL": "pair", "IPG_FP64_KERNEL": "site"})):
        e = dict(os.environ)
        e.pop("IPG_FP32_KERNEL", None)
        e.pop("IPG_FP64_KERNEL", None)
        e.update(env)
        out = tmp_path / f"{tag}.npz"
        subprocess.run([sys.executable, str(script), root, str(out)], env=e, check=True,
                       timeout=600)
        runs[tag] = np.load(out)
    a, b = runs["tile"], runs["plain"]
    assert sorted(a.files) == sorted(b.files) and len(a.files) == 24
    for k in a.files:
        assert np.array_equal(a[k], b[k]), k
