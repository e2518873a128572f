"""The CPU oracle is pinned to the reference: the C restatement against the
golden fixtures (made by the reference harness) and against the reference
harness run live; the FFTW/GSL subset against mathematics."""
import numpy as np
import pytest

CASES = ["blobs_n16", "blobs_n32"]


@pytest.mark.parametrize("case", CASES)
def test_noise_stream_bit_exact(oracle_port, golden, case):
    g = golden(case)
    N, Ny = g["meta"]["N"], g["meta"]["Ny"]
    xa, xb = oracle_port.noise(g["meta"]["seed"], N, Ny)
    assert np.array_equal(xa, g["xiA"]) and np.array_equal(xb, g["xiB"])


@pytest.mark.parametrize("case", CASES)
def test_wilson_lines_and_tau0_bit_exact(oracle_port, golden, case):
    g = golden(case)
    m = g["meta"]
    N, Ny, L = m["N"], m["Ny"], m["L"]
    VA = oracle_port.wilson_lines(N, Ny, L, m["g"], m["m"], 0.0, g["g2muA"], g["xiA"])
    VB = oracle_port.wilson_lines(N, Ny, L, m["g"], m["m"], 0.0, g["g2muB"], g["xiB"])
    assert np.array_equal(VA, g["VA"]) and np.array_equal(VB, g["VB"])
    Ux, Uy, pi, iters, restarts = oracle_port.tau0(N, m["g"], VA, VB)
    assert restarts == 0
    assert np.array_equal(Ux, g["tau0_Ux"]) and np.array_equal(Uy, g["tau0_Uy"])
    assert np.array_equal(pi, g["tau0_pi"])


@pytest.mark.parametrize("case", CASES)
def test_full_event_matches_golden(oracle_port, golden, case):
    g = golden(case)
    m = g["meta"]
    r = oracle_port.run_event(m["N"], m["Ny"], m["L"], m["g"], m["m"], 0.0, m["maxtime"],
                              g["g2muA"], g["g2muB"], g["xiA"], g["xiB"])
    obs = g["obs"]
    assert r["itmax"] == m["itmax"]
    # diagonal T^{mu nu} bit-exact, the rest within rounding of the
    # reassociated off-diagonal expressions
    for k in range(4):
        assert np.array_equal(r["T10"][k], obs[5 + k])
    for k in range(4, 10):
        assert np.abs(r["T10"][k] - obs[5 + k]).max() <= 1e-13 * np.abs(obs[5 + k]).max()
    e = obs[0]
    mask = e > 1e-3 * e.max()
    assert np.max(np.abs(r["eps"][mask] - e[mask]) / e[mask]) < 1e-12
    assert abs(r["ecc2"] - m["eccentricity2"]) < 1e-12 * m["eccentricity2"]
    assert abs(r["gauss"] - m["gauss_violation"]) <= 1e-6 * m["gauss_violation"]


def test_steps_match_golden(oracle_port, golden):
    g = golden("blobs_n16")
    m = g["meta"]
    N, n = m["N"], m["N"] ** 2
    f = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.complex128)).view(np.float64).ravel().copy()
    Ux, Uy, pi = f(g["tau0_Ux"]), f(g["tau0_Uy"]), f(g["tau0_pi"])
    E1, E2, phi = np.zeros(18 * n), np.zeros(18 * n), np.zeros(18 * n)
    lib = oracle_port.lib()
    P = oracle_port._p
    dtau, gg = m["dtau"], m["g"]
    lib.ipgo_evolve_phi(N, dtau, 0.0, P(phi), P(pi))
    lib.ipgo_evolve_u(N, gg, dtau, 0.0, P(Ux), P(Uy), P(E1), P(E2))
    for it in range(1, m["steps_mode_steps"] + 1):
        tau = it * dtau
        lib.ipgo_evolve_pi(N, dtau, tau, P(Ux), P(Uy), P(phi), P(pi))
        lib.ipgo_evolve_e(N, gg, dtau, tau, P(Ux), P(Uy), P(phi), P(E1), P(E2))
        lib.ipgo_evolve_phi(N, dtau, tau, P(phi), P(pi))
        lib.ipgo_evolve_u(N, gg, dtau, tau, P(Ux), P(Uy), P(E1), P(E2))
    mats = lambda a: a.view(np.complex128).reshape(n, 3, 3)
    assert np.array_equal(mats(Ux), g["steps_Ux"])
    assert np.array_equal(mats(E2), g["steps_E2"])
    assert np.array_equal(mats(phi), g["steps_phi"])
    assert np.array_equal(mats(pi), g["steps_pi"])


def test_oracle_matches_live_reference(oracle_port, ref_harness, tmp_path):
    """A case not in the fixtures, checked against the reference run here."""
    from ipglasma_b200.synthetic import gaussian_blobs

    N, L, Ny, seed = 16, 2.0, 3, 7
    A, B = gaussian_blobs(N, L, 2.0, 1.3)
    ref = ref_harness.run_harness(tmp_path / "ref", A, B, N, L, Ny, 2.0, 0.2, seed, 0.15)
    assert ref.meta["newton_restart_draws"] == 0
    xa, xb = oracle_port.noise(seed, N, Ny)
    r = oracle_port.run_event(N, Ny, L, 2.0, 0.2, 0.0, 0.15, A, B, xa, xb)
    assert np.array_equal(r["Ux"], ref.mats("tau0_Ux.bin"))
    obs = ref.observables()
    assert np.abs(r["T10"] - obs[5:15]).max() <= 1e-13 * np.abs(obs[5:15]).max()


# ---------------------------------------------------------------------------
# the FFTW / GSL subset against mathematics
# ---------------------------------------------------------------------------
def test_expm_unitary_and_matches_series(oracle_port):
    rng = np.random.default_rng(3)
    t = np.zeros((8, 3, 3), dtype=complex)
    t[0][0, 1] = t[0][1, 0] = 0.5
    t[1][0, 1], t[1][1, 0] = -0.5j, 0.5j
    t[2][0, 0], t[2][1, 1] = 0.5, -0.5
    t[3][0, 2] = t[3][2, 0] = 0.5
    t[4][0, 2], t[4][2, 0] = -0.5j, 0.5j
    t[5][1, 2] = t[5][2, 1] = 0.5
    t[6][1, 2], t[6][2, 1] = -0.5j, 0.5j
    t[7] = np.diag([1, 1, -2]) / (2 * np.sqrt(3))
    for scale in (1e-3, 0.3, 2.0):
        q = rng.normal(size=8) * scale
        U = oracle_port.expm(q)
        H = np.einsum("a,aij->ij", q, t)
        w, v = np.linalg.eigh(H)
        ref = (v * np.exp(1j * w)) @ v.conj().T
        assert np.abs(U - ref).max() < 1e-13
        assert np.abs(U @ U.conj().T - np.eye(3)).max() < 1e-13
        assert abs(np.linalg.det(U) - 1) < 1e-13
    # Q = 0: coefficients are NaN, mapped to 0, identity returned (Matrix.cpp:416-424)
    assert np.array_equal(oracle_port.expm(np.zeros(8)), np.eye(3))


def test_eig4_residuals():
    import ctypes as ct
    import subprocess
    import tempfile
    from pathlib import Path

    root = Path(__file__).resolve().parent.parent
    src = """
#include <stdio.h>
#include <stdlib.h>
#include "gsl/ipg_eig4.h"
int main(void) {
  srand(11); double worst = 0;
  for (int t = 0; t < 20000; t++) {
    double a[16], er[4], ei[4], vr[16], vi[16];
    for (int i = 0; i < 16; i++) a[i] = rand() / (double)RAND_MAX - 0.5;
    if (t % 4 == 0) for (int i = 0; i < 4; i++) for (int j = 0; j < i; j++) a[4*i+j] = a[4*j+i];
    if (ipg_eig4(a, er, ei, vr, vi) < 0) { printf("fail\\n"); return 1; }
    for (int k = 0; k < 4; k++) for (int i = 0; i < 4; i++) {
      double rr = 0, ri = 0;
      for (int j = 0; j < 4; j++) { rr += a[4*i+j]*vr[4*k+j]; ri += a[4*i+j]*vi[4*k+j]; }
      rr -= er[k]*vr[4*k+i] - ei[k]*vi[4*k+i]; ri -= er[k]*vi[4*k+i] + ei[k]*vr[4*k+i];
      double r = sqrt(rr*rr + ri*ri); if (r > worst) worst = r;
    }
  }
  printf("%g\\n", worst); return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = Path(d) / "t.c"
        c.write_text(src)
        exe = Path(d) / "t"
        subprocess.run(["gcc", "-O2", "-I", str(root / "oracle" / "shim"), str(c), "-o", str(exe),
                        "-lm"], check=True)
        out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    assert float(out) < 1e-12


def test_shim_fft_against_numpy(tmp_path):
    import subprocess
    from pathlib import Path

    root = Path(__file__).resolve().parent.parent
    src = r"""
#include <stdio.h>
#include <stdlib.h>
#include "fftw3.h"
int main(int argc, char **argv) {
  int n0 = atoi(argv[1]), n1 = atoi(argv[2]);
  fftw_complex *a = fftw_malloc(sizeof(fftw_complex) * n0 * n1);
  fftw_plan p = fftw_plan_dft_2d(n0, n1, a, a, FFTW_FORWARD, FFTW_MEASURE);
  FILE *f = fopen(argv[3], "rb"); fread(a, sizeof(fftw_complex), n0 * n1, f); fclose(f);
  fftw_execute(p);
  f = fopen(argv[4], "wb"); fwrite(a, sizeof(fftw_complex), n0 * n1, f); fclose(f);
  return 0;
}
"""
    c = tmp_path / "f.c"
    c.write_text(src)
    exe = tmp_path / "f"
    subprocess.run(["gcc", "-O2", "-I", str(root / "oracle" / "shim"), str(c),
                    str(root / "oracle" / "shim" / "shim_fftw.c"), "-o", str(exe), "-lm"], check=True)
    rng = np.random.default_rng(0)
    for n0, n1 in ((16, 16), (8, 32), (12, 10)):
        x = rng.normal(size=(n0, n1)) + 1j * rng.normal(size=(n0, n1))
        x.astype(np.complex128).tofile(tmp_path / "in.bin")
        subprocess.run([str(exe), str(n0), str(n1), str(tmp_path / "in.bin"),
                        str(tmp_path / "out.bin")], check=True)
        y = np.fromfile(tmp_path / "out.bin", dtype=np.complex128).reshape(n0, n1)
        assert np.abs(y - np.fft.fft2(x)).max() < 1e-12 * np.abs(y).max()
