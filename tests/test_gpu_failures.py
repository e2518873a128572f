"""Failure paths of the C ABI, made to fire from the host, and the device
noise generator's statistics.

The failures are injected on the host only (a NaN in the caller's noise, an
iteration limit the Newton solve cannot meet); nothing here makes a kernel
fault or wait forever.
"""
import numpy as np
import pytest

import ipglasma_b200 as ipg

pytestmark = pytest.mark.gpu

NAN, NONCONVERGED = 4, 3


def blobs_event(N=32, L=6.0, Ny=3, **kw):
    from ipglasma_b200.synthetic import gaussian_blobs

    A, B = gaussian_blobs(N, L)
    ev = ipg.Event(ipg.Config(size=N, L=L, Ny=Ny, maxtime=0.2, **kw))
    ev.set_g2mu(A, B)
    return ev


def test_nan_in_the_fields_is_reported():
    """A NaN in a field the caller loads (ipg_set_field) spreads through the
    evolution into e; ipg_run reports IPG_ERR_NAN instead of returning
    numbers."""
    N = 32
    with blobs_event(N, seed=5) as ev:
        ev.use_device_noise()
        ev.init_fields()
        state = {f: ev.get_field(f) for f in (ipg.UX, ipg.UY, ipg.E1, ipg.E2, ipg.PHI, ipg.PI)}
    state[ipg.PI][N * N // 2 + N // 2, 0, 0] = np.nan
    with ipg.Event(ipg.Config(size=N, L=6.0, Ny=3, maxtime=0.2)) as ev:
        for f, v in state.items():
            ev.set_field(f, v)
        ev.mark_initialized()
        with pytest.raises(ipg.IPGError) as exc:
            ev.run()
        assert exc.value.status == NAN
        assert "non-finite" in str(exc.value)


def test_nan_in_the_noise_is_absorbed_like_the_reference():
    """A NaN in the colour-charge noise reaches the exponent of a Wilson-line
    sheet, where the reference's exponential maps NaN coefficients to 0
    (Matrix.cpp:416-424): that sheet's factor is the identity wherever the
    NaN spread, the fields stay finite and the run completes."""
    N, Ny = 32, 3
    rng = np.random.default_rng(5)
    xa = rng.standard_normal(Ny * N * N * 8)
    xb = rng.standard_normal(Ny * N * N * 8)
    xa[12345] = np.nan
    with blobs_event(N, Ny=Ny) as ev:
        ev.set_noise(xa, xb)
        ev.init_fields(allow_nonconverged=True)
        assert np.all(np.isfinite(ev.get_field(ipg.VA)))
        res = ev.run()
        assert np.isfinite(res.E_T)


def test_newton_iteration_limit_reports_nonconverged_with_fields_set():
    """newton_max_iterations = 1 and newton_max_restarts = 1: every link
    whose starting residual is above the tolerance ends at its best estimate.
    ipg_init_fields returns
    IPG_ERR_NEWTON_NONCONVERGED, the report counts the links, and the fields
    are still set (finite, unitary), so the caller may go on."""
    with blobs_event(newton_max_iterations=1, newton_max_restarts=1, seed=3) as ev:
        ev.use_device_noise()
        with pytest.raises(ipg.IPGError) as exc:
            ev.init_fields()
        assert exc.value.status == NONCONVERGED
    with blobs_event(newton_max_iterations=1, newton_max_restarts=1, seed=3) as ev:
        ev.use_device_noise()
        rep = ev.init_fields(allow_nonconverged=True)
        assert rep.newton_links == 2 * 32 * 32
        assert 0 < rep.newton_failed <= rep.newton_links
        U = ev.get_field(ipg.UX)
        assert np.all(np.isfinite(U))
        assert np.abs(np.einsum("nji,njk->nik", U.conj(), U) - np.eye(3)).max() < 1e-12
        res = ev.run()
        assert np.isfinite(res.E_T)


def test_converged_run_has_no_failures():
    with blobs_event(seed=3) as ev:
        ev.use_device_noise()
        rep = ev.init_fields()
        assert rep.newton_failed == 0
        _, status = ev.newton_iterations()
        # 0: converged, 1: converged after a random restart
        assert np.all((status == 0) | (status == 1))


def test_device_noise_is_the_noise_the_wilson_lines_use():
    """ipg_draw_device_noise returns the draws of the in-kernel generator:
    fed back through ipg_set_noise they give the same Wilson lines."""
    N, Ny = 64, 4
    with blobs_event(N, 7.5, Ny, seed=99) as ev:
        ev.use_device_noise()
        ev.init_fields()
        va, vb = ev.get_field(ipg.VA), ev.get_field(ipg.VB)
        xa, xb = ev.draw_device_noise(0), ev.draw_device_noise(1)
    with blobs_event(N, 7.5, Ny, seed=99) as ev:
        ev.set_noise(xa, xb)
        ev.init_fields()
        assert np.array_equal(ev.get_field(ipg.VA), va)
        assert np.array_equal(ev.get_field(ipg.VB), vb)


def test_device_noise_moments_and_distribution():
    """Philox4x32-10 + Box-Muller draws (replacing the reference's serial
    MT19937-64 + polar Gauss stream, Random.cpp:178-204) are unit normals:
    moments within 5 standard errors, a Kolmogorov-Smirnov test against
    N(0, 1), no correlation between colours, neighbouring sites, sheets or
    nuclei, and different keys give different streams."""
    from scipy import stats

    N, Ny = 256, 4
    with blobs_event(N, 30.0, Ny, seed=2024) as ev:
        xa = ev.draw_device_noise(0)
        xb = ev.draw_device_noise(1)
        ev.reseed(2025)
        xc = ev.draw_device_noise(0, 0, 1)
    z = xa.ravel()
    n = z.size  # 2.1 M
    se = 1.0 / np.sqrt(n)
    assert abs(z.mean()) < 5 * se
    assert abs(z.var() - 1.0) < 5 * np.sqrt(2.0) * se
    assert abs(stats.skew(z)) < 5 * np.sqrt(6.0) * se
    assert abs(stats.kurtosis(z)) < 5 * np.sqrt(24.0) * se
    # the float Box-Muller radius caps |z| at sqrt(-2 ln 2^-24) = 5.77
    assert np.abs(z).max() < 5.8
    ks = stats.kstest(z[::7], "norm")
    assert ks.pvalue > 1e-4, ks
    per_colour = xa.reshape(-1, 8)
    c = np.corrcoef(per_colour.T)
    m = per_colour.shape[0]
    assert np.abs(c - np.eye(8)).max() < 5 / np.sqrt(m)
    for u, v in ((xa[:, :-1, :], xa[:, 1:, :]),           # neighbouring sites
                 (xa[:-1], xa[1:]),                         # sheets
                 (xa, xb),                                  # nuclei
                 (xa[:1], xc)):                             # keys
        r = np.corrcoef(u.ravel(), v.ravel())[0, 1]
        assert abs(r) < 5 / np.sqrt(u.size), r
    assert not np.array_equal(xa[:1], xc)
