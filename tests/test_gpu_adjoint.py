"""Adjoint of the evolution (ipg_forward / ipg_backward): gradients of E_T and
of the T^tautau-weighted eps2 with respect to the tau = 0 fields agree with
central finite differences along random directions, and time reversal between
checkpoints gives the same gradient as storing every step (and stepping each
state into its own slot)."""
import numpy as np
import pytest

import ipglasma_b200 as ipg
from ipglasma_b200.synthetic import gaussian_blobs

pytestmark = pytest.mark.gpu

FIELDS = (ipg.UX, ipg.UY, ipg.E1, ipg.E2, ipg.PHI, ipg.PI)


def fresh(N=32, L=4.0, maxtime=0.25, seed=3):
    ev = ipg.Event(ipg.Config(size=N, L=L, Ny=4, maxtime=maxtime, precision=ipg.FP64,
                              seed=seed))
    A, B = gaussian_blobs(N, L)
    ev.set_g2mu(A, B)
    ev.use_device_noise()
    ev.init_fields()
    return ev


def herm(m):
    return 0.5 * (m + np.conj(np.swapaxes(m, -1, -2)))


def random_direction(rng, n):
    d = {}
    for f in FIELDS:
        z = rng.standard_normal((n, 3, 3)) + 1j * rng.standard_normal((n, 3, 3))
        if f in (ipg.E1, ipg.E2, ipg.PHI, ipg.PI):
            z = herm(z)
            if f in (ipg.E1, ipg.E2):
                tr = np.trace(z, axis1=1, axis2=2) / 3.0
                z = z - tr[:, None, None] * np.eye(3)
        d[f] = z
    return d


def loss_at(ev, state, direction, h, w):
    for f in FIELDS:
        ev.set_field(f, state[f] + h * direction[f])
    ev.mark_initialized()
    et, e2 = ev.forward(5)
    return w[0] * et + w[1] * e2


@pytest.fixture(scope="module")
def setup():
    ev = fresh()
    state = {f: ev.get_field(f) for f in FIELDS}
    yield ev, state
    ev.close()


def test_forward_energy_equals_run():
    ev = fresh()
    et, e2 = ev.forward(5)
    r = ev.run()
    assert et == pytest.approx(r.E_T, rel=1e-12)
    assert 0 < e2 < 1
    ev.close()


@pytest.mark.parametrize("w", [(1.0, 0.0), (0.0, 1.0)], ids=["E_T", "eps2"])
def test_gradient_matches_finite_differences(setup, w):
    ev, state = setup
    for f in FIELDS:
        ev.set_field(f, state[f])
    ev.mark_initialized()
    ev.forward(5)
    grad = ev.backward(*w)
    rng = np.random.default_rng(11)
    n = ev.n
    # the central difference converges as h^2 onto the adjoint value (measured:
    # relative gap 3e-5 at h = 1e-5, 3e-7 at 1e-6 for eps2); 1e-6 keeps the
    # truncation and the rounding of the difference both below 1e-6
    h = 1e-6
    for _ in range(3):
        d = random_direction(rng, n)
        directional = sum(float(np.sum((np.conj(grad[f]) * d[f]).real)) for f in FIELDS)
        fd = (loss_at(ev, state, d, h, w) - loss_at(ev, state, d, -h, w)) / (2 * h)
        assert directional == pytest.approx(fd, rel=2e-6, abs=1e-9 * max(1.0, abs(fd))), \
            (directional, fd)


def test_time_reversal_matches_stored_steps(setup):
    ev, state = setup
    out = []
    for k in (1, 1000):
        for f in FIELDS:
            ev.set_field(f, state[f])
        ev.mark_initialized()
        ev.forward(k)
        out.append(ev.backward(1.0, 0.5))
    for f in FIELDS:
        a, b = out[0][f], out[1][f]
        scale = max(np.abs(a).max(), 1e-300)
        assert np.abs(a - b).max() <= 1e-8 * scale, f


def test_stored_states_allow_repeated_backward(setup):
    """With every state kept (checkpoint_every = 1) the reverse sweep
    overwrites nothing: a second backward with other weights needs no new
    forward and equals the sum of the single-loss gradients."""
    ev, state = setup
    for f in FIELDS:
        ev.set_field(f, state[f])
    ev.mark_initialized()
    ev.forward(1)
    g_et = ev.backward(1.0, 0.0)
    g_e2 = ev.backward(0.0, 1.0)
    g_both = ev.backward(1.0, 1.0)
    for f in FIELDS:
        scale = max(np.abs(g_both[f]).max(), 1e-300)
        assert np.abs(g_et[f] + g_e2[f] - g_both[f]).max() <= 1e-10 * scale, f


# ---- through the initial conditions: g2mu and rho ---------------------------

def input_event(N=32, L=4.0, Ny=4, maxtime=0.25):
    ev = ipg.Event(ipg.Config(size=N, L=L, Ny=Ny, maxtime=maxtime, precision=ipg.FP64,
                              seed=5, newton_tolerance=1e-13))
    A, B = gaussian_blobs(N, L)
    rng = np.random.default_rng(2)
    xi = rng.standard_normal((2, Ny, N * N, 8))
    return ev, A, B, xi


def input_loss(ev, A, B, xi, w):
    ev.set_g2mu(A, B)
    ev.set_noise(xi[0], xi[1])
    rep = ev.init_fields()
    assert rep.newton_restarted == 0 and rep.newton_failed == 0
    et, e2 = ev.forward(5)
    return w[0] * et + w[1] * e2


@pytest.mark.parametrize("w", [(1.0, 0.0), (0.0, 1.0)], ids=["E_T", "eps2"])
def test_input_gradients_match_finite_differences(w):
    ev, A, B, xi = input_event()
    input_loss(ev, A, B, xi, w)
    g = ev.backward(*w, inputs=True, rho=True)
    rng = np.random.default_rng(17)
    h = 3e-6
    # g2mu of nucleus A and B: relative perturbations
    dA = A * rng.uniform(-1, 1, A.shape)
    dB = B * rng.uniform(-1, 1, B.shape)
    directional = float(np.sum(g["g2mu"][0] * dA) + np.sum(g["g2mu"][1] * dB))
    fd = (input_loss(ev, A + h * dA, B + h * dB, xi, w)
          - input_loss(ev, A - h * dA, B - h * dB, xi, w)) / (2 * h)
    assert directional == pytest.approx(fd, rel=5e-5), ("g2mu", directional, fd)
    # the noise: rho = g sqrt(g2mu/Ny) xi, so d rho = amp d xi
    dxi = rng.standard_normal(xi.shape)
    amp = np.stack([2.0 * np.sqrt(A / xi.shape[1]), 2.0 * np.sqrt(B / xi.shape[1])])
    directional = float(np.sum(g["rho"] * amp[:, None, :, None] * dxi))
    fd = (input_loss(ev, A, B, xi + h * dxi, w) - input_loss(ev, A, B, xi - h * dxi, w)) / (2 * h)
    assert directional == pytest.approx(fd, rel=5e-5), ("rho", directional, fd)
    ev.close()


def test_input_gradients_need_initial_conditions():
    ev = fresh()
    for f in FIELDS:
        ev.set_field(f, ev.get_field(f))
    ev.mark_initialized()
    ev.forward(5)
    with pytest.raises(ipg.IPGError):
        ev.backward(1.0, 0.0, inputs=True)
    ev.close()


def _event(prec, N=32, L=4.0, maxtime=0.25, seed=3):
    ev = ipg.Event(ipg.Config(size=N, L=L, Ny=4, maxtime=maxtime, precision=prec, seed=seed,
                              newton_tolerance=1e-12))
    A, B = gaussian_blobs(N, L)
    ev.set_g2mu(A, B)
    rng = np.random.default_rng(seed)
    n = N * N
    ev.set_noise(rng.standard_normal(4 * n * 8), rng.standard_normal(4 * n * 8))
    ev.init_fields()
    return ev


@pytest.mark.parametrize("k", [1, 4], ids=["every_state", "checkpoints"])
def test_fp32_adjoint_matches_fp64_adjoint(k):
    """The FP32 adjoint (an FP32 context: the FP32 bulk form's forward, the
    reverse sweep in FP32 on its states, every state kept or checkpoints with
    the segments recomputed; the initial conditions' adjoint in FP64) against
    the FP64 adjoint of the same event: E_T and eps2 within 3e-5 (measured
    9e-6 and 3e-6), the gradients with respect to the tau = 0 fields, g^2 mu^2
    and rho within 2e-4 in norm (measured 2e-6 to 6e-5)."""
    out = {}
    for prec in (ipg.FP64, ipg.FP32):
        with _event(prec) as ev:
            et, e2 = ev.forward(k)
            g = ev.backward(1.0, 1.0, inputs=True, rho=True)
            out[prec] = (et, e2, {key: np.array(v) for key, v in g.items()})
    (et64, e264, g64), (et32, e232, g32) = out[ipg.FP64], out[ipg.FP32]
    rels = {"E_T": abs(et32 / et64 - 1), "eps2": abs(e232 / e264 - 1)}
    for key in list(FIELDS) + ["g2mu", "rho"]:
        a, b = g32[key], g64[key]
        rels[str(key)] = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    print("FP32ADJ", k, rels)
    assert rels["E_T"] < 3e-5 and rels["eps2"] < 3e-5
    for key, v in rels.items():
        assert v < 2e-4, (key, v)


def test_gradient_at_AuAu256_400_steps_32_directions():
    """The adjoint configuration: Au+Au 256^2 (L = 30 fm, b = 2 fm, Ny = 50,
    seeded Woods-Saxon nuclei), 400 leapfrog steps at dtau = 0.1 a, a
    checkpoint every 20 steps with time reversal in between. The gradient of
    E_T + eps2 with respect to g^2 mu^2 (16 directions of relative
    perturbations) and rho (16 directions in the noise) against central
    finite differences with h = 1e-6 (relative), Newton polished to 1e-14.

    A central difference of the loss carries the loss's own evaluation
    noise divided by 2h: over 400 steps the evolution amplifies the rounding
    of each evaluation, and with h = 1e-6 that noise is not negligible on
    every direction (measured: median gap 2e-5, the worst 7e-4). Each
    direction is therefore differenced at h and at h/2: their spread
    measures the difference's uncertainty. The test asserts that the adjoint
    lies within three times that spread plus 1e-4 relative of the h = 1e-6
    difference on every direction, and that the median gap at h = 1e-6 is
    below 1e-4.
    """
    from ipglasma_b200.synthetic import make_event

    N, L, Ny = 256, 30.0, 50
    a = L / N
    A, B, _, _ = make_event(N, L, "Au", 2.0, seed=8000)
    rng = np.random.default_rng(8100)
    xi = rng.standard_normal((2, Ny, N * N, 8))
    ev = ipg.Event(ipg.Config(size=N, L=L, Ny=Ny, maxtime=400 * 0.1 * a, dtau=0.1,
                              precision=ipg.FP64, seed=8100, newton_tolerance=1e-14))
    assert ev.itmax == 400

    def loss(gA, gB, x):
        ev.set_g2mu(gA, gB)
        ev.set_noise(x[0], x[1])
        rep = ev.init_fields()
        assert rep.newton_failed == 0
        et, e2 = ev.forward(20)
        return et + e2

    loss(A, B, xi)
    g = ev.backward(1.0, 1.0, inputs=True, rho=True)
    amp = np.stack([2.0 * np.sqrt(A / Ny), 2.0 * np.sqrt(B / Ny)])
    h = 1e-6
    rows = []
    for k in range(32):
        if k < 16:
            dA = A * rng.uniform(-1, 1, A.shape)
            dB = B * rng.uniform(-1, 1, B.shape)
            directional = float(np.sum(g["g2mu"][0] * dA) + np.sum(g["g2mu"][1] * dB))

            def D(s):
                return (loss(A + s * dA, B + s * dB, xi) - loss(A - s * dA, B - s * dB, xi)) / (2 * s)
        else:
            dxi = rng.standard_normal(xi.shape)
            directional = float(np.sum(g["rho"] * amp[:, None, :, None] * dxi))

            def D(s):
                return (loss(A, B, xi + s * dxi) - loss(A, B, xi - s * dxi)) / (2 * s)
        d1, d2 = D(h), D(h / 2)
        gap, spread = abs(directional - d1), abs(d1 - d2)
        rows.append((gap / (3 * spread + 1e-4 * abs(d1)), gap / abs(d1), spread / abs(d1), k,
                     directional, d1, d2))
    ev.close()
    print("FD32 h=1e-6 gaps: " + " ".join(f"{r[1]:.1e}" for r in rows))
    print("FD32 h vs h/2 spreads: " + " ".join(f"{r[2]:.1e}" for r in rows))
    assert float(np.median([r[1] for r in rows])) < 1e-4
    worst = max(rows)
    assert worst[0] < 1.0, worst
