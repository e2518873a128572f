"""ipg_get_observables_async: copies started after one event and left
running while the next event is computed on the same context hold exactly
the first event's observables (the next observables stage waits for them),
and the second event's copies match a synchronous read."""
import numpy as np
import pytest

import ipglasma_b200 as ipg
from ipglasma_b200.synthetic import make_event

pytestmark = pytest.mark.gpu


def run(ev, A, B, seed):
    ev.reseed(seed)
    ev.set_g2mu(A, B)
    ev.use_device_noise()
    ev.init_fields(allow_nonconverged=True)
    ev.run()


def buffers(n):
    return (np.empty(n), np.empty((4, n)), np.empty((10, n)), np.empty((10, n)))


@pytest.mark.parametrize("prec", [ipg.FP32, ipg.FP64], ids=["fp32", "fp64"])
def test_async_copies_overlap_the_next_event(prec):
    N, L = 128, 20.0
    A, B, _, _ = make_event(N, L, "Pb", 6.0, 31)
    cfg = ipg.Config(size=N, L=L, Ny=10, maxtime=0.3, precision=prec, seed=1)
    ev = ipg.Event(cfg)
    ref = []
    for seed in (101, 202):
        run(ev, A, B, seed)
        ref.append(ev.observables())
    first, second = buffers(ev.n), buffers(ev.n)
    run(ev, A, B, 101)
    ev.observables_async(*first)
    run(ev, A, B, 202)
    ev.observables_async(*second)
    ev.wait_observables()
    for got, want in ((first, ref[0]), (second, ref[1])):
        for g, w in zip(got, want):
            assert np.array_equal(g, w)
    assert not np.array_equal(first[0], second[0])
    ev.close()


def test_forward_waits_for_pending_observable_copies():
    """ipg_forward rewrites T^{mu nu} on the device: a copy of the previous
    event's observables still running must finish first, so the host arrays
    hold that event's values and not the adjoint forward's."""
    N, L = 128, 20.0
    A, B, _, _ = make_event(N, L, "Pb", 6.0, 31)
    cfg = ipg.Config(size=N, L=L, Ny=10, maxtime=0.3, seed=1, newton_tolerance=1e-12)
    with ipg.Event(cfg) as ev:
        run(ev, A, B, 303)
        want = ev.observables()
        got = buffers(ev.n)
        run(ev, A, B, 303)
        ev.observables_async(*got)
        ev.reseed(404)
        ev.use_device_noise()
        ev.init_fields(allow_nonconverged=True)
        ev.forward(1)
        ev.wait_observables()
        for g, w in zip(got, want):
            assert np.array_equal(g, w)
