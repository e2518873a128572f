"""Batched events (ipg_batch_*): events of different lattice sizes advanced by
one persistent launch per step, the step sequence replayed as a CUDA graph,
must give what each event gives on its own (ipg_run), in both forms, on the
first run and on graph replays."""
import numpy as np
import pytest

import ipglasma_b200 as ipg
from ipglasma_b200.synthetic import gaussian_blobs

pytestmark = pytest.mark.gpu

# same lattice spacing a = 0.078125 fm, so one time grid; maxtime 0.21 fm
# gives an odd step count (27), which flips the U/phi buffer parity per run
SIZES = [(64, 5.0), (128, 10.0), (64, 5.0)]
MAXTIME = 0.21


def make(prec, N, L, seed):
    ev = ipg.Event(ipg.Config(size=N, L=L, Ny=4, maxtime=MAXTIME, precision=prec, seed=seed))
    A, B = gaussian_blobs(N, L)
    ev.set_g2mu(A, B)
    ev.use_device_noise()
    ev.init_fields()
    return ev


def single(prec):
    out = []
    for k, (N, L) in enumerate(SIZES):
        ev = make(prec, N, L, 100 + k)
        r = ev.run()
        eps = ev.observables()[0]
        out.append((r, eps))
        ev.close()
    return out


@pytest.mark.parametrize("prec", [ipg.FP64, ipg.FP32])
def test_batch_matches_single_events_and_replays(prec):
    ref = single(prec)
    events = [make(prec, N, L, 100 + k) for k, (N, L) in enumerate(SIZES)]
    assert events[0].itmax % 2 == 1
    with ipg.Batch(events) as b:
        for rep in range(2):
            res = b.run()
            for k, ev in enumerate(events):
                r0, e0 = ref[k]
                eps = ev.observables()[0]
                # the batched kernel runs the same per-site code as the
                # single-event kernel on the same inputs
                assert np.array_equal(eps, e0), (rep, k, np.abs(eps - e0).max())
                assert res[k].E_T == r0.E_T
                assert res[k].eccentricity[1] == r0.eccentricity[1]
                assert res[k].gauss_violation == r0.gauss_violation
            ms_evo, ms_tot, launches = b.stats()
            assert ms_evo > 0 and ms_tot >= ms_evo
            assert launches == (rep + 1) * events[0].itmax
            # fresh initial fields for the replay (same seeds, same result),
            # all events' initial conditions enqueued side by side
            for k, ev in enumerate(events):
                ev.reseed(100 + k)
            reps = b.init_fields()
            assert all(r.newton_failed == 0 for r in reps)
    for ev in events:
        ev.close()


def test_tune_picks_a_shape_and_caches_it():
    events = [make(ipg.FP32, N, L, 200 + k) for k, (N, L) in enumerate(SIZES)]
    with ipg.Batch(events) as b:
        rep = b.tune()
        assert rep.candidates >= 3 and rep.from_cache == 0
        assert rep.ms_per_step > 0
        assert rep.threads_per_block == 32 * rep.tile_rows
        assert rep.grid % rep.blocks_per_sm == 0
        res = b.run()
    for r in res:
        assert np.isfinite(r.E_T) and r.E_T > 0
    with ipg.Batch(events) as b2:
        rep2 = b2.tune()
        assert rep2.from_cache == 1 and rep2.variant == rep.variant
        assert rep2.blocks_per_sm == rep.blocks_per_sm
    for ev in events:
        ev.close()


def test_tune_restores_state():
    # a size mix of its own, so the tuner really times (no cache hit)
    sizes = [(64, 5.0), (64, 5.0)]
    a = [make(ipg.FP32, N, L, 300 + k) for k, (N, L) in enumerate(sizes)]
    b = [make(ipg.FP32, N, L, 300 + k) for k, (N, L) in enumerate(sizes)]
    with ipg.Batch(a) as ba:
        assert ba.tune().from_cache == 0
        ra = ba.run()
    with ipg.Batch(b) as bb:
        rb = bb.run()
    for x, y in zip(ra, rb):
        assert x.E_T == y.E_T and x.eccentricity[1] == y.eccentricity[1]
    for ev in a + b:
        ev.close()


def test_batch_rejects_mixed_time_grids():
    e1 = make(ipg.FP64, 64, 5.0, 1)
    e2 = ipg.Event(ipg.Config(size=64, L=6.0, Ny=4, maxtime=MAXTIME, precision=ipg.FP64))
    with pytest.raises(ipg.IPGError):
        ipg.Batch([e1, e2])
    e1.close()
    e2.close()


@pytest.mark.parametrize("prec", [ipg.FP64, ipg.FP32])
def test_every_batch_variant_gives_the_same_bits(prec):
    """Plain-load variants (tiles of 2, 4, 8 rows) and the TMA tile variant
    (the single-event tile kernel over every event's tiles, tensor maps per
    event and buffer parity) run the same per-site code: identical results,
    over two runs (both U/phi buffer arrangements)."""
    ref = single(prec)
    n_var = 4 if prec == ipg.FP32 else 3
    for v in range(n_var):
        events = [make(prec, N, L, 100 + k) for k, (N, L) in enumerate(SIZES)]
        with ipg.Batch(events) as b:
            b.set_shape(v, 1)
            for rep in range(2):
                res = b.run()
                for k, ev in enumerate(events):
                    r0, e0 = ref[k]
                    assert np.array_equal(ev.observables()[0], e0), (v, rep, k)
                    assert res[k].E_T == r0.E_T
                for k, ev in enumerate(events):
                    ev.reseed(100 + k)
                b.init_fields()
        for ev in events:
            ev.close()
