"""The host part of Evolution::multiplicity (ipg_multiplicity_finish) against
a numpy restatement of Evolution.cpp:2874-2960 (bin averages, the binned
integrals dN/dy 2 and dE/dy 2, the 3 and 6 GeV cuts) and 3098-3108 (the
pseudorapidity Jacobian of the k sums). No GPU: the function is host code in
the library."""
import math

import numpy as np
import pytest

import ipglasma_b200 as ipg

HBARC = 0.1973269718


def restated(dN, dE, n_sum, E_sum, count, a, pseudo, y=0.0, m=0.35, roots=200.0):
    bins, dkt = 100, 2.83 / 100
    out = dict(dNdy_binned=0.0, dEdy_binned=0.0, dNdy_cut3=0.0, dEdy_cut3=0.0,
               dNdy_cut6=0.0, dEdy_cut6=0.0)
    for ik in range(bins):
        if count[ik] <= 0:
            continue
        nk, Ek = n_sum[ik] / count[ik], E_sum[ik] / count[ik]
        w = (ik + 0.5) * dkt * dkt * 2.0 * math.pi
        if pseudo:
            pt = (ik + 0.5) * dkt / a * HBARC
            w = w * math.cosh(y) / math.sqrt(math.cosh(y) ** 2 + m * m / (pt * pt))
        out["dNdy_binned"] += nk * w
        out["dEdy_binned"] += Ek * w
        if ik * dkt / a * HBARC > 3.0:
            out["dNdy_cut3"] += nk * w
            out["dEdy_cut3"] += Ek * w
        if ik * dkt / a * HBARC > 6.0:
            out["dNdy_cut6"] += nk * w
            out["dEdy_cut6"] += Ek * w
    if pseudo:
        P = 0.13 + 0.32 * (roots / 1000.0) ** 0.115
        J = math.cosh(y) / math.sqrt(math.cosh(y) ** 2 + m * m / (P * P))
        dN, dE = dN * J, dE * J
    out.update(dNdy=dN, dEdy=dE, mean_pt=dE / dN)
    return out


@pytest.mark.parametrize("pseudo", [False, True])
def test_finish_matches_restatement(pseudo):
    rng = np.random.default_rng(3 + pseudo)
    n_sum = rng.uniform(0, 50, 100)
    E_sum = rng.uniform(0, 80, 100)
    count = rng.integers(0, 40, 100)
    count[::7] = 0
    a = 30.0 / 256
    kw = dict(use_pseudorapidity=pseudo, rapidity=0.4, jacobian_m=0.3, roots=5020.0)
    got = ipg.multiplicity_finish(812.5, 701.25, n_sum, E_sum, count, a, **kw)
    want = restated(812.5, 701.25, n_sum, E_sum, count, a, pseudo, 0.4, 0.3, 5020.0)
    for key, v in want.items():
        assert abs(got[key] - v) <= 1e-13 * abs(v), (key, got[key], v)
    np.testing.assert_array_equal(got["count_kt"], count)
    np.testing.assert_allclose(got["n_kt"], np.where(count > 0, n_sum / np.maximum(count, 1), 0),
                               rtol=1e-15)


def test_finish_rejects_bad_spacing():
    with pytest.raises(ipg.IPGError):
        ipg.multiplicity_finish(1, 1, np.zeros(100), np.zeros(100), np.zeros(100, int), 0.0)
