"""Synthetic event inputs: Woods-Saxon nuclei -> thickness -> g^2 mu^2 maps.

The hot path takes the g^2 mu^2 maps of both nuclei as input. For benchmark
and test events they are built as follows (one convention for both the GPU
path and the CPU oracle, which receive the same maps):

1. Nucleons: radii drawn from the Woods-Saxon density by the rejection rule of
   Init::sample_r_from_woods_saxon (Init.cpp:2818-2826), sorted, then placed
   at random directions with a minimum-distance rejection of at most 100
   tries against the already placed nucleons of smaller radius
   (Init::generate_nucleus_configuration_with_woods_saxon, Init.cpp:2749-2816),
   recentred (Init.cpp:3105-3123) and given a uniform random 3D orientation.
2. Geometry: nucleus A shifted by -b/2, B by +b/2 along x.
3. Thickness: T(x) = sum_i exp(-|x - x_i|^2 / (2 B_p)) / (2 pi B_p), B_p in
   GeV^-2 converted with hbar c (Init.cpp:1052-1062).
4. Saturation scale Q_s(x) = Qs_max sqrt(T(x) / max T) per nucleus and
   g^2 mu^2 a^2 = Q_s^2 / QsmuRatio^2 a^2 / (hbar c)^2 / g^2 in lattice units
   (the conversion of Init.cpp:1403-1408).

Random numbers come from numpy's PCG64 seeded per event; this generator is
input preparation, not part of the timed hot path.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

HBARC = 0.1973269718

NUCLEI = {
    # name: (A, R_WS fm, a_WS fm)
    "Au": (197, 6.38, 0.535),
    "Pb": (208, 6.62, 0.546),
    "O": (16, 2.61, 0.513),
}


@dataclass
class NucleusSpec:
    A: int
    R: float
    a_ws: float
    d_min: float = 0.4


def nucleus_spec(name: str, d_min: float = 0.4) -> NucleusSpec:
    A, R, a = NUCLEI[name]
    return NucleusSpec(A, R, a, d_min)


def sample_nucleus(rng: np.random.Generator, spec: NucleusSpec) -> np.ndarray:
    """(A, 3) nucleon positions in fm."""
    rmax = spec.R + 10.0 * spec.a_ws
    radii = np.empty(spec.A)
    for i in range(spec.A):
        while True:
            r = rmax * rng.random() ** (1.0 / 3.0)
            if rng.random() <= 1.0 / (1.0 + np.exp((r - spec.R) / spec.a_ws)):
                radii[i] = r
                break
    radii.sort(kind="stable")
    pos = np.zeros((spec.A, 3))
    dmin2 = spec.d_min ** 2
    for i in range(spec.A):
        r = radii[i]
        for _ in range(100):
            phi = 2.0 * np.pi * rng.random()
            theta = np.arccos(1.0 - 2.0 * rng.random())
            p = r * np.array([np.sin(theta) * np.cos(phi),
                              np.sin(theta) * np.sin(phi), np.cos(theta)])
            j = i - 1
            ok = True
            while j >= 0 and (r - radii[j]) ** 2 <= dmin2:
                if np.sum((p - pos[j]) ** 2) < dmin2:
                    ok = False
                    break
                j -= 1
            if ok:
                break
        pos[i] = p
    pos -= pos.mean(axis=0)
    # uniform random orientation (QR of a Gaussian matrix)
    q, rr = np.linalg.qr(rng.standard_normal((3, 3)))
    q *= np.sign(np.diag(rr))
    return pos @ q.T


def thickness(xy: np.ndarray, N: int, L: float, Bp: float = 4.0) -> np.ndarray:
    """T(x) on the N x N grid (pos = ix*N + iy), fm^-2."""
    a = L / N
    x = -L / 2.0 + a * np.arange(N)
    B = Bp * HBARC ** 2  # fm^2
    T = np.zeros((N, N))
    gx = np.exp(-(x[None, :] - xy[:, 0:1]) ** 2 / (2 * B))  # (A, N)
    gy = np.exp(-(x[None, :] - xy[:, 1:2]) ** 2 / (2 * B))
    T = gx.T @ gy / (2 * np.pi * B)  # separable Gaussian sum
    return T


def g2mu2_map(T: np.ndarray, a: float, g: float, qs_max: float = 1.5,
              qsmu_ratio: float = 0.8) -> np.ndarray:
    tmax = T.max()
    qs2 = (qs_max ** 2) * (T / tmax if tmax > 0 else T)
    return qs2 / qsmu_ratio ** 2 * a * a / HBARC ** 2 / (g * g)


def make_event(N: int, L: float, nucleus: str, b: float, seed: int,
               g: float = 2.0, qs_max: float = 1.5, Bp: float = 4.0):
    """g2mu2A, g2mu2B (flat, pos = ix*N + iy, lattice units) and the nuclei."""
    rng = np.random.Generator(np.random.PCG64(seed))
    spec = nucleus_spec(nucleus)
    nA = sample_nucleus(rng, spec)
    nB = sample_nucleus(rng, spec)
    nA[:, 0] -= b / 2.0
    nB[:, 0] += b / 2.0
    a = L / N
    TA = thickness(nA, N, L, Bp)
    TB = thickness(nB, N, L, Bp)
    return (g2mu2_map(TA, a, g, qs_max).ravel(), g2mu2_map(TB, a, g, qs_max).ravel(),
            nA, nB)


def gaussian_blobs(N: int, L: float, g: float = 2.0, qs_max: float = 1.5):
    """Two-blob test maps for small lattices (cheap, deterministic)."""
    a = L / N
    x = -L / 2.0 + a * np.arange(N)
    X, Y = np.meshgrid(x, x, indexing="ij")
    s = L / 8.0

    def blob(x0, y0, r):
        return np.exp(-((X - x0) ** 2 + (Y - y0) ** 2) / (2 * r * r))

    TA = blob(-0.06 * L, 0.03 * L, s) + 0.5 * blob(0.1 * L, -0.07 * L, 0.55 * s)
    TB = blob(0.07 * L, -0.01 * L, 0.9 * s) + 0.4 * blob(-0.11 * L, 0.09 * L, 0.6 * s)
    return g2mu2_map(TA, a, g, qs_max).ravel(), g2mu2_map(TB, a, g, qs_max).ravel()
