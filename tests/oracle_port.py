"""ctypes binding of the C restatement (oracle/ipg_oracle.c).

Test infrastructure: used only by tests, the smoke check and the CPU-baseline
leg of bench.py, always as the checker.
"""
from __future__ import annotations

import ctypes as ct
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
LIB = ROOT / "oracle" / "_ref" / "libipg_oracle.so"

_lib = None
_D = ct.POINTER(ct.c_double)


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise FileNotFoundError(f"{LIB} missing: run `make -C oracle port`")
        h = ct.CDLL(str(LIB))
        h.ipgo_gauss_stream.argtypes = [ct.c_uint64, ct.c_long, _D]
        h.ipgo_expm.argtypes = [_D, _D]
        h.ipgo_wilson_lines.argtypes = [ct.c_int, ct.c_int, ct.c_double, ct.c_double,
                                        ct.c_double, ct.c_double, _D, _D, _D]
        h.ipgo_tau0.argtypes = [ct.c_int, ct.c_double, _D, _D, _D, _D, _D,
                                ct.POINTER(ct.c_int)]
        h.ipgo_tau0.restype = ct.c_int
        h.ipgo_evolve_phi.argtypes = [ct.c_int, ct.c_double, ct.c_double, _D, _D]
        h.ipgo_evolve_u.argtypes = [ct.c_int, ct.c_double, ct.c_double, ct.c_double, _D, _D, _D, _D]
        h.ipgo_evolve_pi.argtypes = [ct.c_int, ct.c_double, ct.c_double, _D, _D, _D, _D]
        h.ipgo_evolve_e.argtypes = [ct.c_int, ct.c_double, ct.c_double, ct.c_double,
                                    _D, _D, _D, _D, _D]
        h.ipgo_tmunu.argtypes = [ct.c_int, ct.c_double, ct.c_double, ct.c_double, ct.c_int,
                                 _D, _D, _D, _D, _D, _D, _D]
        h.ipgo_landau.argtypes = [ct.c_int, ct.c_double, ct.c_double, ct.c_int, _D, _D, _D, _D]
        h.ipgo_landau.restype = ct.c_int
        h.ipgo_gauss_law.argtypes = [ct.c_int, _D, _D, _D, _D, _D, _D]
        h.ipgo_gauss_law.restype = ct.c_double
        h.ipgo_eccentricity.argtypes = [ct.c_int, ct.c_double, _D, _D, _D, _D]
        h.ipgo_run_event.argtypes = [ct.c_int, ct.c_int, ct.c_double, ct.c_double, ct.c_double,
                                     ct.c_double, ct.c_double, ct.c_double, _D, _D, _D, _D,
                                     _D, _D, _D, _D, _D, _D, _D, _D, _D, _D]
        for fn in (h.ipgo_write_hydro, h.ipgo_write_tmunu):
            fn.restype = ct.c_int
        _lib = h
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(_D)


def _c(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def gauss_stream(seed: int, count: int) -> np.ndarray:
    out = np.empty(count)
    lib().ipgo_gauss_stream(seed, count, _p(out))
    return out


def noise(seed: int, N: int, Ny: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit normals of nucleus A and B in Init::setV's draw order."""
    cnt = Ny * N * N * 8
    z = gauss_stream(seed, 2 * cnt)
    return z[:cnt].copy(), z[cnt:].copy()


def expm(q) -> np.ndarray:
    out = np.empty(18)
    lib().ipgo_expm(_p(_c(q)), _p(out))
    return out.view(np.complex128).reshape(3, 3)


def mats(a: np.ndarray, n: int) -> np.ndarray:
    return a.view(np.complex128).reshape(n, 3, 3)


def wilson_lines(N, Ny, L, g, m, uvdamp, g2mu2, xi) -> np.ndarray:
    V = np.empty(N * N * 18)
    lib().ipgo_wilson_lines(N, Ny, L, g, m, uvdamp, _p(_c(g2mu2)), _p(_c(xi)), _p(V))
    return mats(V, N * N)


def tau0(N, g, VA, VB):
    n = N * N
    VA = _c(np.asarray(VA).view(np.float64).ravel())
    VB = _c(np.asarray(VB).view(np.float64).ravel())
    Ux, Uy, pi = np.empty(18 * n), np.empty(18 * n), np.empty(18 * n)
    it = np.empty(2 * n, dtype=np.int32)
    r = lib().ipgo_tau0(N, g, _p(VA), _p(VB), _p(Ux), _p(Uy), _p(pi),
                        it.ctypes.data_as(ct.POINTER(ct.c_int)))
    return mats(Ux, n), mats(Uy, n), mats(pi, n), it, r


def run_event(N, Ny, L, g, m, uvdamp, maxtime, g2muA, g2muB, xiA, xiB, dtau=-1.0):
    n = N * N
    out = {k: np.empty(18 * n) for k in ("VA", "VB", "Ux", "Uy", "pi")}
    eps, u4, pi10, T10 = np.empty(n), np.empty(4 * n), np.empty(10 * n), np.empty(10 * n)
    sc = np.empty(8)
    lib().ipgo_run_event(N, Ny, L, g, m, uvdamp, maxtime, dtau, _p(_c(g2muA)), _p(_c(g2muB)),
                         _p(_c(xiA)), _p(_c(xiB)), _p(out["VA"]), _p(out["VB"]), _p(out["Ux"]),
                         _p(out["Uy"]), _p(out["pi"]), _p(eps), _p(u4), _p(pi10), _p(T10), _p(sc))
    res = {k: mats(v, n) for k, v in out.items()}
    res.update(eps=eps, u4=u4.reshape(4, n), pi10=pi10.reshape(10, n), T10=T10.reshape(10, n),
               gauss=sc[0], ecc2=sc[1], itmax=int(sc[2]), dtau=sc[3], restarts=int(sc[4]))
    return res


def write_hydro(path, N, L, size_out, L_out, eta_size, deta, it, dtau, eps, u4, pi10,
                gfactor) -> float:
    D = ct.c_double
    etot = D()
    st = lib().ipgo_write_hydro(str(path).encode(), N, D(L), size_out, D(L_out), eta_size,
                                D(deta), it, D(dtau), _p(_c(eps)), _p(_c(u4)), _p(_c(pi10)),
                                D(gfactor), ct.byref(etot))
    assert st == 0
    return etot.value


def write_tmunu(path, N, L, size_out, L_out, eta_size, deta, it, dtau, T10, gfactor) -> None:
    D = ct.c_double
    st = lib().ipgo_write_tmunu(str(path).encode(), N, D(L), size_out, D(L_out), eta_size,
                                D(deta), it, D(dtau), _p(_c(T10)), D(gfactor))
    assert st == 0
