"""B200 implementation of IP-Glasma's per-event hot path.

Python host mirror of the C ABI in ``include/ipglasma_b200.h``. The reference
drives an event with two calls (main.cpp:347-359)::

    init.init(&lat, &group, param, random, &glauber, READFROMFILE)
    evolution.run(&lat, &group, param)

Here the same event is::

    ev = Event(Config(size=256, L=30.0, Ny=50, g=2.0, m=0.2, maxtime=0.4))
    ev.set_g2mu(g2mu2A, g2mu2B)          # Cell::setg2mu2A/B
    ev.use_device_noise()                # or ev.set_noise(xiA, xiB)
    report = ev.init_fields()            # Init::setV + tau=0 block
    result = ev.run()                    # Evolution::run
    eps, u, pi, T = ev.observables()     # Cell getters

All compute runs in ``libipglasma_b200.so`` (hand-written sm_100a kernels);
this module only marshals host arrays. If the library is missing the import
of :func:`lib` raises; there is no CPU path.
"""
from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

__all__ = ["Config", "Event", "Batch", "IPGError", "lib", "FP64", "FP32", "read_qs_table",
           "UX", "UY", "E1", "E2", "PHI", "PI", "VA", "VB", "HBARC", "multiplicity_finish",
           "KT_BINS"]

HBARC = 0.1973269718  # GeV fm, Phys_consts.h
FP64, FP32 = 0, 1
UX, UY, E1, E2, PHI, PI, VA, VB = range(8)

_STATUS = {
    0: "IPG_OK", 1: "IPG_ERR_BAD_CONFIG", 2: "IPG_ERR_CUDA",
    3: "IPG_ERR_NEWTON_NONCONVERGED", 4: "IPG_ERR_NAN", 5: "IPG_ERR_STATE",
    6: "IPG_ERR_NOMEM", 7: "IPG_ERR_TIMEOUT", 8: "IPG_NO_COLLISION",
}

LIB_PATH = Path(__file__).resolve().parent / "libipglasma_b200.so"


class IPGError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{_STATUS.get(status, status)}: {message}")
        self.status = status


class _Config(ct.Structure):
    _fields_ = [
        ("size", ct.c_int), ("Nc", ct.c_int), ("Ny", ct.c_int),
        ("L", ct.c_double), ("g", ct.c_double), ("m", ct.c_double),
        ("UVdamp", ct.c_double), ("maxtime", ct.c_double), ("dtau", ct.c_double),
        ("precision", ct.c_int), ("newton_max_iterations", ct.c_int),
        ("newton_max_restarts", ct.c_int), ("seed", ct.c_uint64),
        ("device", ct.c_int), ("newton_tolerance", ct.c_double),
        ("newton_mode", ct.c_int),
    ]


class _InitReport(ct.Structure):
    _fields_ = [
        ("newton_links", ct.c_int), ("newton_restarted", ct.c_int),
        ("newton_failed", ct.c_int), ("newton_max_iterations", ct.c_int),
        ("newton_mean_iterations", ct.c_double), ("ms_wilson", ct.c_double),
        ("ms_newton", ct.c_double), ("ms_fields", ct.c_double),
    ]


class _IpsatParams(ct.Structure):
    _fields_ = [
        ("BG", ct.c_double), ("QsmuRatio", ct.c_double), ("QsmuRatioB", ct.c_double),
        ("proton_anisotropy", ct.c_double), ("rapidity", ct.c_double), ("roots", ct.c_double),
        ("x_factor", ct.c_double), ("rmax", ct.c_double), ("sigmaNN", ct.c_double),
        ("use_fluctuating_x", ct.c_int), ("average_over_nuclei", ct.c_int),
    ]


class _IpsatReport(ct.Structure):
    _fields_ = [
        ("Npart", ct.c_int), ("Ncoll", ct.c_int), ("Tpp", ct.c_double),
        ("average_Qs", ct.c_double), ("average_Qs_avg", ct.c_double),
        ("average_Qs_min", ct.c_double), ("Qs2min_ST", ct.c_double),
        ("overlap_cells", ct.c_int), ("flags", ct.c_int),
    ]


class _TuneReport(ct.Structure):
    _fields_ = [
        ("variant", ct.c_int), ("tile_rows", ct.c_int), ("threads_per_block", ct.c_int),
        ("blocks_per_sm", ct.c_int), ("grid", ct.c_int), ("ms_per_step", ct.c_double),
        ("candidates", ct.c_int), ("from_cache", ct.c_int),
    ]


class _Result(ct.Structure):
    _fields_ = [
        ("itmax", ct.c_int), ("dtau", ct.c_double), ("tau_final", ct.c_double),
        ("gauss_violation", ct.c_double), ("unitarity_max", ct.c_double),
        ("sum_Ttautau", ct.c_double), ("sum_eps", ct.c_double),
        ("E_T", ct.c_double), ("eccentricity", ct.c_double * 6),
        ("psi", ct.c_double * 6), ("cells_without_u", ct.c_int),
        ("ms_evolution", ct.c_double), ("ms_observables", ct.c_double),
    ]


class _EccReport(ct.Structure):
    _fields_ = [(f, ct.c_double) for f in ("tau", "r_rms", "max_x", "max_y", "area", "Rbar",
                                          "avg_eps", "avg_qs2a_qs2b")]


class _GaugeReport(ct.Structure):
    _fields_ = [
        ("iterations", ct.c_int), ("residual_checks", ct.c_int), ("nan_sites", ct.c_int),
        ("residual", ct.c_double), ("residual_every10", ct.c_double * 401),
        ("ms", ct.c_double),
    ]


class _MultParams(ct.Structure):
    _fields_ = [
        ("max_gauge_iterations", ct.c_int), ("use_pseudorapidity", ct.c_int),
        ("rapidity", ct.c_double), ("jacobian_m", ct.c_double), ("roots", ct.c_double),
    ]


KT_BINS = 100


class _MultResult(ct.Structure):
    _fields_ = [
        ("it", ct.c_int), ("gauge", _GaugeReport),
        ("dNdy", ct.c_double), ("dEdy", ct.c_double),
        ("dNdy_binned", ct.c_double), ("dEdy_binned", ct.c_double),
        ("dNdy_cut3", ct.c_double), ("dEdy_cut3", ct.c_double),
        ("dNdy_cut6", ct.c_double), ("dEdy_cut6", ct.c_double),
        ("mean_pt", ct.c_double),
        ("n_kt", ct.c_double * KT_BINS), ("E_kt", ct.c_double * KT_BINS),
        ("count_kt", ct.c_int * KT_BINS), ("ms_spectrum", ct.c_double),
    ]


def _gauge_dict(g: _GaugeReport) -> dict:
    hist = np.array(g.residual_every10[:])
    return {"iterations": g.iterations, "residual_checks": g.residual_checks,
            "nan_sites": g.nan_sites, "residual": g.residual,
            "residual_every10": hist[~np.isnan(hist)], "ms": g.ms}


def _mult_dict(m: _MultResult) -> dict:
    out = {f: getattr(m, f) for f, _ in _MultResult._fields_
           if f not in ("gauge", "n_kt", "E_kt", "count_kt")}
    out["gauge"] = _gauge_dict(m.gauge)
    out["n_kt"] = np.array(m.n_kt[:])
    out["E_kt"] = np.array(m.E_kt[:])
    out["count_kt"] = np.array(m.count_kt[:])
    return out


def _mult_params(max_gauge_iterations=4000, use_pseudorapidity=False, rapidity=0.0,
                 jacobian_m=0.35, roots=200.0) -> _MultParams:
    return _MultParams(int(max_gauge_iterations), int(bool(use_pseudorapidity)),
                       float(rapidity), float(jacobian_m), float(roots))


def multiplicity_finish(dN, dE, n_sum, E_sum, count, a, **params) -> dict:
    """The host part of Evolution::multiplicity (ipg_multiplicity_finish):
    k sums and per-bin sums -> dN/dy, dE/dy, the binned integrals and cuts."""
    m = _MultResult()
    n_sum = _f64(n_sum, KT_BINS)
    E_sum = _f64(E_sum, KT_BINS)
    cnt = np.ascontiguousarray(count, dtype=np.int32)
    prm = _mult_params(**params)
    rc = lib().ipg_multiplicity_finish(float(dN), float(dE), _ptr(n_sum), _ptr(E_sum), _ptr(cnt),
                                       float(a), ct.byref(prm), ct.byref(m))
    if rc != 0:
        raise IPGError(rc, "ipg_multiplicity_finish rejected its arguments")
    return _mult_dict(m)


_lib = None

_SIGNATURES = {
    "ipg_last_error": (ct.c_char_p, [ct.c_void_p]),
    "ipg_create": (ct.c_int, [ct.POINTER(_Config), ct.POINTER(ct.c_void_p)]),
    "ipg_destroy": (ct.c_int, [ct.c_void_p]),
    "ipg_reseed": (ct.c_int, [ct.c_void_p, ct.c_uint64]),
    "ipg_time_grid": (ct.c_int, [ct.c_void_p, ct.POINTER(ct.c_double), ct.POINTER(ct.c_int)]),
    "ipg_set_g2mu": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "ipg_set_g2mu_device": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "ipg_set_noise": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "ipg_set_nuclei": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_int,
                                  ct.c_double, ct.c_double, ct.c_double, ct.c_double]),
    "ipg_get_g2mu": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "ipg_set_nuclei_ipsat": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_int,
                                        ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                        ct.c_double, ct.POINTER(_IpsatParams), ct.c_void_p,
                                        ct.c_void_p, ct.c_int, ct.c_int, ct.c_double,
                                        ct.POINTER(_IpsatReport)]),
    "ipg_get_thickness": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "ipg_set_noise_device": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "ipg_use_device_noise": (ct.c_int, [ct.c_void_p]),
    "ipg_draw_device_noise": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int,
                                         ct.c_void_p]),
    "ipg_init_fields": (ct.c_int, [ct.c_void_p, ct.POINTER(_InitReport)]),
    "ipg_init_from_wilson_lines": (ct.c_int, [ct.c_void_p, ct.POINTER(_InitReport)]),
    "ipg_run": (ct.c_int, [ct.c_void_p, ct.POINTER(_Result)]),
    "ipg_evolve": (ct.c_int, [ct.c_void_p, ct.c_int]),
    "ipg_gauge_fix": (ct.c_int, [ct.c_void_p, ct.c_int, ct.POINTER(_GaugeReport)]),
    "ipg_eccentricity_report": (ct.c_int, [ct.c_void_p, ct.c_double, ct.c_double,
                                           ct.POINTER(_EccReport)]),
    "ipg_multiplicity": (ct.c_int, [ct.c_void_p, ct.POINTER(_MultParams),
                                    ct.POINTER(_MultResult)]),
    "ipg_run_multiplicity": (ct.c_int, [ct.c_void_p, ct.POINTER(_MultParams),
                                        ct.POINTER(_Result), ct.POINTER(_MultResult),
                                        ct.POINTER(_MultResult)]),
    "ipg_multiplicity_finish": (ct.c_int, [ct.c_double, ct.c_double, ct.c_void_p, ct.c_void_p,
                                           ct.c_void_p, ct.c_double, ct.POINTER(_MultParams),
                                           ct.POINTER(_MultResult)]),
    "ipg_get_observables": (ct.c_int, [ct.c_void_p] + [ct.c_void_p] * 4),
    "ipg_get_observables_async": (ct.c_int, [ct.c_void_p] + [ct.c_void_p] * 4),
    "ipg_wait_observables": (ct.c_int, [ct.c_void_p]),
    "ipg_get_field": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_void_p]),
    "ipg_write_outputs": (ct.c_int, [ct.c_void_p, ct.c_char_p, ct.c_char_p, ct.c_int,
                                     ct.c_double, ct.c_int, ct.c_double, ct.c_int, ct.c_double,
                                     ct.c_double, ct.POINTER(ct.c_double)]),
    "ipg_write_hydro": (ct.c_int, [ct.c_char_p, ct.c_int, ct.c_double, ct.c_int, ct.c_double,
                                   ct.c_int, ct.c_double, ct.c_int, ct.c_double, ct.c_void_p,
                                   ct.c_void_p, ct.c_void_p, ct.c_double,
                                   ct.POINTER(ct.c_double)]),
    "ipg_write_tmunu": (ct.c_int, [ct.c_char_p, ct.c_int, ct.c_double, ct.c_int, ct.c_double,
                                   ct.c_int, ct.c_double, ct.c_int, ct.c_double, ct.c_void_p,
                                   ct.c_double]),
    "ipg_set_field": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_void_p]),
    "ipg_mark_initialized": (ct.c_int, [ct.c_void_p]),
    "ipg_get_newton_iterations": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "ipg_last_leapfrog_ms": (ct.c_int, [ct.c_void_p, ct.POINTER(ct.c_double), ct.POINTER(ct.c_int)]),
    "ipg_kernel_launches": (ct.c_int, [ct.c_void_p, ct.POINTER(ct.c_longlong)]),
    "ipg_forward": (ct.c_int, [ct.c_void_p, ct.c_int, ct.POINTER(ct.c_double),
                               ct.POINTER(ct.c_double)]),
    "ipg_backward": (ct.c_int, [ct.c_void_p, ct.c_double, ct.c_double, ct.c_void_p, ct.c_void_p,
                                ct.c_void_p]),
    "ipg_adjoint_stats": (ct.c_int, [ct.c_void_p, ct.POINTER(ct.c_double),
                                     ct.POINTER(ct.c_double)]),
    "ipg_batch_last_error": (ct.c_char_p, [ct.c_void_p]),
    "ipg_batch_create": (ct.c_int, [ct.POINTER(ct.c_void_p), ct.c_int, ct.POINTER(ct.c_void_p)]),
    "ipg_batch_destroy": (ct.c_int, [ct.c_void_p]),
    "ipg_batch_tune": (ct.c_int, [ct.c_void_p, ct.c_void_p]),
    "ipg_batch_init": (ct.c_int, [ct.c_void_p, ct.c_void_p]),
    "ipg_batch_run": (ct.c_int, [ct.c_void_p, ct.c_void_p]),
    "ipg_batch_set_shape": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int]),
    "ipg_batch_stats": (ct.c_int, [ct.c_void_p, ct.POINTER(ct.c_double), ct.POINTER(ct.c_double),
                                   ct.POINTER(ct.c_longlong)]),
}


def lib() -> ct.CDLL:
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m ipglasma_b200.build`")
        handle = ct.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def _ptr(a: np.ndarray) -> ct.c_void_p:
    return ct.c_void_p(a.ctypes.data)


def _f64(a, n: int | None = None) -> np.ndarray:
    arr = np.ascontiguousarray(a, dtype=np.float64)
    if n is not None and arr.size != n:
        raise ValueError(f"expected {n} values, got {arr.size}")
    return arr


@dataclass
class Config:
    """Per-event configuration (the hot-path keys of the reference input)."""
    size: int = 64
    L: float = 8.0
    Ny: int = 50
    g: float = 2.0
    m: float = 0.2
    UVdamp: float = 0.0
    maxtime: float = 0.4
    dtau: float = 0.0
    precision: int = FP64
    newton_max_iterations: int = 2000
    newton_max_restarts: int = 200
    seed: int = 1
    device: int = 0
    Nc: int = 3
    newton_tolerance: float = 0.0
    newton_mode: int = 0  # 0 the reference's iteration, 1 Newton on the group

    def to_c(self) -> _Config:
        return _Config(self.size, self.Nc, self.Ny, self.L, self.g, self.m,
                       self.UVdamp, self.maxtime, self.dtau, self.precision,
                       self.newton_max_iterations, self.newton_max_restarts,
                       self.seed, self.device, self.newton_tolerance, self.newton_mode)


@dataclass
class InitReport:
    newton_links: int
    newton_restarted: int
    newton_failed: int
    newton_max_iterations: int
    newton_mean_iterations: float
    ms_wilson: float
    ms_newton: float
    ms_fields: float


@dataclass
class Result:
    itmax: int
    dtau: float
    tau_final: float
    gauss_violation: float
    unitarity_max: float
    sum_Ttautau: float
    sum_eps: float
    E_T: float
    eccentricity: list = field(default_factory=list)
    psi: list = field(default_factory=list)
    cells_without_u: int = 0
    ms_evolution: float = 0.0
    ms_observables: float = 0.0


def read_qs_table(path, ny: int = 44):
    """The reference's Q_s^2(T, y) table file (qs2Adj_vs_Tp_vs_Y_200.in,
    read by Init::readNuclearQs, Init.cpp:441-480): records "y T Qs^2", ny
    rapidities per T, T increasing. Returns (Tlist[nT], qs2[nT][ny])."""
    rec = np.loadtxt(path).reshape(-1, ny, 3)
    return rec[:, 0, 1].copy(), rec[:, :, 2].copy()


class Event:
    """One event on one GPU (an ``ipg_ctx``)."""

    def __init__(self, cfg: Config):
        self.cfg = cfg
        self._lib = lib()
        self._pending_obs = None
        h = ct.c_void_p()
        c = cfg.to_c()
        st = self._lib.ipg_create(ct.byref(c), ct.byref(h))
        self._h = h
        if st != 0:
            msg = self._lib.ipg_last_error(h).decode() if h.value else "ipg_create failed"
            if h.value:
                self._lib.ipg_destroy(h)
            self._h = ct.c_void_p()
            raise IPGError(st, msg)
        self.N = cfg.size
        self.n = cfg.size * cfg.size
        d, it = ct.c_double(), ct.c_int()
        self._check(self._lib.ipg_time_grid(self._h, ct.byref(d), ct.byref(it)))
        self.dtau, self.itmax = d.value, it.value

    # -- plumbing -----------------------------------------------------------
    def _check(self, st: int, allow: tuple = ()) -> int:
        if st != 0 and st not in allow:
            raise IPGError(st, self._lib.ipg_last_error(self._h).decode())
        return st

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            # ipg_destroy waits for the context's streams, the copy stream of
            # observables_async included, before the arrays are let go
            self._lib.ipg_destroy(self._h)
            self._h = ct.c_void_p()
        self._pending_obs = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- inputs ---------------------------------------------------------------
    def set_g2mu(self, g2mu2A, g2mu2B) -> None:
        a, b = _f64(g2mu2A, self.n), _f64(g2mu2B, self.n)
        self._check(self._lib.ipg_set_g2mu(self._h, _ptr(a), _ptr(b)))

    def set_g2mu_device(self, ptr_a: int, ptr_b: int) -> None:
        self._check(self._lib.ipg_set_g2mu_device(self._h, ct.c_void_p(ptr_a),
                                                  ct.c_void_p(ptr_b)))

    def set_nuclei(self, xyzA, xyzB, b: float, BG: float = 4.0, qs_max: float = 1.5,
                   qsmu_ratio: float = 0.8) -> None:
        """g2mu maps from nucleon positions ((A, 3) arrays in fm), on the device."""
        a = np.ascontiguousarray(xyzA, dtype=np.float64).reshape(-1, 3)
        bb = np.ascontiguousarray(xyzB, dtype=np.float64).reshape(-1, 3)
        self._check(self._lib.ipg_set_nuclei(self._h, _ptr(a), len(a), _ptr(bb), len(bb), b, BG,
                                             qs_max, qsmu_ratio))

    def set_nuclei_ipsat(self, xyzA, xyzB, b: float, table, *, BG: float = 4.0,
                         QsmuRatio: float = 0.8, QsmuRatioB: float | None = None,
                         proton_anisotropy: float = 0.0, rapidity: float = 0.0,
                         roots: float = 5020.0, x_factor: float = 0.5, rmax: float = 3.0,
                         sigmaNN: float = 70.0, use_fluctuating_x: bool = True,
                         average_over_nuclei: int = 1, phiA=None, phiB=None, normA=None,
                         normB=None, dy: float = 0.25) -> dict:
        """IP-Sat g2mu maps from nucleon positions ((A, 3) arrays in fm) and the
        Q_s^2(T, y) table, given as (Tlist[nT], qs2[nT][ny]) with y = k dy
        (the layout of the reference's qs2Adj_vs_Tp_vs_Y_200.in; see
        :func:`read_qs_table`). Returns the event report as a dict."""
        a = np.ascontiguousarray(xyzA, dtype=np.float64).reshape(-1, 3)
        bb = np.ascontiguousarray(xyzB, dtype=np.float64).reshape(-1, 3)
        Tlist = np.ascontiguousarray(table[0], dtype=np.float64)
        qs2 = np.ascontiguousarray(table[1], dtype=np.float64)
        if qs2.ndim != 2 or qs2.shape[0] != Tlist.size:
            raise ValueError("table: qs2 must be (len(Tlist), ny)")
        opt = [None if v is None else np.ascontiguousarray(v, dtype=np.float64)
               for v in (phiA, phiB, normA, normB)]
        p = _IpsatParams(BG, QsmuRatio, QsmuRatio if QsmuRatioB is None else QsmuRatioB,
                         proton_anisotropy, rapidity, roots, x_factor, rmax, sigmaNN,
                         int(use_fluctuating_x), average_over_nuclei)
        rep = _IpsatReport()
        self._check(self._lib.ipg_set_nuclei_ipsat(
            self._h, _ptr(a), len(a), _ptr(bb), len(bb),
            *[_ptr(v) if v is not None else None for v in opt], b, ct.byref(p), _ptr(Tlist),
            _ptr(qs2), Tlist.size, qs2.shape[1], dy, ct.byref(rep)))
        return {f: getattr(rep, f) for f, _ in _IpsatReport._fields_}

    def thickness(self):
        """T_A, T_B (2, N*N) in GeV^2 of the last set_nuclei_ipsat."""
        out = np.empty((2, self.n))
        self._check(self._lib.ipg_get_thickness(self._h, _ptr(out[0]), _ptr(out[1])))
        return out

    def g2mu(self):
        """The current g2mu maps (2, N*N), lattice units."""
        out = np.empty((2, self.n))
        self._check(self._lib.ipg_get_g2mu(self._h, _ptr(out[0]), _ptr(out[1])))
        return out

    def set_noise(self, xiA, xiB) -> None:
        cnt = self.cfg.Ny * self.n * 8
        a, b = _f64(xiA, cnt), _f64(xiB, cnt)
        self._check(self._lib.ipg_set_noise(self._h, _ptr(a), _ptr(b)))

    def set_noise_device(self, ptr_a: int, ptr_b: int) -> None:
        self._check(self._lib.ipg_set_noise_device(self._h, ct.c_void_p(ptr_a),
                                                   ct.c_void_p(ptr_b)))

    def reseed(self, seed: int) -> None:
        self.cfg.seed = seed
        self._check(self._lib.ipg_reseed(self._h, seed))

    def use_device_noise(self) -> None:
        self._check(self._lib.ipg_use_device_noise(self._h))

    def draw_device_noise(self, nucleus: int, sheet_first: int = 0, sheet_count=None):
        """The unit normals the device draw uses for one nucleus (0 = A,
        1 = B): (sheets, N*N, 8) float64, the layout of :meth:`set_noise`."""
        cnt = self.cfg.Ny - sheet_first if sheet_count is None else sheet_count
        out = np.empty((cnt, self.n, 8))
        self._check(self._lib.ipg_draw_device_noise(self._h, nucleus, sheet_first, cnt,
                                                    _ptr(out)))
        return out

    # -- stages ---------------------------------------------------------------
    def init_fields(self, allow_nonconverged: bool = False) -> InitReport:
        rep = _InitReport()
        allow = (3,) if allow_nonconverged else ()
        self._check(self._lib.ipg_init_fields(self._h, ct.byref(rep)), allow)
        return InitReport(*(getattr(rep, f) for f, _ in _InitReport._fields_))

    def init_from_wilson_lines(self, allow_nonconverged: bool = False) -> InitReport:
        """tau = 0 Newton links and fields from Wilson lines loaded with
        set_field(VA / VB) (the READFROMFILE path of Init::init)."""
        rep = _InitReport()
        allow = (3,) if allow_nonconverged else ()
        self._check(self._lib.ipg_init_from_wilson_lines(self._h, ct.byref(rep)), allow)
        return InitReport(*(getattr(rep, f) for f, _ in _InitReport._fields_))

    def run(self) -> Result:
        res = _Result()
        self._check(self._lib.ipg_run(self._h, ct.byref(res)))
        vals = {f: getattr(res, f) for f, _ in _Result._fields_}
        vals["eccentricity"] = list(res.eccentricity)
        vals["psi"] = list(res.psi)
        return Result(**vals)

    def evolve(self, steps: int) -> None:
        self._check(self._lib.ipg_evolve(self._h, steps))

    def eccentricity_report(self, QsmuRatio=0.8, QsmuRatioB=None) -> dict:
        """The other figures of the reference's eccentricities<id>.dat line
        for the last run (ipg_eccentricity_report)."""
        r = _EccReport()
        qb = QsmuRatio if QsmuRatioB is None else QsmuRatioB
        self._check(self._lib.ipg_eccentricity_report(self._h, float(QsmuRatio), float(qb),
                                                      ct.byref(r)))
        return {f: getattr(r, f) for f, _ in _EccReport._fields_}

    # -- gauge fixing and gluon multiplicity ----------------------------------
    def gauge_fix(self, max_iterations: int = 4000) -> dict:
        """Transverse Coulomb gauge (GaugeFix::FFTChi) of the current fields,
        in place on an FP64 context."""
        rep = _GaugeReport()
        self._check(self._lib.ipg_gauge_fix(self._h, int(max_iterations), ct.byref(rep)))
        return _gauge_dict(rep)

    def multiplicity(self, **params) -> dict:
        """Gauge fixing, then the gluon spectrum of the current fields
        (Evolution::multiplicity); params: max_gauge_iterations,
        use_pseudorapidity, rapidity, jacobian_m, roots."""
        m = _MultResult()
        prm = _mult_params(**params)
        self._check(self._lib.ipg_multiplicity(self._h, ct.byref(prm), ct.byref(m)))
        return _mult_dict(m)

    def run_multiplicity(self, **params):
        """run() with the spectrum at it = 1 and at it = itmax, as the
        reference's computeGluonMultiplicity schedule; returns
        (Result, spectrum at it = 1, spectrum at itmax); (None, spectrum at
        it = 1, None) when no collision happened (dN/dy = 0 at it = 1: the
        evolution stops there)."""
        res, m1, m2 = _Result(), _MultResult(), _MultResult()
        prm = _mult_params(**params)
        st = self._check(self._lib.ipg_run_multiplicity(self._h, ct.byref(prm), ct.byref(res),
                                                        ct.byref(m1), ct.byref(m2)), (8,))
        if st == 8:
            return None, _mult_dict(m1), None
        vals = {f: getattr(res, f) for f, _ in _Result._fields_}
        vals["eccentricity"] = list(res.eccentricity)
        vals["psi"] = list(res.psi)
        return Result(**vals), _mult_dict(m1), _mult_dict(m2)

    # -- outputs --------------------------------------------------------------
    def observables(self):
        n = self.n
        eps = np.empty(n)
        u4 = np.empty((4, n))
        pi10 = np.empty((10, n))
        T10 = np.empty((10, n))
        self._check(self._lib.ipg_get_observables(self._h, _ptr(eps), _ptr(u4),
                                                  _ptr(pi10), _ptr(T10)))
        return eps, u4, pi10, T10

    def observables_async(self, eps=None, u4=None, pi10=None, T10=None) -> None:
        """Start copying the observables into the given float64 arrays (shapes
        of :meth:`observables`; page-locked for overlap; None skips that
        copy) and return at once; they are complete after
        :meth:`wait_observables`. The event keeps the arrays alive until
        then, so the copy never writes into freed host memory."""
        bufs = (eps, u4, pi10, T10)
        for a, size in zip(bufs, (self.n, 4 * self.n, 10 * self.n, 10 * self.n)):
            if a is None:
                continue
            if a.dtype != np.float64 or a.size != size or not a.flags.c_contiguous:
                raise ValueError(f"observable buffer needs {size} contiguous float64")
        self._check(self._lib.ipg_get_observables_async(
            self._h, *(_ptr(a) if a is not None else None for a in bufs)))
        # copies queue up on the context's copy stream: every pending set of
        # arrays stays referenced until wait_observables
        if self._pending_obs is None:
            self._pending_obs = []
        self._pending_obs.append(bufs)

    def wait_observables(self) -> None:
        self._check(self._lib.ipg_wait_observables(self._h))
        self._pending_obs = None

    def write_outputs(self, hydro=None, tmunu=None, size_output=None, L_output=None,
                      eta_size=1, deta=0.0, gfactor=1.0):
        """The hydro and KoMPoST files of the last run (paths; either may be
        None) with the resampling and formatting on the GPU, byte-identical
        to the host writers (ipg_write_outputs). Defaults resample onto the
        lattice itself. Returns the hydro file's Etot (GeV), or None."""
        size_output = self.N if size_output is None else size_output
        L_output = self.cfg.L if L_output is None else L_output
        et = ct.c_double()
        self._check(self._lib.ipg_write_outputs(
            self._h, str(hydro).encode() if hydro else None,
            str(tmunu).encode() if tmunu else None, size_output, L_output, eta_size, deta,
            self.itmax, self.dtau, gfactor, ct.byref(et)))
        return et.value if hydro else None

    def get_field(self, which: int) -> np.ndarray:
        out = np.empty((self.n, 9), dtype=np.complex128)
        self._check(self._lib.ipg_get_field(self._h, which, _ptr(out)))
        return out.reshape(self.n, 3, 3)

    def set_field(self, which: int, mats) -> None:
        arr = np.ascontiguousarray(np.asarray(mats, dtype=np.complex128).reshape(self.n, 9))
        self._check(self._lib.ipg_set_field(self._h, which, _ptr(arr)))

    def mark_initialized(self) -> None:
        self._check(self._lib.ipg_mark_initialized(self._h))

    def newton_iterations(self):
        it = np.empty(2 * self.n, dtype=np.int32)
        st = np.empty(2 * self.n, dtype=np.int32)
        self._check(self._lib.ipg_get_newton_iterations(self._h, _ptr(it), _ptr(st)))
        return it, st

    def last_leapfrog_ms(self):
        ms, k = ct.c_double(), ct.c_int()
        self._check(self._lib.ipg_last_leapfrog_ms(self._h, ct.byref(ms), ct.byref(k)))
        return ms.value, k.value

    # -- adjoint -------------------------------------------------------------
    def forward(self, checkpoint_every: int = 0):
        """E_T and the T^tautau-weighted eps2 from the fresh tau = 0 state;
        saves checkpoints for :meth:`backward`: every state with
        checkpoint_every = 1 (no time reversal in the backward), every k-th
        with k > 1, and 0 picks 1 when the states fit in half of the free
        device memory, else ~sqrt(steps)."""
        et, e2 = ct.c_double(), ct.c_double()
        self._check(self._lib.ipg_forward(self._h, checkpoint_every, ct.byref(et), ct.byref(e2)))
        return et.value, e2.value

    def adjoint_stats(self):
        """Device ms of the last forward and backward."""
        f, b = ct.c_double(), ct.c_double()
        self._check(self._lib.ipg_adjoint_stats(self._h, ct.byref(f), ct.byref(b)))
        return f.value, b.value

    def backward(self, w_ET: float = 1.0, w_eps2: float = 0.0, inputs: bool = False,
                 rho: bool = False, out: dict | None = None):
        """Gradient of w_ET E_T + w_eps2 eps2 w.r.t. the tau = 0 fields:
        dict field -> (N*N, 3, 3) complex array (dL/dRe + i dL/dIm). With
        inputs, also "g2mu" -> (2, N*N) (nuclei A, B); with rho, "rho" ->
        (2, Ny, N*N, 8). ``out`` may hold float64 arrays to fill instead of
        new ones (page-locked arrays make the copies run at link speed):
        "state" (6*18*N*N), "g2mu" (2*N*N), "rho" (16*Ny*N*N); the returned
        arrays are views of them."""
        out = out or {}
        g = out.get("state")
        g = np.empty(6 * 18 * self.n) if g is None else g
        gm = (out.get("g2mu") if out.get("g2mu") is not None else np.empty(2 * self.n)) \
            if inputs else None
        gr = (out.get("rho") if out.get("rho") is not None
              else np.empty(2 * self.cfg.Ny * self.n * 8)) if rho else None
        for a, size in ((g, 6 * 18 * self.n), (gm, 2 * self.n),
                        (gr, 16 * self.cfg.Ny * self.n)):
            if a is not None and (a.dtype != np.float64 or a.size != size
                                  or not a.flags.c_contiguous):
                raise ValueError(f"output buffer needs {size} contiguous float64")
        self._check(self._lib.ipg_backward(
            self._h, w_ET, w_eps2, _ptr(g), _ptr(gm) if gm is not None else None,
            _ptr(gr) if gr is not None else None))
        # (re, im) pairs read as complex numbers without a copy
        z = g.reshape(6, self.n, 18).view(np.complex128)
        res = {f: z[k].reshape(self.n, 3, 3) for k, f in enumerate((UX, UY, E1, E2, PHI, PI))}
        if gm is not None:
            res["g2mu"] = gm.reshape(2, self.n)
        if gr is not None:
            res["rho"] = gr.reshape(2, self.cfg.Ny, self.n, 8)
        return res

    def kernel_launches(self) -> int:
        c = ct.c_longlong()
        self._check(self._lib.ipg_kernel_launches(self._h, ct.byref(c)))
        return c.value


@dataclass
class TuneReport:
    variant: int
    tile_rows: int
    threads_per_block: int
    blocks_per_sm: int
    grid: int
    ms_per_step: float
    candidates: int
    from_cache: int


class Batch:
    """Events advanced together: one persistent launch per leapfrog step over
    every site of every event, the step sequence replayed as a CUDA graph
    (``ipg_batch_*``). The events are :class:`Event` objects sharing device,
    precision and time grid; the batch keeps references to them."""

    def __init__(self, events):
        self.events = list(events)
        self._lib = lib()
        arr = (ct.c_void_p * len(self.events))(*[e._h.value for e in self.events])
        h = ct.c_void_p()
        st = self._lib.ipg_batch_create(arr, len(self.events), ct.byref(h))
        self._h = h
        if st != 0:
            msg = self._lib.ipg_batch_last_error(h).decode() if h.value else "allocation"
            self.close()
            raise IPGError(st, msg)

    def _check(self, st: int, allow=()):
        if st != 0 and st not in allow:
            raise IPGError(st, self._lib.ipg_batch_last_error(self._h).decode())
        return st

    def init_fields(self, allow_nonconverged: bool = False):
        """Initial conditions of every event, side by side on the GPU."""
        reps = (_InitReport * len(self.events))()
        self._check(self._lib.ipg_batch_init(self._h, reps), (3,) if allow_nonconverged else ())
        return [InitReport(*(getattr(r, f) for f, _ in _InitReport._fields_)) for r in reps]

    def tune(self) -> TuneReport:
        rep = _TuneReport()
        self._check(self._lib.ipg_batch_tune(self._h, ct.byref(rep)))
        return TuneReport(*(getattr(rep, f) for f, _ in _TuneReport._fields_))

    def run(self):
        res = (_Result * len(self.events))()
        self._check(self._lib.ipg_batch_run(self._h, res))
        out = []
        for r in res:
            vals = {f: getattr(r, f) for f, _ in _Result._fields_}
            vals["eccentricity"] = list(r.eccentricity)
            vals["psi"] = list(r.psi)
            out.append(Result(**vals))
        return out

    def set_shape(self, variant: int, blocks_per_sm: int) -> None:
        self._check(self._lib.ipg_batch_set_shape(self._h, variant, blocks_per_sm))

    def stats(self):
        ev, tot, k = ct.c_double(), ct.c_double(), ct.c_longlong()
        self._check(self._lib.ipg_batch_stats(self._h, ct.byref(ev), ct.byref(tot), ct.byref(k)))
        return ev.value, tot.value, k.value

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.ipg_batch_destroy(self._h)
            self._h = ct.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
