"""The output writers reproduce the reference's files byte for byte when fed
the reference's own observables (the golden fixtures hold both: the cell
values dumped by the harness and the files Evolution::run wrote)."""
import ctypes as ct

import numpy as np
import pytest

import ipglasma_b200 as ipg


def writer(name):
    fn = getattr(ipg.lib(), name)
    fn.restype = ct.c_int
    return fn


@pytest.mark.parametrize("case", ["blobs_n16", "blobs_n32"])
def test_hydro_and_tmunu_files_byte_identical(golden, tmp_path, case):
    g = golden(case)
    m = g["meta"]
    N, L, it, dtau = m["N"], m["L"], m["itmax"], m["dtau"]
    obs = g["obs"]
    n = N * N
    eps = np.ascontiguousarray(obs[0])
    u4 = np.ascontiguousarray(obs[1:5])
    T10 = np.ascontiguousarray(obs[5:15])
    pi10 = np.ascontiguousarray(obs[15:25])
    D = ct.c_double
    hydro = tmp_path / "hydro.dat"
    etot = ct.c_double()
    st = writer("ipg_write_hydro")(str(hydro).encode(), N, D(L), N, D(L), 1, D(0.0), it, D(dtau),
                                   eps.ctypes.data_as(ct.c_void_p), u4.ctypes.data_as(ct.c_void_p),
                                   pi10.ctypes.data_as(ct.c_void_p), D(1.0), ct.byref(etot))
    assert st == 0
    assert hydro.read_text() == str(g["hydro_file"])
    tm = tmp_path / "tmunu.dat"
    st = writer("ipg_write_tmunu")(str(tm).encode(), N, D(L), N, D(L), 1, D(0.0), it, D(dtau),
                                   T10.ctypes.data_as(ct.c_void_p), D(1.0))
    assert st == 0
    assert tm.read_text() == str(g["tmunu_file"])
    h = ct.create_string_buffer(128)
    t = ct.create_string_buffer(128)
    writer("ipg_output_names")(0, it, D(dtau), D(L / N), h, 128, t, 128)
    assert t.value.decode() == str(g["tmunu_name"])
    assert h.value.decode() == "epsilon-u-Hydro-TauHydro-0.dat"


@pytest.mark.parametrize("case", ["blobs_n16", "blobs_n32"])
def test_oracle_writers_match_reference_files(golden, oracle_port, tmp_path, case):
    """Pins the oracle's serial writers on the files the reference wrote."""
    g = golden(case)
    m = g["meta"]
    N, L, it, dtau = m["N"], m["L"], m["itmax"], m["dtau"]
    obs = g["obs"]
    oracle_port.write_hydro(tmp_path / "h.dat", N, L, N, L, 1, 0.0, it, dtau, obs[0], obs[1:5],
                            obs[15:25], 1.0)
    oracle_port.write_tmunu(tmp_path / "t.dat", N, L, N, L, 1, 0.0, it, dtau, obs[5:15], 1.0)
    assert (tmp_path / "h.dat").read_text() == str(g["hydro_file"])
    assert (tmp_path / "t.dat").read_text() == str(g["tmunu_file"])


def _wild(rng, rows, n):
    """Values over the whole double range: normals times 10^[-320, 300), with
    zeros, negative zeros and subnormals mixed in."""
    m = rng.standard_normal((rows, n)) * 10.0 ** rng.integers(-320, 300, (rows, n))
    m[:, rng.random(n) < 0.1] = 0.0
    m[:, rng.random(n) < 0.05] = -0.0
    return np.ascontiguousarray(m)


# (N, sizeOutput, L, LOutput, etaSizeOutput): same grid, coarser and finer
# resampling, output box larger than the lattice, odd N, several eta slices
STRESS = [(64, 64, 10.0, 10.0, 1), (64, 50, 10.0, 12.0, 3), (96, 128, 20.0, 18.0, 2),
          (33, 40, 7.0, 7.0, 1)]


@pytest.mark.parametrize("threads", ["1", "3", "8"])
@pytest.mark.parametrize("shape", STRESS)
def test_parallel_writers_match_oracle_on_stress_values(oracle_port, tmp_path, monkeypatch,
                                                        shape, threads):
    """The row-parallel to_chars writers give the serial printf("%g") files
    byte for byte, and the same total energy bit for bit, for any number of
    formatting threads."""
    monkeypatch.setenv("IPG_WRITER_THREADS", threads)
    N, so, L, LO, heta = shape
    n = N * N
    rng = np.random.default_rng(N * 1000 + so)
    eps, u4, pi10, T10 = _wild(rng, 1, n)[0], _wild(rng, 4, n), _wild(rng, 10, n), \
        _wild(rng, 10, n)
    eps[rng.random(n) < 0.3] = 1e-12       # below the hydro threshold
    T10[0, rng.random(n) < 0.3] = 1e-17    # below the Tmunu threshold
    it, dtau, deta, gf = 37, 0.1, 0.1, 1.3
    D = ct.c_double
    V = lambda a: a.ctypes.data_as(ct.c_void_p)  # noqa: E731
    etot = ct.c_double()
    st = writer("ipg_write_hydro")(str(tmp_path / "h.dat").encode(), N, D(L), so, D(LO), heta,
                                   D(deta), it, D(dtau), V(eps), V(u4), V(pi10), D(gf),
                                   ct.byref(etot))
    assert st == 0
    st = writer("ipg_write_tmunu")(str(tmp_path / "t.dat").encode(), N, D(L), so, D(LO), heta,
                                   D(deta), it, D(dtau), V(T10), D(gf))
    assert st == 0
    ref_etot = oracle_port.write_hydro(tmp_path / "ho.dat", N, L, so, LO, heta, deta, it, dtau,
                                       eps, u4, pi10, gf)
    oracle_port.write_tmunu(tmp_path / "to.dat", N, L, so, LO, heta, deta, it, dtau, T10, gf)
    assert (tmp_path / "h.dat").read_bytes() == (tmp_path / "ho.dat").read_bytes()
    assert (tmp_path / "t.dat").read_bytes() == (tmp_path / "to.dat").read_bytes()
    assert etot.value == ref_etot


def test_writer_reports_unwritable_path(tmp_path):
    D = ct.c_double
    z = np.zeros(10 * 16)
    st = writer("ipg_write_tmunu")(str(tmp_path / "no" / "such" / "t.dat").encode(), 4, D(1.0),
                                   4, D(1.0), 1, D(0.0), 1, D(0.1),
                                   z.ctypes.data_as(ct.c_void_p), D(1.0))
    assert st != 0
