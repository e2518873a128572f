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
