"""Output files written on the GPU (ipg_write_outputs) are byte-identical to
the host writers (ipg_write_hydro / ipg_write_tmunu, themselves pinned to the
reference's files) on the same run's observables, for resampled grids,
several eta slices, and values that send a file to the host formatter."""
import ctypes as ct

import numpy as np
import pytest

import ipglasma_b200 as ipg
from ipglasma_b200.synthetic import make_event

pytestmark = pytest.mark.gpu


def host_files(ev, hpath, tpath, size_output, L_output, eta_size, deta, gfactor):
    lib = ipg.lib()
    eps, u4, pi10, T10 = ev.observables()
    p = lambda a: np.ascontiguousarray(a).ctypes.data_as(ct.c_void_p)
    et = ct.c_double()
    assert lib.ipg_write_hydro(str(hpath).encode(), ev.N, ev.cfg.L, size_output, L_output,
                               eta_size, deta, ev.itmax, ev.dtau, p(eps), p(u4), p(pi10),
                               gfactor, ct.byref(et)) == 0
    assert lib.ipg_write_tmunu(str(tpath).encode(), ev.N, ev.cfg.L, size_output, L_output,
                               eta_size, deta, ev.itmax, ev.dtau, p(T10), gfactor) == 0
    return et.value


@pytest.fixture(scope="module", params=[ipg.FP64, ipg.FP32], ids=["fp64", "fp32"])
def event(request):
    N, L = 128, 20.0
    A, B, _, _ = make_event(N, L, "Pb", 6.0, 77)
    ev = ipg.Event(ipg.Config(size=N, L=L, Ny=10, maxtime=0.3, precision=request.param,
                              seed=11))
    ev.set_g2mu(A, B)
    ev.use_device_noise()
    ev.init_fields(allow_nonconverged=True)
    ev.run()
    yield ev
    ev.close()


@pytest.mark.parametrize("grid", [(None, None, 1, 0.0, 1.0), (100, 16.0, 1, 0.0, 1.0),
                                  (128, 20.0, 3, 0.5, 1.0), (64, 24.0, 2, 0.25, 1.0),
                                  (128, 20.0, 1, 0.0, 1e9)],
                         ids=["lattice", "coarser-smaller", "eta3", "beyond-lattice",
                              "host-fallback"])
def test_gpu_files_byte_identical(event, tmp_path, grid):
    size_output, L_output, eta_size, deta, gfactor = grid
    size_output = event.N if size_output is None else size_output
    L_output = event.cfg.L if L_output is None else L_output
    et_gpu = event.write_outputs(tmp_path / "h_gpu.dat", tmp_path / "t_gpu.dat", size_output,
                                 L_output, eta_size, deta, gfactor)
    et_host = host_files(event, tmp_path / "h_host.dat", tmp_path / "t_host.dat", size_output,
                         L_output, eta_size, deta, gfactor)
    for name in ("h", "t"):
        a = (tmp_path / f"{name}_gpu.dat").read_bytes()
        b = (tmp_path / f"{name}_host.dat").read_bytes()
        assert len(a) > 1000
        assert a == b, name
    assert et_gpu == et_host


def test_gpu_writer_needs_a_finished_run(tmp_path):
    ev = ipg.Event(ipg.Config(size=32, L=4.0, Ny=2, maxtime=0.1, precision=ipg.FP64, seed=1))
    with pytest.raises(ipg.IPGError):
        ev.write_outputs(tmp_path / "h.dat", None)
    ev.close()
