"""The FP32 form's Wilson lines against the FP64 form's on the same event.

On FP32 contexts the Poisson transforms run in FP32 and each sheet's
exponential exp(-i A_k.t) is taken in FP32 by scaling and squaring, while
the ordered product over the Ny sheets is accumulated in FP64 and
reunitarised in FP64 after every sheet batch (Init.cpp:1678-1849 is the FP64
path the plain form follows). V_A and V_B of the two forms agree to FP32
accuracy and the FP32 form's V stay in SU(3) to FP64 rounding."""
import numpy as np
import pytest

import ipglasma_b200 as ipg

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,L,nucleus,b", [(256, 30.0, "Au", 2.0), (512, 40.0, "Pb", 6.0)])
def test_fp32_wilson_lines_close_to_fp64(N, L, nucleus, b):
    from ipglasma_b200.synthetic import make_event

    A, B, _, _ = make_event(N, L, nucleus, b, seed=17)
    V = {}
    for prec in (ipg.FP64, ipg.FP32):
        with ipg.Event(ipg.Config(size=N, L=L, Ny=50, maxtime=0.2, seed=23, precision=prec,
                                  newton_mode=1, newton_tolerance=1e-6)) as ev:
            ev.set_g2mu(A, B)
            ev.use_device_noise()
            ev.init_fields(allow_nonconverged=True)
            V[prec] = (ev.get_field(ipg.VA), ev.get_field(ipg.VB))
    worst = 0.0
    for v32, v64 in zip(V[ipg.FP32], V[ipg.FP64]):
        gap = float(np.abs(v32 - v64).max())
        worst = max(worst, gap)
        assert gap < 2e-5, gap
        # unitarity of the FP32 form's lines: V V^dag = 1 to FP64 rounding
        vvd = v32 @ np.conj(np.swapaxes(v32, -1, -2))
        assert np.abs(vvd - np.eye(3)).max() < 1e-13
        assert np.abs(np.linalg.det(v32) - 1).max() < 1e-13
    print("FP32WILSON", N, nucleus, worst)
