"""The same-box reference GPU bar: the reference's own GPU demag convolution
(ConvolutionCUDA<., DemagKernelCUDA> with cuFFT, Boris/ConvolutionCUDA.h:383,478), built for sm_100a
from its sources by baseline/Makefile, must compute the same field as the reference's CPU build
before its time is compared with this path's (bench.py). FP64 build within 1e-9 of max |H|, FP32
build within 1e-5; this path's mixed and FP64 fields against the FP64 bar likewise."""
import numpy as np
import pytest

from oracle_libs import ReferenceGPUDemag, reference, reference_gpu, ref_hdemag, sphere_random

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [(64, 48, 1), (32, 24, 8), (40, 32, 5)])
def test_reference_gpu_bar_matches_reference_cpu(bm, n):
    if reference() is None or reference_gpu("f32") is None:
        pytest.skip("reference builds absent")
    h = (3e-9, 3e-9, 2e-9)
    M = sphere_random(int(np.prod(n)), seed=sum(n), Ms=8e5)
    Href, _ = ref_hdemag(M, n, h)
    scale = np.abs(Href).max()
    for prec, tol in (("f64", 1e-9), ("f32", 1e-5)):
        g = ReferenceGPUDemag(n, h, prec)
        H = g.field(M)
        g.close()
        assert np.abs(H - Href).max() / scale < tol, prec
    for prec, tol in ((bm.FP64, 1e-9), (bm.MIXED, 1e-5)):
        c = bm.Context(precision=prec)
        c.add_mesh(n, h)
        c.set_modules(0, bm.DEMAG)
        c.set_m(M)
        assert np.abs(c.demag_field() - Href).max() / scale < tol
        assert c.time_demag(0, reps=3) > 0
        c.close()
