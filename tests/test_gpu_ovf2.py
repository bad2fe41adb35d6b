"""loadovf2mag / saveovf2mag through a context on cuda:0 (Boris/Commands.cpp:5025,5192) against the
reference's own OVF 2.0 reader, renormalisation and remap (oracle/_ref/libborisref.so): M after the
load equals the reference's loaded VEC bit for bit (FP64 context), and the saved file equals the
reference writer's bytes for the same M."""
import os

import numpy as np
import pytest

from oracle_libs import reference, dp, ip
from test_ovf2 import ref_write, vortex

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def R():
    r = reference()
    if r is None:
        pytest.skip("reference build unavailable")
    return r


@pytest.mark.parametrize("mesh_n", [(16, 8, 2), (32, 16, 1), (12, 6, 3)])
@pytest.mark.parametrize("renorm", [0.0, 6e5])
def test_load_then_save_matches_reference(bm, R, tmp_path, mesh_n, renorm):
    src_n, h = (16, 8, 2), (5e-9, 5e-9, 3e-9)
    M = vortex(src_n, seed=9)
    src = tmp_path / "src.ovf"
    ref_write(R, str(src), M, src_n, h, (0.0, 0.0, 0.0), "bin8")
    want = np.zeros(3 * int(np.prod(mesh_n)))
    assert R.ref_ovf2_load(os.fsencode(str(src)), renorm, ip(np.asarray(mesh_n, dtype=np.int32)), dp(want)) == 0

    c = bm.Context(precision=bm.FP64)
    hm, origin = (4e-9, 4e-9, 2e-9), (1e-8, 0.0, 0.0)
    c.add_mesh(mesh_n, hm, origin)
    c.set_material(0, Ms=8e5, A=1.3e-11, alpha=0.3)
    c.setode("RK4", 1e-14)
    c.demag_field(0)                      # the device state exists before the load
    c.loadovf2mag(str(src), renormalize=renorm)
    got = c.get_m().reshape(-1)
    assert np.array_equal(got, want)

    for kind, norm in [("bin8", False), ("text", True)]:
        ours = tmp_path / "a" / ("out_%s.ovf" % kind)
        theirs = tmp_path / "b" / ("out_%s.ovf" % kind)
        ours.parent.mkdir(exist_ok=True)
        theirs.parent.mkdir(exist_ok=True)
        c.saveovf2mag(str(ours), data_type=kind, normalize=norm)
        ref_write(R, str(theirs), got, mesh_n, hm, origin, kind, 8e5 if norm else 1.0)
        assert ours.read_bytes() == theirs.read_bytes()
    c.close()


def test_load_refuses_empty_cells(bm, R, tmp_path):
    """Zero-length values (empty cells of the reference's mesh shape) are refused; M is unchanged."""
    n, h = (8, 4, 1), (5e-9, 5e-9, 3e-9)
    M = vortex(n, seed=2)
    c = bm.Context(precision=bm.FP64)
    c.add_mesh(n, h)
    c.set_material(0, Ms=8e5, A=1.3e-11, alpha=0.3)
    c.set_m(M)
    c.demag_field(0)
    Z = M.copy()
    Z[5] = 0.0
    p = tmp_path / "holes.ovf"
    ref_write(R, str(p), Z, n, h, (0.0, 0.0, 0.0), "bin8")
    with pytest.raises(bm.BorisError):
        c.loadovf2mag(str(p))
    assert np.array_equal(c.get_m(), M)
    c.close()

