"""CPU tests of the supermesh demag (SDemag with the multilayered convolution off): the oracle's
restatement against the reference's own compiled code (oracle/_ref: the supermesh rectangle and
cells of SuperMesh::UpdateConfiguration, the weighted VEC mesh transfer over several meshes,
Convolution<DemagKernel> with PBC, SDemag's energy), and the oracle solver in supermesh mode against
the per-mesh convolution where the two must agree."""
import numpy as np
import pytest

from oracle_libs import SuperMesh, OracleSolver, reference, orc_hdemag, sphere_random

# (meshes [(n, h, origin)], requested supermesh cellsize, supermesh PBC images)
CASES = [
    # two films stacked with a gap, same cellsize
    ([((16, 8, 1), (5e-9, 5e-9, 3e-9), (0, 0, 0)), ((12, 8, 1), (5e-9, 5e-9, 3e-9), (0, 0, 6e-9))], (5e-9, 5e-9, 3e-9),
     (0, 0, 0)),
    # different cellsizes and offsets; the supermesh cellsize adjusted to divide the rectangle
    ([((16, 8, 2), (4e-9, 4e-9, 3e-9), (0, 0, 0)), ((10, 6, 1), (5e-9, 6e-9, 4e-9), (8e-9, 10e-9, 8e-9))],
     (5e-9, 5e-9, 3.5e-9), (0, 0, 0)),
    # side by side in x with a gap, one cell thick
    ([((20, 10, 1), (3e-9, 3e-9, 3e-9), (0, 0, 0)), ((8, 8, 1), (3e-9, 3e-9, 3e-9), (80e-9, 0, 0))], (4e-9, 4e-9, 3e-9),
     (0, 0, 0)),
    # a bilayer on a finer z grid with x, y PBC
    ([((16, 16, 1), (4e-9, 4e-9, 3e-9), (0, 0, 0)), ((16, 16, 1), (4e-9, 4e-9, 3e-9), (0, 0, 5e-9))], (4e-9, 4e-9, 1e-9),
     (3, 3, 0)),
    # three meshes, one overlapping another's footprint
    ([((12, 12, 2), (2e-9, 2e-9, 2e-9), (0, 0, 0)), ((6, 6, 2), (4e-9, 4e-9, 2e-9), (4e-9, 4e-9, 4e-9)),
      ((8, 4, 1), (3e-9, 3e-9, 3e-9), (30e-9, 0, 0))], (3e-9, 3e-9, 2e-9), (0, 0, 0)),
    # the reference's default supermesh cellsize (5 nm) over a 4 nm mesh
    ([((10, 10, 3), (4e-9, 4e-9, 4e-9), (0, 0, 0))], (5e-9, 5e-9, 5e-9), (0, 0, 0)),
]


def _ids(c):
    return "%dmesh_h%.1f_pbc%d%d%d" % (len(c[0]), c[1][0] * 1e9, *c[2])


def need_ref():
    if reference() is None:
        pytest.skip("reference CPU build unavailable")


@pytest.mark.parametrize("case", CASES, ids=_ids)
def test_supermesh_geometry_vs_reference(case):
    need_ref()
    meshes, hr, pbc = case
    o = SuperMesh(meshes, hr, pbc, "oracle")
    r = SuperMesh(meshes, hr, pbc, "reference")
    io, ir = o.info(), r.info()
    assert io["n"] == ir["n"]
    assert np.allclose(io["h"], ir["h"], rtol=1e-14, atol=0)
    assert np.allclose(io["rect"], ir["rect"], rtol=0, atol=1e-20)


@pytest.mark.parametrize("case", CASES, ids=_ids)
def test_supermesh_field_and_energy_vs_reference(case):
    need_ref()
    meshes, hr, pbc = case
    o = SuperMesh(meshes, hr, pbc, "oracle")
    r = SuperMesh(meshes, hr, pbc, "reference")
    rng = np.random.default_rng(len(meshes) + sum(pbc))
    M = rng.normal(size=(sum(o.ncell), 3)) * 8e5
    H, e = o.eval(M)
    Hr, er = r.eval(M)
    assert np.abs(H - Hr).max() <= 1e-9 * np.abs(Hr).max()
    assert abs(e - er) <= 1e-9 * abs(er)


def test_supermesh_on_the_mesh_grid_is_the_mesh_convolution():
    """One mesh whose grid is the supermesh grid: the transfers are the identity and the field is the
    mesh's own demag field."""
    n, h = (12, 10, 3), (4e-9, 4e-9, 3e-9)
    sm = SuperMesh([(n, h, (0, 0, 0))], h, (0, 0, 0))
    M = sphere_random(int(np.prod(n)), seed=3, Ms=8e5)
    H, _ = sm.eval(M)
    Href, _ = orc_hdemag(M, n, h)
    assert np.abs(H - Href).max() <= 1e-12 * np.abs(Href).max()


def test_supermesh_solver_matches_per_mesh_demag_on_one_grid():
    """The oracle solver in supermesh mode over one mesh on the supermesh grid follows the per-mesh
    convolution's trajectory."""
    mesh = dict(n=(16, 8, 2), h=(5e-9, 5e-9, 3e-9), Ms=8e5, A=1.3e-11, alpha=0.5, modules=1 | 2 | 16, Ha=(1e3, 0, 0))
    M = sphere_random(256, seed=8, Ms=8e5)
    a = OracleSolver([mesh], evaluation=0, dt=1e-13)
    a.set_m(M)
    a.run(10)
    b = OracleSolver([mesh], evaluation=0, dt=1e-13)
    b.supermesh([(0.0, 0.0, 0.0)], h_request=mesh["h"])
    b.set_m(M)
    b.run(10)
    assert np.abs(a.get_m() - b.get_m()).max() / 8e5 < 1e-12
