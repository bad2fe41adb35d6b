"""OVF 2.0 magnetisation I/O (host code of the C ABI) against the reference's own reader and writer
(OVF2::Read_OVF2_VEC / Write_OVF2_VEC, Boris/OVF2_Handlers.cpp:364,701, compiled into
oracle/_ref/libborisref.so) and against the files the reference ships (tests/golden/ovf2_vortex.json).

Bars: values bit-exact; written files byte-identical to the reference writer's for every data type;
the same files accepted and refused by both readers."""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle_libs import reference, dp, ip, REF_TREE

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "ovf2_vortex.json")
EINVAL, EUNSUPPORTED = 1, 5


@pytest.fixture(scope="module")
def bm():
    import boris2_b200
    from boris2_b200 import build
    build.build()
    boris2_b200.lib()
    return boris2_b200


@pytest.fixture(scope="module")
def R():
    r = reference()
    if r is None:
        pytest.skip("reference build unavailable")
    return r


def ref_read(R, path):
    n3 = np.zeros(3, dtype=np.int32)
    h3 = np.zeros(3)
    r6 = np.zeros(6)
    if R.ref_ovf2_read(os.fsencode(path), ip(n3), dp(h3), dp(r6), None) != 0:
        return None
    data = np.zeros(3 * int(np.prod(n3)))
    assert R.ref_ovf2_read(os.fsencode(path), ip(n3), dp(h3), dp(r6), dp(data)) == 0
    return {"n": tuple(int(v) for v in n3), "h": tuple(h3), "rect": tuple(r6), "data": data.reshape(-1, 3)}


def ref_write(R, path, data, n, h, origin, kind, norm=1.0):
    n3 = np.asarray(n, dtype=np.int32)
    a = np.ascontiguousarray(np.asarray(data, dtype=np.float64).reshape(-1))
    rc = R.ref_ovf2_write(os.fsencode(path), ip(n3), dp(np.asarray(h, dtype=np.float64)),
                          dp(np.asarray(origin, dtype=np.float64)), dp(a), kind.encode(), float(norm))
    assert rc == 0


def vortex(n, seed=0, Ms=8e5):
    nx, ny, nz = n
    rng = np.random.default_rng(seed)
    x, y, z = np.meshgrid(np.arange(nx) - nx / 2 + 0.5, np.arange(ny) - ny / 2 + 0.5, np.arange(nz), indexing="xy")
    x = np.transpose(x, (2, 0, 1)).reshape(-1)
    y = np.transpose(y, (2, 0, 1)).reshape(-1)
    r = np.hypot(x, y) + 1e-9
    m = np.stack([-y / r, x / r, np.exp(-r * r / 4.0)], axis=1) + 0.05 * rng.standard_normal((nx * ny * nz, 3))
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    return Ms * m


# ------------------------------------------------------------------ the files the reference ships
def test_vortex_files_match_golden(bm, tmp_path):
    gold = json.load(open(GOLDEN))
    for name, g in gold.items():
        path = os.path.join(REF_TREE, "Boris", name)
        if not os.path.exists(path):
            pytest.skip("reference tree not present")
        f = bm.ovf2_read(path)
        assert f["n"] == tuple(g["n"])
        assert f["h"] == pytest.approx(g["h"], rel=0, abs=0)
        assert f["rect"] == pytest.approx(g["rect"], rel=0, abs=0)
        assert hashlib.sha256(f["data"].astype("<f8").tobytes()).hexdigest() == g["data_sha256"]
        # writing the values back gives the reference's file byte for byte
        out = tmp_path / name
        bm.ovf2_write(str(out), f["data"], f["n"], f["h"], f["rect"][:3], "bin8")
        raw = out.read_bytes()
        assert len(raw) == g["file_bytes"]
        assert hashlib.sha256(raw).hexdigest() == g["file_sha256"]


def test_vortex_files_read_like_reference(bm, R):
    for name in ["vortex_hh_clk_up.ovf", "vortex_hh_cclk_dn.ovf"]:
        path = os.path.join(REF_TREE, "Boris", name)
        if not os.path.exists(path):
            pytest.skip("reference tree not present")
        a = bm.ovf2_read(path)
        b = ref_read(R, path)
        assert a["n"] == b["n"] and a["h"] == b["h"] and a["rect"] == b["rect"]
        assert np.array_equal(a["data"], b["data"])


# ------------------------------------------------------------------ writer: byte-identical output
@pytest.mark.parametrize("kind", ["bin8", "bin4", "text"])
@pytest.mark.parametrize("n,h,origin,norm", [
    ((16, 8, 1), (5e-9, 5e-9, 3e-9), (0.0, 0.0, 0.0), 1.0),
    ((10, 6, 4), (2e-9, 3e-9, 1.5e-9), (1e-7, -4e-8, 2.5e-9), 8e5),
    ((7, 5, 3), (1e-9, 1e-9, 1e-9), (3.3e-9, 0.0, -1e-9), 1.0),
])
def test_writer_matches_reference_bytes(bm, R, tmp_path, kind, n, h, origin, norm):
    M = vortex(n, seed=sum(n))
    ours = tmp_path / "a" / "state.ovf"
    theirs = tmp_path / "b" / "state.ovf"
    ours.parent.mkdir()
    theirs.parent.mkdir()
    bm.ovf2_write(str(ours), M, n, h, origin, kind, norm)
    ref_write(R, str(theirs), M, n, h, origin, kind, norm)
    assert ours.read_bytes() == theirs.read_bytes()


@pytest.mark.parametrize("kind", ["bin8", "bin4", "text"])
def test_round_trip_both_readers(bm, R, tmp_path, kind):
    n, h, origin = (12, 9, 2), (4e-9, 5e-9, 6e-9), (2e-8, 0.0, 1e-9)
    M = vortex(n, seed=3)
    p = tmp_path / ("m_%s.ovf" % kind)
    bm.ovf2_write(str(p), M, n, h, origin, kind)
    a = bm.ovf2_read(str(p))
    b = ref_read(R, str(p))
    assert a["n"] == n == b["n"]
    assert np.allclose(a["h"], h, rtol=1e-12, atol=0)
    assert np.array_equal(a["data"], b["data"])
    if kind == "bin8":
        assert np.array_equal(a["data"], M)
    elif kind == "bin4":
        assert np.array_equal(a["data"], M.astype(np.float32).astype(np.float64))
    else:
        assert np.allclose(a["data"], M, rtol=1e-5, atol=0)


# ------------------------------------------------------------------ reader: variants and refusals
def _file(path, header_lines, payload=b"", eol="\n", first="# OOMMF OVF 2.0"):
    text = eol.join([first] + header_lines) + eol
    with open(path, "wb") as fh:
        fh.write(text.encode() + payload)


def _header(n=(3, 2, 1), h=(1.0, 1.0, 1.0), unit="m", meshtype="rectangular", valuedim="3", rect=None,
            extra=()):
    if rect is None:
        rect = (0, 0, 0, n[0] * h[0], n[1] * h[1], n[2] * h[2])
    lines = ["# Segment count: 1", "# Begin: Segment", "# Begin: Header", "# Title: t", "# Desc: anything",
             "# meshunit: " + unit, "# meshtype: " + meshtype, "# valueunits: A/m A/m A/m"]
    lines += ["# %smin: %r" % (a, v) for a, v in zip("xyz", rect[:3])]
    lines += ["# %smax: %r" % (a, v) for a, v in zip("xyz", rect[3:])]
    lines += ["# %snodes: %d" % (a, v) for a, v in zip("xyz", n)]
    lines += ["# %sstepsize: %r" % (a, v) for a, v in zip("xyz", h)]
    lines += ["# valuedim: " + valuedim] + list(extra) + ["# End: Header"]
    return lines


def _bin8(vals, check=123456789012345.0):
    return np.concatenate([[check], np.asarray(vals, dtype=np.float64).reshape(-1)]).astype("<f8").tobytes()


def _status(bm, path):
    import ctypes
    n3 = (ctypes.c_int * 3)()
    return bm.lib().bm_ovf2_read(os.fsencode(str(path)), n3, None, None, None, 0)


def test_reader_variants_match_reference(bm, R, tmp_path):
    vals = np.arange(18, dtype=np.float64) * 1.5 - 7.0
    cases = {
        "crlf_capital_data": (_header(), b"# Begin: Data Binary 8\r\n" + _bin8(vals), "\r\n"),
        "nm_unit": (_header(h=(2.0, 3.0, 4.0), unit="nm"), b"# Begin: data binary 8\n" + _bin8(vals), "\n"),
        "binary4": (_header(), b"# Begin: data binary 4\n" +
                    np.concatenate([[1234567.0], vals]).astype("<f4").tobytes(), "\n"),
        "text_tabs_short_row": (_header(), b"# Begin: data text\n" + b"1\t2\t3\n 4 5 6\n7 8\n10 11 12 13\n"
                                b"-1e-3 2.5E2 3\n0 0 1\n", "\n"),
    }
    for name, (hdr, payload, eol) in cases.items():
        p = tmp_path / (name + ".ovf")
        text = eol.join(["# OOMMF OVF 2.0"] + hdr) + eol
        p.write_bytes(text.encode() + payload)
        a = bm.ovf2_read(str(p))
        b = ref_read(R, str(p))
        assert b is not None, name
        assert a["n"] == b["n"] and np.allclose(a["h"], b["h"], rtol=1e-15, atol=0), name
        assert a["rect"] == b["rect"], name
        assert np.array_equal(a["data"], b["data"]), name
    # nm scales lengths by 1e-9
    a = bm.ovf2_read(str(tmp_path / "nm_unit.ovf"))
    assert np.allclose(a["h"], (2e-9, 3e-9, 4e-9), rtol=1e-15, atol=0)
    # a row with fewer than three numbers leaves that cell at zero
    a = bm.ovf2_read(str(tmp_path / "text_tabs_short_row.ovf"))
    assert np.array_equal(a["data"][2], [0.0, 0.0, 0.0]) and np.array_equal(a["data"][3], [10.0, 11.0, 12.0])


def test_reader_refusals_match_reference(bm, R, tmp_path):
    vals = np.ones(18)
    good = b"# Begin: data binary 8\n" + _bin8(vals)
    cases = {
        "version": (dict(), good, "# OOMMF OVF 1.0", EUNSUPPORTED),
        "meshtype": (dict(meshtype="irregular"), good, None, EINVAL),
        "valuedim": (dict(valuedim="1"), good, None, EINVAL),
        "unit": (dict(unit="um"), good, None, EINVAL),
        "check_value": (dict(), b"# Begin: data binary 8\n" + _bin8(vals, check=1.0), None, EINVAL),
        "nodes_mismatch": (dict(rect=(0, 0, 0, 4.0, 2.0, 1.0)), good, None, EINVAL),
    }
    for name, (kw, payload, first, code) in cases.items():
        p = tmp_path / (name + ".ovf")
        _file(p, _header(**kw), payload, first=first or "# OOMMF OVF 2.0")
        assert ref_read(R, str(p)) is None, name
        assert _status(bm, p) == code, name
    assert _status(bm, tmp_path / "missing.ovf") == EINVAL
    # without a data segment the reference returns no error and an empty mesh (which its
    # loadovf2mag would then map to an all-zero M); this reader refuses the file instead
    for name, payload in {"no_data": b"", "unknown_data_kind": b"# Begin: data binary 2\n" + _bin8(vals)}.items():
        p = tmp_path / (name + ".ovf")
        _file(p, _header(), payload)
        assert ref_read(R, str(p))["n"] == (0, 0, 0), name
        assert _status(bm, p) == EINVAL, name


def test_truncated_file_refused(bm, tmp_path):
    """The reference reads past the end silently; this reader refuses a file that ends early."""
    p = tmp_path / "short.ovf"
    _file(p, _header(), b"# Begin: data binary 8\n" + _bin8(np.ones(17)))
    with pytest.raises(bm.BorisError):
        bm.ovf2_read(str(p))
    import ctypes
    n3 = (ctypes.c_int * 3)()
    data = np.zeros(3)   # capacity too small for 6 cells
    _file(p, _header(), b"# Begin: data binary 8\n" + _bin8(np.ones(18)))
    assert bm.lib().bm_ovf2_read(os.fsencode(str(p)), n3, None, None, bm._dp(data), 3) == EINVAL


def test_writer_refusals(bm, tmp_path):
    M = np.ones((6, 3))
    with pytest.raises(bm.BorisError):
        bm.ovf2_write(str(tmp_path / "x.ovf"), M, (3, 2, 1), (1e-9,) * 3, data_type="bin2")
    with pytest.raises(bm.BorisError):
        bm.ovf2_write(str(tmp_path / "x.ovf"), M, (3, 2, 1), (1e-9, 0.0, 1e-9))
    with pytest.raises(bm.BorisError):
        bm.ovf2_write(str(tmp_path / "x.ovf"), M, (3, 2, 1), (1e-9,) * 3, norm=0.0)
    with pytest.raises(bm.BorisError):
        bm.ovf2_write(str(tmp_path / "no_such_dir" / "x.ovf"), M, (3, 2, 1), (1e-9,) * 3)


# ------------------------------------------------------------------ load path: renormalise + remap
@pytest.mark.parametrize("dst", [(16, 8, 1), (32, 16, 1), (8, 4, 1), (11, 13, 1), (16, 8, 3), (5, 3, 2)])
@pytest.mark.parametrize("renorm", [0.0, 1.0, 4.8e5])
def test_load_path_matches_reference(bm, R, tmp_path, dst, renorm):
    src_n, h = (16, 8, 2), (5e-9, 5e-9, 3e-9)
    M = vortex(src_n, seed=5)
    M[7] = 0.0                      # an empty cell stays empty under renormalisation
    p = tmp_path / "src.ovf"
    ref_write(R, str(p), M, src_n, h, (0.0, 0.0, 0.0), "bin8")
    want = np.zeros(3 * int(np.prod(dst)))
    assert R.ref_ovf2_load(os.fsencode(str(p)), renorm, ip(np.asarray(dst, dtype=np.int32)), dp(want)) == 0
    f = bm.ovf2_read(str(p))
    d = f["data"]
    if abs(renorm) > 1e-12:
        d = bm.renormalize(d, renorm)
    got = bm.map_cells(d, f["n"], dst)
    assert np.array_equal(got.reshape(-1), want)
