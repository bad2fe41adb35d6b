"""ctypes access to the oracle (test infrastructure only).

  liboracle.so    oracle/oracle.c — the project's FP64 CPU restatement of the path
  libborisref.so  the reference's own CPU sources compiled by oracle/Makefile (demag,
                  stencils, multilayer convolution, OVF 2.0 reader and writer)

Both are built from oracle/Makefile when missing (the reference build only where the
reference tree is present; its .so travels with the repository otherwise).
"""
import ctypes
import os
import re
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "_build", "liboracle.so")
REF_SO = os.path.join(ORACLE_DIR, "_ref", "libborisref.so")


def _reference_tree():
    """Root of the reference source tree: $BORIS2_REFERENCE, else the default of oracle/Makefile's
    REF variable (the one recipe that names where the reference is mounted)."""
    env = os.environ.get("BORIS2_REFERENCE")
    if env:
        return env
    try:
        with open(os.path.join(ORACLE_DIR, "Makefile")) as f:
            for line in f:
                m = re.match(r"\s*REF\s*\?=\s*(\S+)", line)
                if m:
                    return m.group(1)
    except OSError:
        pass
    return ""


REF_TREE = _reference_tree()

P = ctypes.c_void_p
D = ctypes.c_double
I = ctypes.c_int
DP = ctypes.POINTER(ctypes.c_double)
IP = ctypes.POINTER(ctypes.c_int)

_orc = None
_ref = None


def dp(a):
    return a.ctypes.data_as(DP)


class MeshDesc(ctypes.Structure):
    _fields_ = [("nx", I), ("ny", I), ("nz", I), ("hx", D), ("hy", D), ("hz", D),
                ("Ms", D), ("A", D), ("D", D), ("alpha", D), ("grel", D), ("K1", D), ("K2", D),
                ("ea", D * 3), ("Ms_map", DP), ("K1_map", DP), ("modules", I),
                ("Ha", DP), ("nHa", I), ("Ha_tspan", D), ("pbc", I * 3)]


class OrcStats(ctypes.Structure):
    _fields_ = [("accepted", ctypes.c_long), ("rejected", ctypes.c_long), ("evals", ctypes.c_long),
                ("time", D), ("dT", D), ("last_lte", D)]


def oracle():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_SO):
            subprocess.run(["make", "-C", ORACLE_DIR, "oracle"], check=True, capture_output=True)
        L = ctypes.CDLL(ORACLE_SO)
        L.orc_demag_create.restype = P
        L.orc_demag_create.argtypes = [I, I, I, D, D, D, I, I, I]
        L.orc_demag_apply.restype = D
        L.orc_demag_apply.argtypes = [P, DP, DP, I]
        L.orc_demag_destroy.argtypes = [P]
        L.orc_solver_create.restype = P
        L.orc_solver_create.argtypes = [I, ctypes.POINTER(MeshDesc), I, D, D, D, D, D]
        L.orc_set_m.argtypes = [P, I, DP]
        L.orc_get_m.argtypes = [P, I, DP]
        L.orc_compute_heff.argtypes = [P, I, DP]
        L.orc_run.argtypes = [P, I, ctypes.POINTER(OrcStats)]
        L.orc_solver_destroy.argtypes = [P]
        L.orc_newell_f.restype = D
        L.orc_newell_f.argtypes = [D, D, D]
        L.orc_newell_g.restype = D
        L.orc_newell_g.argtypes = [D, D, D]
        L.orc_asymptotic.argtypes = [D, D, D, D, D, D, DP]
        L.orc_selfdemag.argtypes = [D, D, D, DP]
        L.orc_tensor.argtypes = [I, I, I, I, I, I, D, D, D, DP, DP]
        L.orc_kernels.argtypes = [I, I, I, I, I, I, D, D, D, DP, DP]
        L.orc_field_exchange.argtypes = [I, I, I, D, D, D, DP, D, DP, DP]
        L.orc_field_idmi.argtypes = [I, I, I, D, D, D, DP, D, D, DP, DP]
        L.orc_field_aniuni.argtypes = [I, DP, DP, DP, D, DP, DP]
        L.bm_oracle_fft.argtypes = [I, DP, I]
        L.orc_ml_create.restype = P
        L.orc_ml_create.argtypes = [I, IP, DP, DP, I, IP]
        L.orc_ml_info.argtypes = [P, IP, IP, IP, IP, DP, IP]
        L.orc_ml_eval.argtypes = [P, DP, DP]
        L.orc_ml_transfer.argtypes = [P, I, DP, DP, DP, DP]
        L.orc_ml_destroy.argtypes = [P]
        L.orc_solver_set_multilayer.argtypes = [P, DP, I, IP]
        L.orc_solver_set_evalspeedup.argtypes = [P, I]
        L.orc_solver_set_evalspeedup_self.argtypes = [P, I]
        L.orc_solver_get_mxh.argtypes = [P, DP]
        L.orc_solver_get_dmdt.argtypes = [P, DP]
        L.orc_selfdemag_metres.argtypes = [D, D, D, DP]
        L.orc_adjoint_rk4.argtypes = [ctypes.POINTER(MeshDesc), DP, DP, I, D, DP, DP, DP, DP]
        L.orc_solver_set_field_hook.argtypes = [P, I, P, P]
        L.orc_tensor_pbc.argtypes = [I, I, I, I, I, I, D, D, D, IP, DP, DP]
        L.orc_kernels_from_tensor.argtypes = [DP, DP, I, I, I, I, DP, DP]
        L.orc_pbc_dims.argtypes = [I, I, I, IP, IP]
        L.orc_selfdemag_pbc.argtypes = [D, D, D, IP, IP, DP]
        L.orc_demag_create_pbc.restype = P
        L.orc_demag_create_pbc.argtypes = [I, I, I, D, D, D, IP]
        L.orc_field_exchange_pbc.argtypes = [I, I, I, D, D, D, DP, D, DP, IP, DP]
        L.orc_field_idmi_pbc.argtypes = [I, I, I, D, D, D, DP, D, D, DP, IP, DP]
        L.orc_sm_create.restype = P
        L.orc_sm_create.argtypes = [I, IP, DP, DP, DP, IP]
        L.orc_sm_info.argtypes = [P, IP, DP, DP, ctypes.POINTER(ctypes.c_long)]
        L.orc_sm_eval.restype = D
        L.orc_sm_eval.argtypes = [P, DP, DP]
        L.orc_sm_destroy.argtypes = [P]
        L.orc_solver_set_supermesh.argtypes = [P, DP, DP, IP]
        _orc = L
    return _orc


def ref_available():
    return os.path.exists(REF_SO) or os.path.isdir(REF_TREE)


REFGPU_DIR = os.path.join(ROOT, "baseline", "_ref")
_refgpu = {}


def reference_gpu(precision="f32"):
    """The reference's own GPU demag convolution (ConvolutionCUDA<., DemagKernelCUDA>, cuFFT) built for
    sm_100a by baseline/Makefile, in FP32 ("f32", SINGLEPRECISION 1) or FP64 ("f64"); None when
    neither the .so nor the reference tree is present. Loading it needs no GPU; calling it does."""
    if precision not in _refgpu:
        so = os.path.join(REFGPU_DIR, "librefgpu_%s.so" % precision)
        if REF_TREE and os.path.isdir(REF_TREE):
            reference()   # the CPU objects it links
            subprocess.run(["make", "-C", os.path.join(ROOT, "baseline"), "-j8", "REF=" + REF_TREE], check=True,
                           capture_output=True)
        elif not os.path.exists(so):
            return None
        L = ctypes.CDLL(so)
        L.refgpu_create.restype = P
        L.refgpu_create.argtypes = [I, I, I, D, D, D, I]
        L.refgpu_set_m.argtypes = [P, DP]
        L.refgpu_eval.restype = D
        L.refgpu_eval.argtypes = [P, I]
        L.refgpu_get_h.argtypes = [P, DP]
        L.refgpu_destroy.argtypes = [P]
        _refgpu[precision] = L
    return _refgpu[precision]


class ReferenceGPUDemag:
    """One reference GPU convolution of an n, h mesh (kernels built on the GPU as the reference does
    by default)."""

    def __init__(self, n, h, precision="f32"):
        self.L = reference_gpu(precision)
        self.n = int(np.prod(n))
        self.h = self.L.refgpu_create(n[0], n[1], n[2], h[0], h[1], h[2], 1)
        assert self.h, "reference GPU convolution could not be built"

    def field(self, M):
        Mf = np.ascontiguousarray(np.asarray(M, dtype=np.float64).reshape(-1))
        assert self.L.refgpu_set_m(P(self.h), dp(Mf)) == 0
        H = np.zeros(3 * self.n)
        assert self.L.refgpu_get_h(P(self.h), dp(H)) == 0
        return H.reshape(-1, 3)

    def time(self, reps=20):
        ms = self.L.refgpu_eval(P(self.h), int(reps))
        assert ms > 0, "reference GPU evaluation failed"
        return ms

    def close(self):
        if self.h:
            self.L.refgpu_destroy(P(self.h))
            self.h = None

    def __del__(self):
        self.close()


def reference():
    """The reference's compiled CPU code (None when neither the .so nor the tree is present)."""
    global _ref
    if _ref is None:
        if os.path.isdir(REF_TREE):
            # incremental: rebuilds only what changed since the last build
            subprocess.run(["make", "-C", ORACLE_DIR, "-j8", "ref", "REF=" + REF_TREE], check=True, capture_output=True)
        elif not os.path.exists(REF_SO):
            return None
        L = ctypes.CDLL(REF_SO)
        L.ref_selfdemag.argtypes = [D, D, D, DP]
        L.ref_tensor.argtypes = [I, I, I, I, I, I, D, D, D, DP, DP]
        L.ref_kernels.argtypes = [I, I, I, D, D, D, DP, DP]
        L.ref_hdemag.argtypes = [I, I, I, D, D, D, DP, DP, DP]
        L.ref_demag_create.restype = P
        L.ref_demag_create.argtypes = [I, I, I, D, D, D]
        L.ref_demag_eval.restype = D
        L.ref_demag_eval.argtypes = [P, DP, DP]
        L.ref_demag_destroy.argtypes = [P]
        L.ref_exchange.argtypes = [I, I, I, D, D, D, DP, DP, DP, DP]
        L.ref_idmi.argtypes = [I, I, I, D, D, D, DP, DP, DP, DP, DP]
        L.ref_tensor_shifted.argtypes = [I, I, I, I, I, I, I, DP, DP, DP, I, DP, DP]
        L.ref_tensor_pbc.argtypes = [I, I, I, D, D, D, IP, DP, DP, IP]
        L.ref_kernels_pbc.argtypes = [I, I, I, D, D, D, IP, DP, DP]
        L.ref_hdemag_pbc.argtypes = [I, I, I, D, D, D, IP, DP, DP, DP]
        L.ref_stencil_pbc.argtypes = [I, I, I, D, D, D, IP, I, DP, DP, DP, DP, DP]
        L.ref_selfdemag_pbc.argtypes = [D, D, D, I, I, I, IP, DP]
        L.ref_sm_create.restype = P
        L.ref_sm_create.argtypes = [I, IP, DP, DP, DP, IP]
        L.ref_sm_info.argtypes = [P, IP, DP, DP]
        L.ref_sm_eval.restype = D
        L.ref_sm_eval.argtypes = [P, DP, DP]
        L.ref_sm_destroy.argtypes = [P]
        L.ref_ml_create.restype = P
        L.ref_ml_create.argtypes = [I, IP, DP, DP, I, IP]
        L.ref_ml_info.argtypes = [P, IP, IP, IP, IP, DP, IP]
        L.ref_ml_eval.argtypes = [P, DP, DP]
        L.ref_ml_transfer.argtypes = [P, I, DP, DP, DP, DP]
        L.ref_ml_destroy.argtypes = [P]
        L.ref_film_fields_create.restype = P
        L.ref_film_fields_create.argtypes = [I, I, I, D, D, D, I, D, D, D]
        L.ref_film_fields_add.argtypes = [P, DP, DP]
        L.ref_film_fields_destroy.argtypes = [P]
        L.ref_film_fields_demag.argtypes = [P, DP, DP]
        L.ref_ovf2_read.argtypes = [ctypes.c_char_p, IP, DP, DP, DP]
        L.ref_ovf2_write.argtypes = [ctypes.c_char_p, IP, DP, DP, DP, ctypes.c_char_p, D]
        L.ref_ovf2_load.argtypes = [ctypes.c_char_p, D, IP, DP]
        _ref = L
    return _ref


# ---------------------------------------------------------------- convenience wrappers
def orc_hdemag(M, n, h, N=None):
    """FP64 demag field of M (n cells x 3) on mesh n with cellsize h (oracle)."""
    nx, ny, nz = n
    if N is None:
        N = (2 * nx, 2 * ny, 2 * nz if nz > 1 else 1)
    L = oracle()
    d = L.orc_demag_create(nx, ny, nz, h[0], h[1], h[2], N[0], N[1], N[2])
    Mf = np.ascontiguousarray(np.asarray(M, dtype=np.float64).reshape(-1))
    H = np.zeros_like(Mf)
    dot = L.orc_demag_apply(P(d), dp(Mf), dp(H), 0)
    L.orc_demag_destroy(P(d))
    return H.reshape(-1, 3), dot


def ip(a):
    return a.ctypes.data_as(IP)


class MultiLayer:
    """The multilayered convolution of the oracle (which="oracle") or of the reference build
    (which="reference"). meshes: list of (n, h, origin); mode 0 3D, 1 2D, 2 2D-layered."""

    def __init__(self, meshes, mode=0, ncommon=None, which="oracle"):
        self.lib = oracle() if which == "oracle" else reference()
        self.pre = "orc_" if which == "oracle" else "ref_"
        self.meshes = meshes
        n3 = np.array([m[0] for m in meshes], dtype=np.int32).reshape(-1)
        h3 = np.array([m[1] for m in meshes], dtype=np.float64).reshape(-1)
        o3 = np.array([m[2] for m in meshes], dtype=np.float64).reshape(-1)
        self._nc = np.array(ncommon, dtype=np.int32) if ncommon is not None else None
        self.h = getattr(self.lib, self.pre + "ml_create")(len(meshes), ip(n3), dp(h3), dp(o3), mode,
                                                          ip(self._nc) if self._nc is not None else None)
        assert self.h
        self.ncell = [int(np.prod(m[0])) for m in meshes]

    def info(self):
        L = np.zeros(1, np.int32)
        nc = np.zeros(3, np.int32)
        lm = np.zeros(256, np.int32)
        tr = np.zeros(256, np.int32)
        rc = np.zeros(256 * 6)
        kk = np.zeros(256 * 256, np.int32)
        getattr(self.lib, self.pre + "ml_info")(P(self.h), ip(L), ip(nc), ip(lm), ip(tr), dp(rc), ip(kk))
        n = int(L[0])
        return {"L": n, "n_common": tuple(int(v) for v in nc), "layer_mesh": lm[:n].tolist(),
                "transfer": tr[:n].tolist(), "rects": rc[:6 * n].reshape(n, 6).copy(),
                "kinds": kk[:n * n].reshape(n, n).copy()}

    def eval(self, M):
        Mf = np.ascontiguousarray(np.asarray(M, dtype=np.float64).reshape(-1))
        H = np.zeros_like(Mf)
        getattr(self.lib, self.pre + "ml_eval")(P(self.h), dp(Mf), dp(H))
        return H.reshape(-1, 3)

    def transfer(self, layer, M, Hc, ncommon_cells):
        Mf = np.ascontiguousarray(np.asarray(M, dtype=np.float64).reshape(-1))
        Hcf = np.ascontiguousarray(np.asarray(Hc, dtype=np.float64).reshape(-1))
        Mc = np.zeros(3 * ncommon_cells)
        m = self.info()["layer_mesh"][layer]
        Hm = np.zeros(3 * self.ncell[m])
        rc = getattr(self.lib, self.pre + "ml_transfer")(P(self.h), layer, dp(Mf), dp(Mc), dp(Hcf), dp(Hm))
        assert rc == 0
        return Mc.reshape(-1, 3), Hm.reshape(-1, 3)

    def close(self):
        if self.h:
            getattr(self.lib, self.pre + "ml_destroy")(P(self.h))
            self.h = None

    def __del__(self):
        self.close()


def _i3(v):
    return (ctypes.c_int * 3)(*(int(x) for x in v))


def orc_hdemag_pbc(M, n, h, pbc):
    """FP64 demag field of M with PBC images per axis (oracle: the reference's algorithm, N = n along
    periodic axes)."""
    L = oracle()
    d = L.orc_demag_create_pbc(n[0], n[1], n[2], h[0], h[1], h[2], _i3(pbc))
    Mf = np.ascontiguousarray(np.asarray(M, dtype=np.float64).reshape(-1))
    H = np.zeros_like(Mf)
    dot = L.orc_demag_apply(P(d), dp(Mf), dp(H), 0)
    L.orc_demag_destroy(P(d))
    return H.reshape(-1, 3), dot


def ref_hdemag_pbc(M, n, h, pbc):
    R = reference()
    Mf = np.ascontiguousarray(np.asarray(M, dtype=np.float64).reshape(-1))
    H = np.zeros_like(Mf)
    e = np.zeros(1)
    assert R.ref_hdemag_pbc(n[0], n[1], n[2], h[0], h[1], h[2], _i3(pbc), dp(Mf), dp(H), dp(e)) == 0
    return H.reshape(-1, 3), e[0]


def pbc_dims(n, pbc):
    N3 = (ctypes.c_int * 3)()
    oracle().orc_pbc_dims(n[0], n[1], n[2], _i3(pbc), N3)
    return tuple(N3)


def orc_tensor_pbc(n, h, pbc):
    """(diag, odiag) on the PBC N grid, shape (Nz, Ny, Nx, 3) each."""
    N = pbc_dims(n, pbc)
    np_ = N[0] * N[1] * N[2]
    dg = np.zeros(3 * np_)
    od = np.zeros(3 * np_)
    oracle().orc_tensor_pbc(n[0], n[1], n[2], N[0], N[1], N[2], h[0], h[1], h[2], _i3(pbc), dp(dg), dp(od))
    return dg.reshape(N[2], N[1], N[0], 3), od.reshape(N[2], N[1], N[0], 3)


def ref_tensor_pbc(n, h, pbc):
    R = reference()
    N3 = (ctypes.c_int * 3)()
    assert R.ref_tensor_pbc(n[0], n[1], n[2], h[0], h[1], h[2], _i3(pbc), None, None, N3) == 0
    N = tuple(N3)
    np_ = N[0] * N[1] * N[2]
    dg = np.zeros(3 * np_)
    od = np.zeros(3 * np_)
    assert R.ref_tensor_pbc(n[0], n[1], n[2], h[0], h[1], h[2], _i3(pbc), dp(dg), dp(od), N3) == 0
    return dg.reshape(N[2], N[1], N[0], 3), od.reshape(N[2], N[1], N[0], 3)


def orc_kernels_pbc(n, h, pbc):
    """Octant spectra (kdiag, kodiag), each (Kz, Ky, Kx, 3), of the oracle's PBC convolution."""
    N = pbc_dims(n, pbc)
    dg, od = orc_tensor_pbc(n, h, pbc)
    K = (N[0] // 2 + 1, N[1] // 2 + 1, N[2] // 2 + 1)
    nk = K[0] * K[1] * K[2]
    kd = np.zeros(3 * nk)
    ko = np.zeros(3 * nk)
    oracle().orc_kernels_from_tensor(dp(np.ascontiguousarray(dg.reshape(-1))), dp(np.ascontiguousarray(od.reshape(-1))),
                                     n[2], N[0], N[1], N[2], dp(kd), dp(ko))
    return kd.reshape(K[2], K[1], K[0], 3), ko.reshape(K[2], K[1], K[0], 3)


def ref_kernels_pbc(n, h, pbc):
    """The reference's PBC kernel spectra; 2D: kodiag is Kxy only, returned in component 0."""
    N = pbc_dims(n, pbc)
    K = (N[0] // 2 + 1, N[1] // 2 + 1, N[2] // 2 + 1)
    nk = K[0] * K[1] * K[2]
    kd = np.zeros(3 * nk)
    ko = np.zeros(3 * nk)
    assert reference().ref_kernels_pbc(n[0], n[1], n[2], h[0], h[1], h[2], _i3(pbc), dp(kd), dp(ko)) == 0
    if n[2] == 1:
        k2 = ko[:nk].copy()
        ko = np.zeros(3 * nk)
        ko[0::3] = k2
    return kd.reshape(K[2], K[1], K[0], 3), ko.reshape(K[2], K[1], K[0], 3)


def orc_stencil_pbc(M, n, h, pbc, A, Ms, D=0.0, idmi=False):
    L = oracle()
    nc = n[0] * n[1] * n[2]
    Mf = np.ascontiguousarray(np.asarray(M, dtype=np.float64).reshape(-1))
    Msc = np.full(nc, float(Ms)) if np.isscalar(Ms) else np.ascontiguousarray(np.asarray(Ms, dtype=np.float64))
    H = np.zeros_like(Mf)
    if idmi:
        L.orc_field_idmi_pbc(n[0], n[1], n[2], h[0], h[1], h[2], dp(Mf), A, D, dp(Msc), _i3(pbc), dp(H))
    else:
        L.orc_field_exchange_pbc(n[0], n[1], n[2], h[0], h[1], h[2], dp(Mf), A, dp(Msc), _i3(pbc), dp(H))
    return H.reshape(-1, 3)


def ref_stencil_pbc(M, n, h, pbc, A, Ms, D=0.0, idmi=False):
    R = reference()
    nc = n[0] * n[1] * n[2]
    Mf = np.ascontiguousarray(np.asarray(M, dtype=np.float64).reshape(-1))
    Ac = np.full(nc, float(A))
    Dc = np.full(nc, float(D))
    Msc = np.full(nc, float(Ms)) if np.isscalar(Ms) else np.ascontiguousarray(np.asarray(Ms, dtype=np.float64))
    H = np.zeros_like(Mf)
    assert R.ref_stencil_pbc(n[0], n[1], n[2], h[0], h[1], h[2], _i3(pbc), 4 if idmi else 2, dp(Mf), dp(Ac), dp(Dc),
                             dp(Msc), dp(H)) == 0
    return H.reshape(-1, 3)


class SuperMesh:
    """The supermesh demag of the oracle (which="oracle") or of the reference build (which="reference").
    meshes: list of (n, h, origin); h_request: supermesh cellsize asked for; pbc: its images."""

    def __init__(self, meshes, h_request=(5e-9, 5e-9, 5e-9), pbc=(0, 0, 0), which="oracle"):
        self.lib = oracle() if which == "oracle" else reference()
        self.pre = "orc_" if which == "oracle" else "ref_"
        n3 = np.array([m[0] for m in meshes], dtype=np.int32).reshape(-1)
        h3 = np.array([m[1] for m in meshes], dtype=np.float64).reshape(-1)
        o3 = np.array([m[2] for m in meshes], dtype=np.float64).reshape(-1)
        hr = np.array(h_request, dtype=np.float64)
        self.h = getattr(self.lib, self.pre + "sm_create")(len(meshes), ip(n3), dp(h3), dp(o3), dp(hr), _i3(pbc))
        assert self.h
        self.ncell = [int(np.prod(m[0])) for m in meshes]

    def info(self):
        n = np.zeros(3, np.int32)
        h = np.zeros(3)
        r = np.zeros(6)
        out = {}
        if self.pre == "orc_":
            ne = ctypes.c_long(0)
            self.lib.orc_sm_info(P(self.h), ip(n), dp(h), dp(r), ctypes.byref(ne))
            out["nonempty"] = ne.value
        else:
            self.lib.ref_sm_info(P(self.h), ip(n), dp(h), dp(r))
        out.update({"n": tuple(int(v) for v in n), "h": tuple(h), "rect": r.reshape(2, 3)})
        return out

    def eval(self, M):
        Mf = np.ascontiguousarray(np.asarray(M, dtype=np.float64).reshape(-1))
        H = np.zeros_like(Mf)
        e = getattr(self.lib, self.pre + "sm_eval")(P(self.h), dp(Mf), dp(H))
        return H.reshape(-1, 3), e

    def close(self):
        if self.h:
            getattr(self.lib, self.pre + "sm_destroy")(P(self.h))
            self.h = None

    def __del__(self):
        self.close()


def ref_hdemag(M, n, h):
    R = reference()
    Mf = np.ascontiguousarray(np.asarray(M, dtype=np.float64).reshape(-1))
    H = np.zeros_like(Mf)
    e = np.zeros(1)
    rc = R.ref_hdemag(n[0], n[1], n[2], h[0], h[1], h[2], dp(Mf), dp(H), dp(e))
    assert rc == 0
    return H.reshape(-1, 3), e[0]


class OracleSolver:
    """Oracle solver over one or more meshes (a common time step, like ODECommon)."""

    def __init__(self, meshes, evaluation=0, dt=1e-13, tol=1e-4, dT_incr=2.0, dT_min=1e-15, dT_max=3e-12):
        self._keep = []
        arr = (MeshDesc * len(meshes))()
        for i, m in enumerate(meshes):
            d = arr[i]
            d.nx, d.ny, d.nz = m["n"]
            d.hx, d.hy, d.hz = m["h"]
            d.Ms = m.get("Ms", 8e5); d.A = m.get("A", 1.3e-11); d.D = m.get("D", 0.0)
            d.alpha = m.get("alpha", 0.5); d.grel = m.get("grel", 1.0)
            d.K1 = m.get("K1", 0.0); d.K2 = m.get("K2", 0.0)
            ea = m.get("ea", (0.0, 0.0, 1.0))
            en = np.linalg.norm(ea)
            for k in range(3):
                d.ea[k] = ea[k] / en if en > 0 else 0.0
            for key in ("Ms_map", "K1_map"):
                if m.get(key) is not None:
                    a = np.ascontiguousarray(np.asarray(m[key], dtype=np.float64).reshape(-1))
                    self._keep.append(a)
                    setattr(d, key, dp(a))
            d.modules = m.get("modules", 1 | 2 | 16)
            Ha = np.ascontiguousarray(np.asarray(m.get("Ha", (0.0, 0.0, 0.0)), dtype=np.float64).reshape(-1))
            self._keep.append(Ha)
            d.Ha = dp(Ha)
            d.nHa = Ha.size // 3
            d.Ha_tspan = m.get("Ha_tspan", 0.0)
            for k, v in enumerate(m.get("pbc", (0, 0, 0))):
                d.pbc[k] = int(v)
        self._arr = arr
        self._meshes = meshes
        self._ref_fields = []
        self.n = [m["n"][0] * m["n"][1] * m["n"][2] for m in meshes]
        self.h = oracle().orc_solver_create(len(meshes), arr, evaluation, dt, tol, dT_incr, dT_min, dT_max)

    def multilayer(self, origins, mode=0, ncommon=None):
        """Demag of all meshes with the demag bit as one multilayered convolution."""
        o3 = np.ascontiguousarray(np.asarray(origins, dtype=np.float64).reshape(-1))
        nc = np.array(ncommon, dtype=np.int32) if ncommon is not None else None
        self._keep += [o3, nc]
        rc = oracle().orc_solver_set_multilayer(P(self.h), dp(o3), mode, ip(nc) if nc is not None else None)
        assert rc == 0

    def evalspeedup(self, level, metres=False):
        """metres: the self term on cellsizes in metres, as the reference computes it."""
        assert oracle().orc_solver_set_evalspeedup_self(P(self.h), int(bool(metres))) == 0
        assert oracle().orc_solver_set_evalspeedup(P(self.h), int(level)) == 0

    def supermesh(self, origins, h_request=(5e-9, 5e-9, 5e-9), pbc=(0, 0, 0)):
        """Demag of all meshes with the demag bit as one supermesh convolution."""
        o3 = np.ascontiguousarray(np.asarray(origins, dtype=np.float64).reshape(-1))
        hr = np.array(h_request, dtype=np.float64)
        self._keep += [o3, hr]
        assert oracle().orc_solver_set_supermesh(P(self.h), dp(o3), dp(hr), _i3(pbc)) == 0

    def use_reference_fields(self, mesh=0):
        """Take this mesh's demag and exchange / iDMI terms from the reference's own compiled code
        (Convolution<DemagKernel> and the VEC_VC stencils, oracle/_ref); Zeeman, anisotropy, LLG
        and the RK stages stay the restatement's. Returns False when the reference build is absent."""
        R = reference()
        if R is None:
            return False
        m = self._meshes[mesh]
        mods = m.get("modules", 1 | 2 | 16) & (1 | 2 | 4)
        hnd = R.ref_film_fields_create(m["n"][0], m["n"][1], m["n"][2], m["h"][0], m["h"][1], m["h"][2], mods,
                                       m.get("Ms", 8e5), m.get("A", 1.3e-11), m.get("D", 0.0))
        assert hnd, "reference field object could not be built"
        self._ref_fields.append(hnd)
        fn = ctypes.cast(R.ref_film_fields_add, ctypes.c_void_p)
        assert oracle().orc_solver_set_field_hook(P(self.h), mesh, fn, P(hnd)) == 0
        return True

    def reference_hdemag(self, M, mesh=0):
        """H_demag of M from the reference's compiled convolution held for this mesh by
        use_reference_fields (kernels built once)."""
        hnd = self._ref_fields[mesh]
        Mf = np.ascontiguousarray(np.asarray(M, dtype=np.float64).reshape(-1))
        H = np.zeros_like(Mf)
        assert reference().ref_film_fields_demag(P(hnd), dp(Mf), dp(H)) == 0
        return H.reshape(-1, 3)

    def set_m(self, M, mesh=0):
        a = np.ascontiguousarray(np.asarray(M, dtype=np.float64).reshape(-1))
        oracle().orc_set_m(P(self.h), mesh, dp(a))

    def get_m(self, mesh=0):
        a = np.zeros(3 * self.n[mesh])
        oracle().orc_get_m(P(self.h), mesh, dp(a))
        return a.reshape(-1, 3)

    def heff(self, mesh=0):
        a = np.zeros(3 * self.n[mesh])
        oracle().orc_compute_heff(P(self.h), mesh, dp(a))
        return a.reshape(-1, 3)

    def run(self, steps):
        st = OrcStats()
        rc = oracle().orc_run(P(self.h), steps, ctypes.byref(st))
        assert rc == 0
        return {k: getattr(st, k) for k, _ in OrcStats._fields_}

    def get_mxh(self):
        """Get_mxh: the value of the last step that computed it; the next step computes it."""
        v = ctypes.c_double()
        assert oracle().orc_solver_get_mxh(P(self.h), ctypes.byref(v)) == 0
        return v.value

    def get_dmdt(self):
        """Get_dmdt: the value of the last step that computed it; the next step computes it."""
        v = ctypes.c_double()
        assert oracle().orc_solver_get_dmdt(P(self.h), ctypes.byref(v)) == 0
        return v.value

    def close(self):
        if self.h:
            oracle().orc_solver_destroy(P(self.h))
            self.h = None
        for hnd in getattr(self, "_ref_fields", []):
            reference().ref_film_fields_destroy(P(hnd))
        self._ref_fields = []

    def __del__(self):
        self.close()


def sphere_random(n, seed, Ms=1.0):
    """Per-cell unit vectors uniform on the sphere (seeded), scaled by Ms."""
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    return v * (np.asarray(Ms).reshape(-1, 1) if np.ndim(Ms) else Ms)


def tilted_z(n, seed, max_deg=15.0, Ms=1.0):
    """+z with per-cell tilts theta ~ U[0, max_deg], phi ~ U[0, 2 pi) (seeded)."""
    rng = np.random.default_rng(seed)
    th = np.deg2rad(rng.uniform(0.0, max_deg, n))
    ph = rng.uniform(0.0, 2 * np.pi, n)
    v = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], axis=1)
    return v * Ms


def orc_adjoint(mesh, m0, target, steps, dt):
    """FP64 loss and gradients (Ms map, K1 map, field samples) of the oracle's discrete RK4 adjoint.
    mesh: dict with n, h, Ms_map, K1_map, A, alpha, ea, modules, Ha (nHa x 3), Ha_tspan."""
    d = MeshDesc()
    d.nx, d.ny, d.nz = mesh["n"]
    d.hx, d.hy, d.hz = mesh["h"]
    d.Ms = 8e5; d.A = mesh.get("A", 1.3e-11); d.D = 0.0; d.alpha = mesh.get("alpha", 0.02)
    d.grel = mesh.get("grel", 1.0); d.K1 = 0.0; d.K2 = 0.0
    ea = mesh.get("ea", (0.0, 0.0, 1.0))
    for k in range(3):
        d.ea[k] = ea[k]
    keep = []
    for key in ("Ms_map", "K1_map"):
        a = np.ascontiguousarray(np.asarray(mesh[key], dtype=np.float64).reshape(-1))
        keep.append(a)
        setattr(d, key, dp(a))
    Ha = np.ascontiguousarray(np.asarray(mesh["Ha"], dtype=np.float64).reshape(-1))
    keep.append(Ha)
    d.Ha = dp(Ha)
    d.nHa = Ha.size // 3
    d.Ha_tspan = mesh["Ha_tspan"]
    d.modules = mesh.get("modules", 1 | 2 | 8 | 16)
    for k, v in enumerate(mesh.get("pbc", (0, 0, 0))):
        d.pbc[k] = int(v)
    n = int(np.prod(mesh["n"]))
    m0a = np.ascontiguousarray(np.asarray(m0, dtype=np.float64).reshape(-1))
    ta = np.ascontiguousarray(np.asarray(target, dtype=np.float64).reshape(-1))
    loss = np.zeros(1)
    gMs = np.zeros(n)
    gK = np.zeros(n)
    gHa = np.zeros(Ha.size)
    rc = oracle().orc_adjoint_rk4(ctypes.byref(d), dp(m0a), dp(ta), steps, dt, dp(loss), dp(gMs), dp(gK), dp(gHa))
    assert rc == 0
    return loss[0], gMs, gK, gHa.reshape(-1, 3)
