"""boris2_b200 — B200-native micromagnetic field-and-integrate path behind a C ABI.

Python access to ``libboris_b200.so`` (see include/boris_b200.h) through ctypes. The
names follow the reference's command and module vocabulary:

=====================  ============================================================
this module            reference (Boris2)
=====================  ============================================================
``Context``            SuperMesh + ODECommon (one simulation, one GPU)
``add_mesh``           a ferromagnetic Mesh with n, h, meshRect
``set_material``       MeshParams (Ms, A, D, alpha, grel, K1, K2, mcanis_ea1)
``set_modules``        addmodule / delmodule (demag, exchange, iDMexchange, aniuni, Zeeman)
``set_field``          Zeeman applied field (setfield / equation)
``setode``             setode LLG RK4|RKDP54 (Boris/DiffEq_Common.cpp:79)
``setdt``              setdt (Boris/Commands.cpp:1914)
``astepctrl``          astepctrl (Boris/Commands.cpp:1931)
``update_field``       Module::UpdateField / MeshBase::UpdateModules (Heff)
``demag_field``        Demag::UpdateField (Boris/Demag.cpp:170)
``run``                AdvanceTime over ODECommon_Base::Iterate
``multiconvolution``   multiconvolution / 2dmulticonvolution / ncommon (SDemag multilayer)
=====================  ============================================================

Errors from the library raise :class:`BorisError` with the library's message, the
equivalent of the reference's BError return values. There is no CPU fallback: if the
CUDA library is missing or no GPU is present, loading or creating a context fails.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libboris_b200.so")

DEMAG, EXCH, IDMI, ANIUNI, ZEEMAN = 1, 2, 4, 8, 16
RK4, RKDP54 = 0, 1
FP64, MIXED = 0, 1
ML_OFF, ML_3D, ML_2D, ML_2D_LAYERED, ML_SUPERMESH = -1, 0, 1, 2, 3

_lib = None


class BorisError(RuntimeError):
    """A non-zero status from the C ABI; ``code`` is the status (BM_EINVAL ... BM_ENONFINITE)."""

    def __init__(self, msg, code=None):
        super().__init__(msg)
        self.code = code


OK, EINVAL, ECUDA, ENOMEM, ESTATE, EUNSUPPORTED, ENONFINITE = 0, 1, 2, 3, 4, 5, 6
PBC_MAX_IMAGES = 1000   # BM_PBC_MAX_IMAGES


class Stats(ctypes.Structure):
    _fields_ = [("accepted", ctypes.c_longlong), ("rejected", ctypes.c_longlong),
                ("attempts", ctypes.c_longlong), ("time", ctypes.c_double),
                ("dT", ctypes.c_double), ("last_lte", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_P = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int
_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)

_SIGS = {
    "bm_create": (_I, [_I, ctypes.POINTER(_P)]),
    "bm_destroy": (_I, [_P]),
    "bm_last_error": (ctypes.c_char_p, []),
    "bm_version": (_I, []),
    "bm_add_mesh": (_I, [_P, _I, _I, _I, _D, _D, _D, _D, _D, _D, _IP]),
    "bm_set_material": (_I, [_P, _I, _D, _D, _D, _D, _D, _D, _DP, _D]),
    "bm_set_material_maps": (_I, [_P, _I, _DP, _DP]),
    "bm_set_modules": (_I, [_P, _I, _I]),
    "bm_set_pbc": (_I, [_P, _I, _I, _I, _I]),
    "bm_get_pbc": (_I, [_P, _I, _IP]),
    "bm_set_field": (_I, [_P, _I, _DP, _I, _D]),
    "bm_set_ode": (_I, [_P, _I, _D]),
    "bm_set_astepctrl": (_I, [_P, _D, _D, _D, _D]),
    "bm_set_precision": (_I, [_P, _I]),
    "bm_set_m": (_I, [_P, _I, _DP]),
    "bm_get_m": (_I, [_P, _I, _DP]),
    "bm_compute_hdemag": (_I, [_P, _I, _DP, _DP]),
    "bm_compute_heff": (_I, [_P, _I, _DP]),
    "bm_run": (_I, [_P, _I, ctypes.POINTER(Stats)]),
    "bm_get_stats": (_I, [_P, ctypes.POINTER(Stats)]),
    "bm_get_mxh": (_I, [_P, _DP]),
    "bm_get_dmdt": (_I, [_P, _DP]),
    "bm_mesh_info": (_I, [_P, _I, _IP, _IP]),
    "bm_device_m": (_I, [_P, _I, ctypes.POINTER(_P), _IP]),
    "bm_sync": (_I, [_P]),
    "bm_kernels_per_step": (_I, [_P, _IP]),
    "bm_run_timed": (_I, [_P, _I, ctypes.POINTER(Stats), _DP]),
    "bm_time_kernels": (_I, [_P, _I, _I, _DP, _DP]),
    "bm_time_step": (_I, [_P, _I, _DP, _DP, _IP]),
    "bm_time_demag": (_I, [_P, _I, _I, _DP]),
    "bm_demag_field_device": (_I, [_P, _I, _P, _P, _I, _I, _DP, _P]),
    "bm_set_m_device": (_I, [_P, _I, _P, _I, _P]),
    "bm_get_m_device": (_I, [_P, _I, _P, _I, _P]),
    "bm_tiles": (_I, [_P, _I, _IP]),
    "bm_debug_kernels": (_I, [_P, _I, _DP]),
    "bm_debug_tensor": (_I, [_I, _I, _I, _I, _D, _D, _D, _DP]),
    "bm_debug_tensor_pbc": (_I, [_I, _I, _I, _I, _D, _D, _D, _IP, _DP]),
    "bm_debug_fft": (_I, [_I, _I, _I, _I, _I, _DP]),
    "bm_fft_noalloc": (_I, [_I, _I, _I, _I, _P, _P, _P]),
    "bm_set_multiconvolution": (_I, [_P, _I, _IP]),
    "bm_set_supermesh_cellsize": (_I, [_P, _D, _D, _D]),
    "bm_set_supermesh_pbc": (_I, [_P, _I, _I, _I]),
    "bm_supermesh_info": (_I, [_P, _IP, _DP, _DP, ctypes.POINTER(ctypes.c_longlong)]),
    "bm_ml_info": (_I, [_P, _IP, _IP, _IP, _IP, _DP, _IP]),
    "bm_prepare": (_I, [_P]),
    "bm_ml_time_kernels": (_I, [_P, _I, _DP, _DP]),
    "bm_ml_tile": (_I, [_P, _IP]),
    "bm_set_batched": (_I, [_P, _I]),
    "bm_set_memory_limit": (_I, [_P, ctypes.c_longlong]),
    "bm_adjoint_rk4": (_I, [_P, _I, _I, _DP, _I, _DP, _DP, _DP, _DP, _DP]),
    "bm_set_evalspeedup": (_I, [_P, _I]),
    "bm_self_demag": (_I, [_D, _D, _D, _DP]),
    "bm_self_demag_metres": (_I, [_D, _D, _D, _DP]),
    "bm_set_evalspeedup_self": (_I, [_P, _I]),
    "bm_ovf2_read": (_I, [ctypes.c_char_p, _IP, _DP, _DP, _DP, ctypes.c_longlong]),
    "bm_ovf2_write": (_I, [ctypes.c_char_p, _IP, _DP, _DP, _DP, ctypes.c_char_p, _D]),
    "bm_map_cells": (_I, [_DP, _IP, _DP, _IP]),
    "bm_renormalize": (_I, [_DP, ctypes.c_longlong, _D]),
    "bm_load_ovf2_mag": (_I, [_P, _I, ctypes.c_char_p, _D]),
    "bm_save_ovf2_mag": (_I, [_P, _I, ctypes.c_char_p, ctypes.c_char_p, _I]),
}


def lib():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise BorisError("libboris_b200.so not built (run boris2_b200/build.py): %s" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise BorisError("boris_b200 error %d: %s" % (rc, lib().bm_last_error().decode()), rc)


def _dp(a):
    return a.ctypes.data_as(_DP)


def _vec(a, n):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))
    if a.size != 3 * n:
        raise ValueError("expected %d values (3 per cell), got %d" % (3 * n, a.size))
    return a


def self_demag(h, metres=False):
    """Self-demagnetising coefficients -N of a cell of size h (host only); metres: as the reference's
    evaluation speedup computes them on the cellsize in metres."""
    out = np.empty(3)
    f = lib().bm_self_demag_metres if metres else lib().bm_self_demag
    _check(f(float(h[0]), float(h[1]), float(h[2]), _dp(out)))
    return out


def ovf2_read(path):
    """Read an OOMMF OVF 2.0 vector file (host only): dict with n (nodes), h (cellsize, m),
    rect (xmin, ymin, zmin, xmax, ymax, zmax, m) and data ((n cells, 3), x fastest)."""
    n3 = (ctypes.c_int * 3)()
    h3 = np.empty(3)
    r6 = np.empty(6)
    p = os.fsencode(path)
    _check(lib().bm_ovf2_read(p, n3, _dp(h3), _dp(r6), None, 0))
    n = tuple(n3)
    data = np.empty(3 * n[0] * n[1] * n[2])
    _check(lib().bm_ovf2_read(p, None, None, None, _dp(data), data.size))
    return {"n": n, "h": tuple(h3), "rect": tuple(r6), "data": data.reshape(-1, 3)}


def ovf2_write(path, data, n, h, origin=(0.0, 0.0, 0.0), data_type="bin8", norm=1.0):
    """Write an OOMMF OVF 2.0 vector file (host only); data_type "bin4", "bin8" or "text",
    every value divided by norm."""
    n3 = (ctypes.c_int * 3)(*[int(v) for v in n])
    a = _vec(data, int(n[0]) * int(n[1]) * int(n[2]))
    h3 = np.asarray(h, dtype=np.float64)
    o3 = np.asarray(origin, dtype=np.float64)
    _check(lib().bm_ovf2_write(os.fsencode(path), n3, _dp(h3), _dp(o3), _dp(a), data_type.encode(), float(norm)))


def map_cells(data, src_n, dst_n):
    """Nearest-cell remap of (cells, 3) vectors from src_n to dst_n cells (host only)."""
    a = _vec(data, int(np.prod(src_n)))
    out = np.empty(3 * int(np.prod(dst_n)))
    _check(lib().bm_map_cells(_dp(a), (ctypes.c_int * 3)(*src_n), _dp(out), (ctypes.c_int * 3)(*dst_n)))
    return out.reshape(-1, 3)


def renormalize(data, length):
    """Scale every vector longer than 1e-12 to `length` (host only); returns a new array."""
    a = np.array(np.asarray(data, dtype=np.float64).reshape(-1), copy=True)
    _check(lib().bm_renormalize(_dp(a), a.size // 3, float(length)))
    return a.reshape(-1, 3)


class Context:
    """One simulation on one GPU (SuperMesh + ODE solver of the reference)."""

    def __init__(self, device=0, precision=MIXED):
        self._h = _P()
        _check(lib().bm_create(int(device), ctypes.byref(self._h)))
        self.meshes = []
        self._nHa = 1
        _check(lib().bm_set_precision(self._h, int(precision)))

    def close(self):
        if self._h:
            lib().bm_destroy(self._h)
            self._h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------------ meshes
    def add_mesh(self, n, h, origin=(0.0, 0.0, 0.0)):
        mid = _I()
        _check(lib().bm_add_mesh(self._h, int(n[0]), int(n[1]), int(n[2]), float(h[0]), float(h[1]),
                                 float(h[2]), float(origin[0]), float(origin[1]), float(origin[2]),
                                 ctypes.byref(mid)))
        self.meshes.append((tuple(int(v) for v in n), tuple(float(v) for v in h)))
        return mid.value

    def ncells(self, mesh=0):
        n = self.meshes[mesh][0]
        return n[0] * n[1] * n[2]

    def set_material(self, mesh=0, Ms=8e5, A=1.3e-11, alpha=0.5, grel=1.0, K1=0.0, K2=0.0,
                     ea=(0.0, 0.0, 1.0), D=0.0):
        e = np.asarray(ea, dtype=np.float64)
        _check(lib().bm_set_material(self._h, mesh, Ms, A, alpha, grel, K1, K2, _dp(e), D))

    def set_material_maps(self, mesh=0, Ms_map=None, K1_map=None):
        n = self.ncells(mesh)
        a = None if Ms_map is None else np.ascontiguousarray(np.asarray(Ms_map, dtype=np.float64).reshape(n))
        b = None if K1_map is None else np.ascontiguousarray(np.asarray(K1_map, dtype=np.float64).reshape(n))
        _check(lib().bm_set_material_maps(self._h, mesh, None if a is None else _dp(a), None if b is None else _dp(b)))

    def set_modules(self, mesh=0, modules=DEMAG | EXCH | ZEEMAN):
        _check(lib().bm_set_modules(self._h, mesh, int(modules)))

    def set_pbc(self, mesh=0, images=(0, 0, 0)):
        """Periodic boundary conditions: images per axis (0 = not periodic), as the reference's
        Demag::Set_PBC / "pbc" command."""
        x, y, z = (int(v) for v in images)
        _check(lib().bm_set_pbc(self._h, mesh, x, y, z))

    def get_pbc(self, mesh=0):
        out = (ctypes.c_int * 3)()
        _check(lib().bm_get_pbc(self._h, mesh, out))
        return tuple(out)

    def set_field(self, mesh=0, Ha=(0.0, 0.0, 0.0), t_span=0.0):
        a = np.ascontiguousarray(np.asarray(Ha, dtype=np.float64).reshape(-1, 3))
        _check(lib().bm_set_field(self._h, mesh, _dp(a), a.shape[0], float(t_span)))
        self._nHa = a.shape[0]

    def set_precision(self, precision):
        _check(lib().bm_set_precision(self._h, int(precision)))

    def adjoint_rk4(self, target, steps, ckpt_every=100, m0_scales_with_Ms=True, nHa=None):
        """Run `steps` RK4 steps from the current state and return (loss, dMs, dK1, dHa, times_ms):
        the loss (1/n) sum |m(T) - target|^2 and its exact gradients with respect to the per-cell Ms
        and K1 maps and the applied-field samples (reverse mode through every stage, checkpoints every
        ckpt_every steps). times_ms = (forward run, backward sweep) device time."""
        n = self.ncells(0)
        t = _vec(target, n)
        loss = ctypes.c_double(0.0)
        dMs = np.zeros(n)
        dK1 = np.zeros(n)
        k = self._nHa if nHa is None else int(nHa)
        dHa = np.zeros(3 * max(k, 1))
        tm = np.zeros(2)
        _check(lib().bm_adjoint_rk4(self._h, int(steps), int(ckpt_every), _dp(t), int(bool(m0_scales_with_Ms)),
                                    ctypes.byref(loss), _dp(dMs), _dp(dK1), _dp(dHa), _dp(tm)))
        return loss.value, dMs, dK1, dHa[:3 * k].reshape(-1, 3), tuple(tm)

    def set_memory_limit(self, nbytes):
        """Device bytes the context may use (0: the free device memory); set-up refuses with
        ENOMEM before allocating when its meshes need more."""
        _check(lib().bm_set_memory_limit(self._h, int(nbytes)))

    def set_batched(self, on=True):
        """Advance all meshes with one launch per pass over a (mesh, tile) work list."""
        _check(lib().bm_set_batched(self._h, int(bool(on))))

    def multiconvolution(self, mode=ML_3D, ncommon=None):
        """Multilayered demag over all meshes with the demag module (ML_OFF turns it off):
        ML_3D = ``multiconvolution 1``, ML_2D / ML_2D_LAYERED = ``2dmulticonvolution 1 / 2``;
        ncommon = ``ncommon nx ny nz`` (None: ``ncommonauto``)."""
        nc = None if ncommon is None else (ctypes.c_int * 3)(*[int(v) for v in ncommon])
        _check(lib().bm_set_multiconvolution(self._h, int(mode), nc))

    def ml_info(self):
        """Layers of the multilayered convolution: count, n_common, mesh and transfer flag per
        layer, rectangles (start, end) and kernel kinds per (layer, source)."""
        L = _I()
        nc = (ctypes.c_int * 3)()
        lm = (ctypes.c_int * 8)()
        tr = (ctypes.c_int * 8)()
        rc = np.zeros(48)
        kk = (ctypes.c_int * 64)()
        _check(lib().bm_ml_info(self._h, ctypes.byref(L), nc, lm, tr, _dp(rc), kk))
        n = L.value
        return {"L": n, "n_common": tuple(nc), "layer_mesh": list(lm)[:n], "transfer": list(tr)[:n],
                "rects": rc[:6 * n].reshape(n, 6).copy(), "kinds": np.array(list(kk)[:n * n]).reshape(n, n)}

    def supermesh_cellsize(self, h):
        """Requested supermesh cellsize (the reference's ``fmscellsize``; default 5 nm)."""
        _check(lib().bm_set_supermesh_cellsize(self._h, float(h[0]), float(h[1]), float(h[2])))

    def supermesh_pbc(self, images=(0, 0, 0)):
        """PBC images of the supermesh convolution, also every mesh's stencil PBC (SDemag::Set_PBC)."""
        x, y, z = (int(v) for v in images)
        _check(lib().bm_set_supermesh_pbc(self._h, x, y, z))

    def supermesh_info(self):
        n = (ctypes.c_int * 3)()
        h = np.zeros(3)
        r = np.zeros(6)
        ne = ctypes.c_longlong(0)
        _check(lib().bm_supermesh_info(self._h, n, _dp(h), _dp(r), ctypes.byref(ne)))
        return {"n": tuple(n), "h": tuple(h), "rect": r.reshape(2, 3).copy(), "nonempty": ne.value}

    def prepare(self):
        _check(lib().bm_prepare(self._h))

    def ml_tile(self):
        """Columns per block of the fused multilayer z pass."""
        w = _I()
        _check(lib().bm_ml_tile(self._h, ctypes.byref(w)))
        return w.value

    def ml_time_kernels(self, reps=10):
        """ms and algorithmic bytes of the parts of one multilayer demag evaluation: transfer
        in + x forward, y forward, z pass + products, y inverse, x inverse + transfer out, all."""
        ms = np.zeros(6)
        by = np.zeros(6)
        _check(lib().bm_ml_time_kernels(self._h, int(reps), _dp(ms), _dp(by)))
        return ms, by

    # ------------------------------------------------------------------ ODE
    def setode(self, evaluation="RK4", dt=None):
        ev = {"RK4": RK4, "RKDP54": RKDP54}[evaluation] if isinstance(evaluation, str) else int(evaluation)
        if dt is None:
            dt = 1e-13 if ev == RK4 else 0.5e-12   # Boris/DiffEq_Defs.h defaults
        self._eval = ev
        _check(lib().bm_set_ode(self._h, ev, float(dt)))

    def setdt(self, dt):
        _check(lib().bm_set_ode(self._h, getattr(self, "_eval", RK4), float(dt)))

    def evalspeedup(self, level):
        """The reference's evalspeedup: 0 off, 1 step .. 6 quintic extrapolation of the demag field
        between RK4 steps."""
        _check(lib().bm_set_evalspeedup(self._h, int(level)))

    def evalspeedup_self(self, metres):
        """The speedup's self term: False the cell's -N on normalised cellsizes (default), True as the
        reference computes it on cellsizes in metres."""
        _check(lib().bm_set_evalspeedup_self(self._h, int(bool(metres))))

    def astepctrl(self, err_fail, dT_incr, dT_min, dT_max):
        _check(lib().bm_set_astepctrl(self._h, float(err_fail), float(dT_incr), float(dT_min), float(dT_max)))

    # ------------------------------------------------------------------ state
    def set_m(self, M, mesh=0):
        a = _vec(M, self.ncells(mesh))
        _check(lib().bm_set_m(self._h, mesh, _dp(a)))

    def get_m(self, mesh=0, out=None):
        n = self.ncells(mesh)
        out = np.empty(3 * n) if out is None else out
        _check(lib().bm_get_m(self._h, mesh, _dp(out)))
        return out.reshape(n, 3)

    def loadovf2mag(self, path, mesh=0, renormalize=0.0):
        """The reference's loadovf2mag: M from an OVF 2.0 file, mapped to this mesh's cells and
        renormalised to `renormalize` when it is non-zero."""
        _check(lib().bm_load_ovf2_mag(self._h, mesh, os.fsencode(path), float(renormalize)))

    def saveovf2mag(self, path, mesh=0, data_type="bin8", normalize=False):
        """The reference's saveovf2mag: M to an OVF 2.0 file, divided by Ms when normalize."""
        _check(lib().bm_save_ovf2_mag(self._h, mesh, os.fsencode(path), data_type.encode(), int(bool(normalize))))

    def demag_field(self, mesh=0, with_energy=False):
        n = self.ncells(mesh)
        H = np.empty(3 * n)
        e = ctypes.c_double(0.0)
        _check(lib().bm_compute_hdemag(self._h, mesh, _dp(H), ctypes.byref(e)))
        return (H.reshape(n, 3), e.value) if with_energy else H.reshape(n, 3)

    def update_field(self, mesh=0):
        n = self.ncells(mesh)
        H = np.empty(3 * n)
        _check(lib().bm_compute_heff(self._h, mesh, _dp(H)))
        return H.reshape(n, 3)

    def run(self, steps):
        st = Stats()
        _check(lib().bm_run(self._h, int(steps), ctypes.byref(st)))
        return st.as_dict()

    def run_timed(self, steps):
        """Run and return (stats, device milliseconds measured on the library's stream)."""
        st = Stats()
        ms = ctypes.c_double(0.0)
        _check(lib().bm_run_timed(self._h, int(steps), ctypes.byref(st), ctypes.byref(ms)))
        return st.as_dict(), ms.value

    def time_kernels(self, mesh=0, reps=20):
        """Average ms per launch and algorithmic bytes of each kernel of one field evaluation:
        [y pass / ymid2d, zmid, yinv, stage]."""
        ms = np.zeros(4)
        by = np.zeros(4)
        _check(lib().bm_time_kernels(self._h, mesh, int(reps), _dp(ms), _dp(by)))
        return ms, by

    def time_demag(self, mesh=0, reps=20):
        """Device ms of one demag field evaluation (x transform, y / z passes, inverse x into H)."""
        ms = ctypes.c_double(0.0)
        _check(lib().bm_time_demag(self._h, mesh, int(reps), ctypes.byref(ms)))
        return ms.value

    TIME_KINDS = ("stage", "yfwd", "zmid", "yinv", "ymid2d", "other", "yzy", "")

    def time_step(self, steps=3):
        """Run `steps` steps eagerly (the step graph's launches, timed one by one with CUDA events)
        and return {kind: {"ms": summed device ms, "bytes": summed algorithmic bytes, "launches": n}}
        for the kinds in TIME_KINDS that launched. The simulation advances."""
        ms = np.zeros(8)
        by = np.zeros(8)
        nl = (ctypes.c_int * 8)()
        _check(lib().bm_time_step(self._h, int(steps), _dp(ms), _dp(by), nl))
        return {k: {"ms": float(ms[i]), "bytes": float(by[i]), "launches": int(nl[i])}
                for i, k in enumerate(self.TIME_KINDS) if nl[i] > 0}

    def tiles(self, mesh=0):
        """Autotuned tile shapes: 2D y width, 3D y width and variant (1: radix-16 Stockham, 2: two-level
        register transform fed by pipelined bulk tensor copies), z width,
        stage rows per block (negative when the per-cell rows are prefetched), stage x-transform
        variant (1: radix-8 Stockham, 2: radix-16 Stockham, 3: radix 16 at the lower FP32 register
        cap), yzy (1: the fused y -> z -> y cluster pass of a 3D mesh), z-pass variant (1: the parity
        split, two threads per pencil line)."""
        t = (ctypes.c_int * 4)()
        _check(lib().bm_tiles(self._h, mesh, t))
        sgn = -1 if t[3] < 0 else 1
        return {"ymid2d_W": t[0], "ypass_W": t[1] % 100, "ypass_yv": t[1] // 100, "zmid_W": t[2] % 1000,
                "yzy": (t[2] // 1000) % 10, "zmid_zv": t[2] // 10000, "stage_rows": sgn * (abs(t[3]) % 100),
                "stage_xv": abs(t[3]) // 100}

    def stats(self):
        st = Stats()
        _check(lib().bm_get_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def get_mxh(self):
        """The reference's Get_mxh: max over cells of |M x Heff| / |M|^2 at the first evaluation of the
        last step that computed it (0 before any); the call asks the next step to compute it."""
        v = ctypes.c_double()
        _check(lib().bm_get_mxh(self._h, ctypes.byref(v)))
        return v.value

    def get_dmdt(self):
        """The reference's Get_dmdt: max over cells of |M - M_step_start| / (dT GAMMA |M|^2) after the
        last stage of the last step that computed it (0 before any); the call asks the next step."""
        v = ctypes.c_double()
        _check(lib().bm_get_dmdt(self._h, ctypes.byref(v)))
        return v.value

    def fft_sizes(self, mesh=0):
        n3 = (ctypes.c_int * 3)()
        N3 = (ctypes.c_int * 3)()
        _check(lib().bm_mesh_info(self._h, mesh, n3, N3))
        return tuple(N3)

    def device_m(self, mesh=0):
        p = _P()
        eb = _I()
        _check(lib().bm_device_m(self._h, mesh, ctypes.byref(p), ctypes.byref(eb)))
        return p.value, eb.value

    def sync(self):
        _check(lib().bm_sync(self._h))

    def kernels_per_step(self):
        c = _I()
        _check(lib().bm_kernels_per_step(self._h, ctypes.byref(c)))
        return c.value

    def debug_kernels(self, mesh=0):
        N = self.fft_sizes(mesh)
        nk = (N[0] // 2 + 1) * (N[1] // 2 + 1) * (N[2] // 2 + 1)
        K = np.empty(6 * nk)
        _check(lib().bm_debug_kernels(self._h, mesh, _dp(K)))
        return K.reshape(6, N[2] // 2 + 1, N[1] // 2 + 1, N[0] // 2 + 1)


def debug_tensor(n, h, device=0, pbc=None):
    oct6 = np.empty(6 * n[0] * n[1] * n[2])
    if pbc is None:
        _check(lib().bm_debug_tensor(device, int(n[0]), int(n[1]), int(n[2]), float(h[0]), float(h[1]), float(h[2]),
                                     _dp(oct6)))
    else:
        p3 = (ctypes.c_int * 3)(*(int(v) for v in pbc))
        _check(lib().bm_debug_tensor_pbc(device, int(n[0]), int(n[1]), int(n[2]), float(h[0]), float(h[1]), float(h[2]),
                                         p3, _dp(oct6)))
    return oct6.reshape(n[2], n[1], n[0], 6)


def debug_fft(x, precision=FP64, inverse=False, device=0):
    """Batched 1D complex FFT along the last axis on the GPU (unnormalised)."""
    x = np.asarray(x, dtype=np.complex128)
    L = x.shape[-1]
    flat = np.array(x.reshape(-1, L), dtype=np.complex128, copy=True)
    buf = np.ascontiguousarray(flat.view(np.float64).reshape(-1))
    _check(lib().bm_debug_fft(device, L, flat.shape[0], int(precision), int(bool(inverse)), _dp(buf)))
    return buf.view(np.complex128).reshape(x.shape)
