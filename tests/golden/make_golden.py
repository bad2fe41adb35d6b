"""Generate tests/golden/reference_golden.npz from the reference's own compiled CPU code
(oracle/_ref/libborisref.so, built by oracle/Makefile from the reference tree).

The reference ships no golden vectors (it has no test suite), so these fixtures are
outputs of its Convolution<., DemagKernel>, DemagKernel::Calculate_Demag_Kernels and
DemagTFunc::SelfDemag on small seeded inputs. Run from the repository root:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from oracle_libs import reference, dp, sphere_random  # noqa: E402


def main():
    R = reference()
    if R is None:
        raise SystemExit("reference build unavailable")
    out = {}
    cases = {"film2d": ((16, 8, 1), (5e-9, 5e-9, 3e-9)), "box3d": ((10, 6, 4), (2e-9, 2e-9, 2e-9)),
             "odd3d": ((5, 3, 3), (2e-9, 3e-9, 1e-9))}
    for tag, (n, h) in cases.items():
        N = n[0] * n[1] * n[2]
        M = sphere_random(N, seed=4321 + N, Ms=8e5)
        H = np.zeros(3 * N)
        e = np.zeros(1)
        Mf = np.ascontiguousarray(M.reshape(-1))
        assert R.ref_hdemag(n[0], n[1], n[2], h[0], h[1], h[2], dp(Mf), dp(H), dp(e)) == 0
        out["M_" + tag] = M
        out["hdemag_" + tag] = H.reshape(-1, 3)
        out["edemag_" + tag] = e
        out["n_" + tag] = np.array(n)
        out["h_" + tag] = np.array(h)
    kcases = {"k2d": ((8, 6, 1), (5, 5, 3)), "k3d": ((6, 5, 4), (2, 2, 2)), "kfar": ((50, 45, 1), (4, 4, 3))}
    for tag, (n, h) in kcases.items():
        Nf = (2 * n[0], 2 * n[1], 2 * n[2] if n[2] > 1 else 1)
        nk = (Nf[0] // 2 + 1) * (Nf[1] // 2 + 1) * (Nf[2] // 2 + 1)
        kd = np.zeros(3 * nk)
        ko = np.zeros(3 * nk if n[2] > 1 else nk)
        assert R.ref_kernels(n[0], n[1], n[2], h[0], h[1], h[2], dp(kd), dp(ko)) == 0
        out["kdiag_" + tag] = kd
        out["kodiag_" + tag] = ko
        out["kn_" + tag] = np.array(n)
        out["kh_" + tag] = np.array(h, dtype=float)
    rows = []
    for h in [(5, 5, 3), (2, 2, 2), (1, 2, 3.5), (4, 4, 1)]:
        o = np.zeros(3)
        R.ref_selfdemag(h[0], h[1], h[2], dp(o))
        rows.append(list(h) + list(o))
    out["selfdemag"] = np.array(rows)
    path = os.path.join(HERE, "reference_golden.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
