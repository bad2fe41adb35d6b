"""Generate tests/golden/ovf2_vortex.json from the OVF 2.0 files the reference ships
(Boris/vortex_hh_*.ovf, written by the reference's own OVF2::Write_OVF2_VEC), read with the
reference's own reader (OVF2::Read_OVF2_VEC, compiled into oracle/_ref/libborisref.so).

For each file: the SHA-256 of the whole file, the header the reference reads (nodes, cellsize,
rectangle) and the SHA-256 and component sums of the values it reads. The files themselves are
not copied. Run from the repository root:
    python tests/golden/make_ovf2_golden.py
"""
import ctypes
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from oracle_libs import reference, dp, ip, REF_TREE  # noqa: E402

FILES = ["vortex_hh_clk_up.ovf", "vortex_hh_clk_dn.ovf", "vortex_hh_cclk_up.ovf", "vortex_hh_cclk_dn.ovf"]


def main():
    R = reference()
    if R is None or not os.path.isdir(REF_TREE):
        raise SystemExit("reference tree and build unavailable")
    out = {}
    for f in FILES:
        path = os.path.join(REF_TREE, "Boris", f)
        raw = open(path, "rb").read()
        n3 = np.zeros(3, dtype=np.int32)
        h3 = np.zeros(3)
        r6 = np.zeros(6)
        assert R.ref_ovf2_read(path.encode(), ip(n3), dp(h3), dp(r6), None) == 0
        data = np.zeros(3 * int(np.prod(n3)))
        assert R.ref_ovf2_read(path.encode(), ip(n3), dp(h3), dp(r6), dp(data)) == 0
        out[f] = {"file_sha256": hashlib.sha256(raw).hexdigest(), "file_bytes": len(raw),
                  "n": [int(v) for v in n3], "h": [float(v) for v in h3], "rect": [float(v) for v in r6],
                  "data_sha256": hashlib.sha256(data.astype("<f8").tobytes()).hexdigest(),
                  "sums": [float(v) for v in data.reshape(-1, 3).sum(axis=0)]}
    with open(os.path.join(HERE, "ovf2_vortex.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", os.path.join(HERE, "ovf2_vortex.json"))


if __name__ == "__main__":
    main()
