"""CPU checks of the C ABI library: it builds, loads, exports every declared symbol, and
fails loudly (error status, no crash, no CPU fallback) when no GPU is present."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "boris_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char|void)\s*\**\s*(bm_\w+)\s*\(", src, flags=re.M)))


def test_header_parses():
    syms = declared_symbols()
    assert "bm_create" in syms and "bm_run" in syms and "bm_compute_hdemag" in syms
    assert len(syms) >= 25


def test_library_exports_all_symbols():
    import boris2_b200
    from boris2_b200 import build
    build.build()
    L = ctypes.CDLL(boris2_b200.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_wrapper_covers_header():
    import boris2_b200
    assert set(declared_symbols()) <= set(boris2_b200._SIGS)


def test_no_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    import boris2_b200
    with pytest.raises(boris2_b200.BorisError):
        boris2_b200.Context()


def test_plan_sizes():
    """The FFT planner accepts 2^p and 3*2^p and rejects other lengths (host logic)."""
    import subprocess
    import tempfile
    src = r'''
#include "fft.cuh"
#include <cstdio>
int main(){ int ok=1; FFTPlan P;
  for (int L=1; L<=4096; L++) { bool nice=false; for(int p=1;p<=4096;p*=2){ if(p==L||3*p==L) nice=true; }
    bool r = bm_make_plan(L,P); if (r!=nice) { printf("L=%d\n",L); ok=0; }
    if (r) { int prod=1; for(int i=0;i<P.np;i++) prod*=P.radix[i]; if(prod!=L) ok=0;
      for(int i=0;i+1<P.np;i++) if (P.radix[i] < P.radix[i+1] && P.radix[i+1]!=3) ok=0; } }
  printf(ok?"OK\n":"FAIL\n"); return !ok; }
'''
    with tempfile.TemporaryDirectory() as d:
        f = os.path.join(d, "t.cpp")
        open(f, "w").write(src)
        exe = os.path.join(d, "t")
        r = subprocess.run(["g++", "-std=c++17", "-x", "c++", "-D__host__=", "-D__device__=", "-D__forceinline__=inline",
                            "-I", os.path.join(ROOT, "boris2_b200", "csrc"), "-I/usr/local/cuda/include", f, "-o", exe],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        out = subprocess.run([exe], capture_output=True, text=True)
        assert out.returncode == 0 and "OK" in out.stdout, out.stdout
