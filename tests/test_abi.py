"""The C-ABI libraries load and export every symbol their headers declare
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

from conftest import REPO


def declared(header):
    src = open(os.path.join(REPO, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(\w+)\s*\(", src, flags=re.M)
    return sorted({n for n in names if n not in ("if", "while", "for", "return", "sizeof")})


def exported(path):
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_gravcuda_exports_every_declared_symbol():
    from pgrav import _build, gravcuda
    path = _build.build_cuda()
    names = declared("gravcuda.h")
    assert "grav_mn_CUDA" in names and "WalkInitSinkCUDA" in names
    missing = [n for n in names if n not in exported(path)]
    assert not missing, missing
    assert sorted(gravcuda.EXPORTS) == names
    ctypes.CDLL(path)  # loads without a GPU


def test_nlnhost_exports_every_declared_symbol():
    from pgrav import _build
    path = _build.build_host()
    names = declared("nlnhost.h")
    missing = [n for n in names if n not in exported(path)]
    assert not missing, missing


def test_reference_names_kept():
    """Every entry point of the reference nln/gravcuda.h:13-69 is declared."""
    ref = ["CUDA_Init", "CUDA_Finalize", "vecwidthCUDA", "qallocCUDA", "WalkInitSrcCUDA",
           "WalkTerminateSrcCUDA", "WalkInitSinkCUDA", "WalkTerminateSinkCUDA", "grav_mn_CUDA",
           "grav_mns_CUDA", "grav_mnss_CUDA", "grav_qns_CUDA", "grav_qnss_CUDA"]
    names = declared("gravcuda.h")
    assert all(r in names for r in ref)
