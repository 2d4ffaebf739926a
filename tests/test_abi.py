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


def _compile_with_reference_header(tmp_path, our_header_text, first="ours"):
    """Compile one C unit that declares every entry point twice: from
    include/gravcuda.h and from the reference's nln/gravcuda.h with CUDA
    defined (the prototypes nln/mac.c is built against).  A conflicting
    prototype is a compile error.  Returns the compiler's result."""
    import subprocess
    from oracle import oracle as O
    inc = tmp_path / "inc"
    inc.mkdir(exist_ok=True)
    for name in os.listdir(os.path.join(REPO, "include")):
        if name.endswith(".h") and name != "gravcuda.h":
            (inc / name).write_text(open(os.path.join(REPO, "include", name)).read())
    (inc / "gravcuda.h").write_text(our_header_text)
    ours = '#include "gravcuda.h"\n'
    theirs = f'#define CUDA 1\n#include "{O.REF_NLN}/gravcuda.h"\n'
    src = tmp_path / "both.c"
    src.write_text("#include <stdint.h>\n"
                   f'#include "{O.REF_NLN}/segment.h"\n'
                   "#define SEGMENT_DEFINED 1\n" +
                   (ours + theirs if first == "ours" else theirs + ours) +
                   "int main(void) { return 0; }\n")
    return subprocess.run(["gcc", "-std=gnu99", "-Werror", "-fsyntax-only", "-I", str(inc),
                           str(src)], capture_output=True, text=True)


def _reference_header_present():
    from oracle import oracle as O
    return os.path.exists(os.path.join(O.REF_NLN, "gravcuda.h"))


@pytest.mark.skipif(not _reference_header_present(), reason="reference tree absent")
@pytest.mark.parametrize("first", ["ours", "reference"])
def test_prototypes_agree_with_reference_header(tmp_path, first):
    """Signatures, not just names: every Part 1 prototype of include/gravcuda.h
    must be compatible with nln/gravcuda.h:13-69 (both orders of inclusion)."""
    text = open(os.path.join(REPO, "include", "gravcuda.h")).read()
    r = _compile_with_reference_header(tmp_path, text, first)
    assert r.returncode == 0, r.stderr


@pytest.mark.skipif(not _reference_header_present(), reason="reference tree absent")
def test_prototype_drift_is_caught(tmp_path):
    """The check above fails on a drifted signature (planted in a temporary
    copy of the header, never in the product)."""
    text = open(os.path.join(REPO, "include", "gravcuda.h")).read()
    drifted = text.replace("const int source_n, const int sz, const float e, int *ncut,",
                           "const int source_n, const int sz, const double e, int *ncut,", 1)
    assert drifted != text
    r = _compile_with_reference_header(tmp_path, drifted)
    assert r.returncode != 0 and "grav_mn_CUDA" in r.stderr
