"""In-tree build of the native libraries (no JIT cache: the .so files live next
to this file so they travel with the repository snapshot).

* ``lib/libnlnhost.so``  host tree / moments / MAC walk / list packing (g++, OpenMP)
* ``lib/libgravcuda.so`` the gravcuda.h C ABI and its sm_100a kernels (nvcc)
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)                 # the ahotsph-2hot-apps_b200 directory
REPO = os.path.dirname(ROOT)
CSRC = os.path.join(ROOT, "csrc")
INCLUDE = os.path.join(REPO, "include")
LIBDIR = os.path.join(PKG, "lib")
HOST_SO = os.path.join(LIBDIR, "libnlnhost.so")
CUDA_SO = os.path.join(LIBDIR, "libgravcuda.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _cxx():
    # the image exports CXX=/opt/gcc/bin/g++, a wrapper without OpenMP
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _run(cmd):
    print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)


def host_sources():
    d = os.path.join(CSRC, "host")
    return sorted(os.path.join(d, f) for f in os.listdir(d) if f.endswith(".cpp"))


def cuda_sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def cuda_headers():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h")))


def build_host(force=False):
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = host_sources()
    deps = srcs + [os.path.join(INCLUDE, "nlnhost.h"), os.path.join(CSRC, "host", "tree_math.h")]
    if force or _newer(HOST_SO, deps):
        # no contraction into FMAs: the tree arithmetic (csrc/host/tree_math.h) must round
        # exactly as the GPU builder's does
        _run([_cxx(), "-O3", "-mavx2", "-mfma", "-ffp-contract=off", "-fPIC", "-fopenmp",
              "-std=c++17", "-shared", "-I", INCLUDE, "-o", HOST_SO] + srcs)
    return HOST_SO


# Sources compiled on their own with these extra flags: the GPU tree builder
# must not contract a * b + c into fused multiply-adds, so that its
# arithmetic rounds exactly as the host builder's (csrc/host/tree_math.h).
SEPARATE = {"build.cu": ["-fmad=false"]}


def build_cuda(force=False, verbose_ptxas=False):
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = cuda_sources()
    deps = srcs + cuda_headers() + [os.path.join(CSRC, "host", f)
                                    for f in os.listdir(os.path.join(CSRC, "host"))] + \
        [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    if force or _newer(CUDA_SO, deps):
        base = [_nvcc()] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler",
                                   "-fPIC,-fopenmp", "-ccbin", _cxx(), "-I", INCLUDE, "-I", CSRC]
        if verbose_ptxas:
            base += ["-Xptxas", "-v"]
        objs = []
        for src in srcs:
            flags = SEPARATE.get(os.path.basename(src))
            if flags is None:
                continue
            obj = os.path.join(LIBDIR, os.path.basename(src) + ".o")
            _run(base + flags + ["-c", "-o", obj, src])
            objs.append(obj)
        rest = [x for x in srcs if os.path.basename(x) not in SEPARATE]
        _run(base + ["-shared", "-o", CUDA_SO] + rest + objs + ["-lcudart", "-lgomp"])
    return CUDA_SO


DRIVE_SO = os.path.join(LIBDIR, "libmacdrive.so")


def build_drive(force=False):
    """lib/libmacdrive.so: a C caller of the drop-in ABI as nln/mac.c drives it
    (timing without an interpreter in the loop), linked to libgravcuda.so."""
    cuda = build_cuda(force)
    src = os.path.join(CSRC, "drive", "mac_drive.c")
    if force or _newer(DRIVE_SO, [src, cuda, os.path.join(INCLUDE, "gravcuda.h")]):
        cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
        _run([cc, "-O2", "-fPIC", "-shared", "-std=gnu99", "-I", INCLUDE, "-o", DRIVE_SO, src,
              "-L", LIBDIR, "-lgravcuda", "-Wl,-rpath,$ORIGIN"])
    return DRIVE_SO


def build_all(force=False):
    build_host(force)
    build_cuda(force)
    build_drive(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
