"""Build recipe of the CUDA library (libdmfted.so) for sm_100a.

The library is built in-tree next to this file so the shared object travels
with the repository.  Usage: python dmft-ed_b200/build.py [--force]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libdmfted.so")
SOURCES = ["api.cu", "fock.cu", "hxv.cu", "lanczos.cu", "gf.cu", "observables.cu", "chi2.cu",
           "batch.cu", "noalloc.cu", "dense.cu", "diag.cu", "fit.cu",
           "restart.cu", "edio.cu"]
HEADERS = ["internal.cuh", "reduce.cuh", "hxv.cuh", "tridiag.cuh", "sector.cuh", "jterms.cuh",
           "fortfmt.h"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-O3",
    "--expt-relaxed-constexpr",
    "-rdc=false",
]


def _stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "dmfted.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, checked=False):
    """Compile every .cu file to an object and link libdmfted.so.  checked=True
    adds the device-side index checks (-DDMFTED_DEVICE_CHECKS)."""
    if not force and not checked and not _stale():
        return OUT
    nvcc = os.environ.get("NVCC", "nvcc")
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs, cmds = [], []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        extra = ["-DDMFTED_DEVICE_CHECKS"] if checked else []
        cmd = [nvcc, *NVCC_FLAGS, *extra, "-I", os.path.join(ROOT, "include"), "-c",
               os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        cmds.append(cmd)
        objs.append(obj)
    # one nvcc per source file, in parallel (the files are independent)
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for r in list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds)):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise subprocess.CalledProcessError(r.returncode, r.args)
    cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", OUT, *objs]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv or "--checked" in sys.argv, verbose="-v" in sys.argv,
          checked="--checked" in sys.argv)
    print(OUT)
