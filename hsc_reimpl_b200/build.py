"""Build the in-tree CUDA library ``libhsc_b200.so`` for sm_100a with nvcc.

    python -m hsc_reimpl_b200.build        # or hsc_reimpl_b200.build.build()

Each .cu under csrc/ is compiled to an object with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and linked into one
shared library (static CUDA runtime; the host pattern analysis uses OpenMP).  Objects go to
csrc/_build/.
"""
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = CSRC / "_build"
LIB = HERE / "libhsc_b200.so"
SOURCES = ["hsc_api.cu", "hsc_setup.cu", "hsc_pcg.cu", "hsc_aca.cu", "hsc_learned.cu", "hsc_assemble.cu", "hsc_coupling.cu",
           "hsc_noalloc.cu", "hsc_partition.cpp", "hsc_block.cu",
           "hsc_aca_comp.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "-Xcompiler", "-fopenmp", "--expt-relaxed-constexpr",
         f"-I{HERE.parent / 'include'}"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def build(force=False, verbose=False, checked=False):
    """Build libhsc_b200.so; ``checked=True`` builds libhsc_b200_checked.so with
    the index guards of hsc_check.cuh compiled in."""
    build_dir = BUILD / "checked" if checked else BUILD
    lib = HERE / ("libhsc_b200_checked.so" if checked else "libhsc_b200.so")
    extra = ["-DHSC_CHECKED"] if checked else []
    build_dir.mkdir(parents=True, exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [HERE.parent / "include" / "hsc_c_api.h"]
    newest_header = max(h.stat().st_mtime for h in headers)
    objs, jobs = [], []
    for src in SOURCES:
        s = CSRC / src
        o = build_dir / (s.stem + ".o")
        if force or not o.exists() or o.stat().st_mtime < max(s.stat().st_mtime, newest_header):
            cmd = [NVCC, *FLAGS, *extra, "-c", str(s), "-o", str(o)]
            if verbose:
                print(" ".join(cmd))
            jobs.append(cmd)
        objs.append(str(o))
    # the translation units are independent: compile them in parallel
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        for f in [pool.submit(_run, cmd) for cmd in jobs]:
            f.result()
    if force or not lib.exists() or lib.stat().st_mtime < max(Path(o).stat().st_mtime for o in objs):
        _run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-cudart", "static",
              "-o", str(lib), *objs, "-lpthread", "-lgomp"])
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, checked="--checked" in sys.argv))
