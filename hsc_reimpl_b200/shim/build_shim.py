"""Compile the LinearHSC shim test driver against the libuipc mock and libhsc_b200.so."""
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
OUT = HERE / "_build" / "shim_driver"


def build():
    OUT.parent.mkdir(exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wno-unused-function",
           f"-I{HERE / 'uipc_mock'}", f"-I{HERE}", f"-I{ROOT / 'include'}", "-I/usr/local/cuda/include",
           str(HERE / "shim_driver.cpp"), "-o", str(OUT),
           f"-L{ROOT / 'hsc_reimpl_b200'}", "-lhsc_b200", f"-Wl,-rpath,{ROOT / 'hsc_reimpl_b200'}",
           "-L/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath,/usr/local/cuda/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr)
    return OUT


if __name__ == "__main__":
    print(build())
