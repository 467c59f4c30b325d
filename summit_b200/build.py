"""Build liblds.so in-tree for sm_100a (``python -m summit_b200.build``)."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT = PKG / "liblds.so"
# The bounds-checked build (-DLDS_CHECKED): the tensor-core kernels check
# their tile, bin, sketch-column, member-row and output indices, record the
# first failure in a device error word (lds_checked_errors) and skip the
# access instead of trapping.  Loaded instead of liblds.so when the
# environment sets SUMMIT_B200_CHECKED=1.
OUT_CHECKED = PKG / "liblds_checked.so"
SOURCES = ["lds_kernels.cu", "lds_umma.cu", "lds_umma_p1.cu", "lds_band.cu", "lds_gram.cu", "lds_gxe.cu", "lds_proj.cu", "lds_jack.cu", "lds_dense.cu", "lds_probes.cu", "lds_cv.cu", "lds_mlp.cu", "lds_check.cu", "lds_generalized.cu", "lds_host.cu",
           "lds_noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def build(force: bool = False, verbose: bool = False, checked: bool = False) -> Path:
    out = OUT_CHECKED if checked else OUT
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [
        PKG.parent / "include" / "lds.h"]
    if out.exists() and not force:
        newest = max(p.stat().st_mtime for p in deps if p.exists())
        if out.stat().st_mtime >= newest:
            return out
    cmd = [nvcc(), *ARCH, "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "-shared", "-cudart", "static",
           *(["-DLDS_CHECKED"] if checked else []),
           *[str(CSRC / s) for s in SOURCES], "-o", str(out)]
    if verbose:
        print(" ".join(cmd))
    tmp_out = out.with_suffix(".so.tmp")
    cmd[-1] = str(tmp_out)
    subprocess.run(cmd, check=True)
    os.replace(tmp_out, out)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, checked="--checked" in sys.argv))
