"""Build the in-tree CUDA library ``ramses_b200/lib/libramses_b200.so`` for
sm_100a with nvcc (no JIT cache: the .so travels with the source tree).

The FP64 units are compiled with ``--fmad=false`` so that no multiply-add is
contracted (bit-identical to the reference operation order); the FP32-mixed
unit uses fast FP32 division/sqrt and contraction.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libramses_b200.so"
OBJDIR = PKG / "_build"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "-I", str(PKG.parent / "include")]
UNITS = {
    "rb_runtime.cu": ["--fmad=false"],
    "tile_f64.cu": ["--fmad=false"],
    "tile_mixed.cu": ["-use_fast_math"],
    "rb_noalloc.cu": ["--fmad=false"],
    "rb_server.cu": ["--fmad=false"],
}
HEADERS = sorted(list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(CSRC.glob("*.inc"))
                 + [PKG.parent / "include" / "ramses_b200.h"])


def _newest_header() -> float:
    return max(h.stat().st_mtime for h in HEADERS)


def _compile(unit: str, flags, verbose: bool) -> Path:
    src = CSRC / unit
    obj = OBJDIR / (unit + ".o")
    if obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, _newest_header()):
        return obj
    cmd = [NVCC, *COMMON, *flags, "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed for %s" % unit)
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJDIR.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    if force:
        for o in OBJDIR.glob("*.o"):
            o.unlink()
    with ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        objs = list(ex.map(lambda kv: _compile(kv[0], kv[1], verbose), UNITS.items()))
    if LIB.exists() and LIB.stat().st_mtime >= max(o.stat().st_mtime for o in objs):
        return LIB
    tmp = LIB.with_suffix(".so.tmp%d" % os.getpid())
    cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-cudart", "static", *map(str, objs), "-o", str(tmp)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc link failed")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
