"""Build and run ``opcount.cpp``: exact floating-point operation counts of
the oracle's hydro stages per cell update (TEST AND MEASUREMENT
INFRASTRUCTURE ONLY; the product package never imports it).

    python -m oracle.opcount [riemann] [slope_type]   # prints the JSON
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "opcount.cpp"
BIN = HERE / "_build" / "opcount"


def build(force: bool = False) -> Path:
    BIN.parent.mkdir(exist_ok=True)
    deps = [SRC, HERE / "ramses_oracle.c", HERE / "ramses_oracle.h"]
    if not force and BIN.exists() and BIN.stat().st_mtime >= max(p.stat().st_mtime for p in deps):
        return BIN
    tmp = BIN.with_name("opcount.tmp%d" % os.getpid())
    subprocess.run(["g++", "-O1", "-std=c++17", "-Wno-unused-function", str(SRC), "-o", str(tmp)], check=True)
    os.replace(tmp, BIN)
    return BIN


def counts(riemann: int = 3, slope_type: int = 2) -> dict:
    out = subprocess.run([str(build()), str(riemann), str(slope_type)], check=True, capture_output=True, text=True)
    return json.loads(out.stdout)


def total_ops(entry: dict) -> float:
    """Every counted operation: flops + compares + abs + copysign + negations."""
    return entry["flops"] + entry["cmp"] + entry["abs"] + entry["copysign"] + entry["neg"]


if __name__ == "__main__":
    r = int(sys.argv[1]) if len(sys.argv) > 1 else 3
    s = int(sys.argv[2]) if len(sys.argv) > 2 else 2
    print(json.dumps(counts(r, s), indent=1))
