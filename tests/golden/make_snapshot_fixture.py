"""Generate tests/golden/snapshot_sedov_l3_4.npz: a snapshot written by
ramses_b200.snapshot.write_snapshot (a seeded two-level Sedov state, see
tests/test_snapshot_cpu.py:snapshot_case) and read back by the reference's
own reader, tests/visu/visu_ramses.py load_snapshot. The CPU test checks
that the writer's files still decode to exactly these arrays. Run where the
reference tree is available; the fixture is committed.

    python tests/golden/make_snapshot_fixture.py <reference>/tests/visu
"""
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
sys.path.insert(0, str(HERE.parent))

if len(sys.argv) != 2:
    sys.exit("usage: make_snapshot_fixture.py <path of the reference's tests/visu directory>")
sys.path.insert(0, sys.argv[1])
import visu_ramses  # noqa: E402

from test_snapshot_cpu import FIELDS, snapshot_case  # noqa: E402

from ramses_b200 import snapshot  # noqa: E402

tree, u, gamma, meta = snapshot_case()
with tempfile.TemporaryDirectory() as d:
    cwd = os.getcwd()
    os.chdir(d)
    try:
        snapshot.write_snapshot(".", 7, tree, u, gamma, **meta)
        data = visu_ramses.load_snapshot(7)["data"]
    finally:
        os.chdir(cwd)
order = np.lexsort((data["z"], data["y"], data["x"], data["level"]))
np.savez_compressed(HERE / "snapshot_sedov_l3_4.npz", **{k: np.asarray(data[k])[order] for k in FIELDS})
print("wrote", HERE / "snapshot_sedov_l3_4.npz", len(order), "cells")
