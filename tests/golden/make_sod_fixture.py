"""Generate tests/golden/sod_tube_ana.csv from the reference's own Sod
known-answer table (tests/hydro/sod-tube/sod-tube-ana.dat: index, x, u, rho,
P, e at t=0.245, gamma=1.4, left (1,0,1), right (0.125,0,0.1), interface at
x=0.5). Every 4th row is kept (x, u, rho, P). Run once where the reference
tree is available; the CSV is committed.

    python tests/golden/make_sod_fixture.py <reference>/tests/hydro/sod-tube/sod-tube-ana.dat
"""
import sys
from pathlib import Path

import numpy as np

if len(sys.argv) != 2:
    sys.exit("usage: make_sod_fixture.py <path of the reference's tests/hydro/sod-tube/sod-tube-ana.dat>")
SRC = Path(sys.argv[1])
OUT = Path(__file__).resolve().parent / "sod_tube_ana.csv"

d = np.loadtxt(SRC)
sub = d[::4][:, [1, 2, 3, 4]]
np.savetxt(OUT, sub, delimiter=",", header="x,u,rho,p  (t=0.245; source: reference sod-tube-ana.dat, every 4th row)",
           fmt="%.4e")
print("wrote", OUT, sub.shape)
