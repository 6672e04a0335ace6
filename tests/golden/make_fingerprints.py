"""Generate tests/golden/fingerprints.json: whole-state fingerprints
(tests/helpers.py fingerprint, after the reference's check_solution) of the
FP64 oracle on two seeded runs, 64^3 uniform Sedov (hllc, slope 1, C=0.8) for
10 coarse steps and the AMR Sedov tree 4->6 (nsubcycle 2) for 5 coarse steps.

Run from the repository root:  python tests/golden/make_fingerprints.py
"""
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import oracle  # noqa: E402
from helpers import fingerprint, sedov_amr, sedov_uniform  # noqa: E402

CASES = {"sedov64_uniform_10": (lambda: sedov_uniform(6), 10),
         "sedov_amr_4_6_5": (lambda: sedov_amr(4, 6), 5)}


def main():
    out = {}
    for name, (make, steps) in CASES.items():
        tree, hp, u = make()
        orc = oracle.OracleRun(tree, hp, u, nsubcycle=[2] * 33)
        for _ in range(steps):
            orc.coarse_step()
        out[name] = {"steps": steps, "t": orc.t, "fingerprint": fingerprint(tree, orc.uold, hp.gamma)}
    (ROOT / "tests" / "golden" / "fingerprints.json").write_text(json.dumps(out, indent=1) + "\n")
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
