"""Generate tests/golden/<test>_regression.json from one of the reference's own
regression tests (tests/hydro/<test>/: the namelist <test>.nml and the
checksums <test>-ref.dat that tests/visu/visu_ramses.py's check_solution
compares a run's snapshot against). The JSON holds the namelist values the
1D oracle run needs and the reference checksums; the test
tests/test_oracle_regression_cpu.py reruns the namelist in the oracle and
compares. Run once where the reference tree is available; the JSON is
committed.

    python tests/golden/make_regression_fixture.py <reference>/tests/hydro/sod-tube
"""
import json
import re
import sys
from pathlib import Path


def parse_namelist(text):
    """Fortran namelist groups -> {group: {key: [values]}} for the value
    forms these files use: numbers (d exponents), r*value repeats,
    quoted strings and logicals."""
    groups = {}
    for m in re.finditer(r"&(\w+)(.*?)\n\s*/", text, re.S):
        body = {}
        for line in m.group(2).splitlines():
            line = line.split("!")[0].strip()
            if "=" not in line:
                continue
            key, val = line.split("=", 1)
            vals = []
            for tok in [t.strip() for t in val.split(",") if t.strip()]:
                rep = 1
                rm = re.fullmatch(r"(\d+)\*(.+)", tok)
                if rm:
                    rep, tok = int(rm.group(1)), rm.group(2)
                if tok.lower() in (".true.", ".false."):
                    v = tok.lower() == ".true."
                elif tok[0] in "'\"":
                    v = tok.strip("'\"")
                else:
                    v = float(tok.lower().replace("d", "e"))
                vals += [v] * rep
            body[key.strip().lower()] = vals
        groups[m.group(1).upper()] = body
    return groups


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_regression_fixture.py <path of the reference's tests/hydro/<test> directory>")
    src = Path(sys.argv[1])
    name = src.name
    nml = parse_namelist((src / (name + ".nml")).read_text())
    ref = {}
    for line in (src / (name + "-ref.dat")).read_text().splitlines():
        if ":" in line:
            k, v = line.split(":", 1)
            ref[k.strip()] = float(v)
    flags = (src / "config.txt").read_text().strip()
    out = {
        "source": "reference tests/hydro/%s/%s.nml and %s-ref.dat" % (name, name, name),
        "build_flags": flags,
        "namelist": nml,
        "checksums": ref,
        # tests/visu/visu_ramses.py check_solution: var_tol {"all": 3e-13},
        # threshold 2e-14, min_variance 1e-14 (its defaults; the test passes none)
        "checker": {"tolerance": 3.0e-13, "threshold": 2.0e-14, "min_variance": 1.0e-14},
    }
    dst = Path(__file__).resolve().parent / (name.replace("-", "_") + "_regression.json")
    dst.write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")
    print("wrote", dst)


if __name__ == "__main__":
    main()
