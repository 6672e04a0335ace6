"""The oracle against the reference's own regression checksums.

The reference's regression suite runs each namelist under tests/hydro/ and
compares the final snapshot with <test>-ref.dat through
tests/visu/visu_ramses.py's check_solution: per variable a sum over the leaf
cells (log10|.| for density and pressure, |.| otherwise, values within
min_variance of the mean replaced by the mean, values below threshold
dropped), each within a relative tolerance of 3e-13. sod-tube is the one
pure-hydro 1D test (NDIM=1: hllc, moncen slopes, interpol_type 2, levels 3
to 10 refined on density, velocity and pressure gradients with nexpand 1,
walls at both ends, nsubcycle 1,1,1,2 from levelmin, snapshot at the first
coarse step starting after t = 0.245).

The oracle's NDIM=1 restatement of the whole run (oracle/ramses_oracle_1d.c:
init_refine, adaptive_loop, amr_step with flag_fine/refine_fine/
make_grid_fine, godunov_fine, courant_fine, make_boundary_hydro; the Riemann
solvers shared with the 3D restatement) is rerun from the committed
namelist values and checked with the same sums and tolerance. The fixture
comes from tests/golden/make_regression_fixture.py.
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest

import oracle
from ramses_b200.params import HydroParams

GOLDEN = Path(__file__).resolve().parent / "golden"


def per_level(values, levelmin, nlevelmax, default):
    """Level-dependent namelist arrays as RAMSES holds them after
    read_params (amr/read_params.f90:440-457): entry k of the namelist
    applies to level levelmin + k - 1; levels below levelmin take 1."""
    out = []
    for lvl in range(1, nlevelmax + 1):
        k = lvl - levelmin
        out.append(1 if k < 0 else (int(values[k]) if k < len(values) else default))
    return out


def run_namelist_1d(nml):
    amr, hyd, ref, ini, bnd, run, outp = (nml.get(g, {}) for g in (
        "AMR_PARAMS", "HYDRO_PARAMS", "REFINE_PARAMS", "INIT_PARAMS", "BOUNDARY_PARAMS", "RUN_PARAMS",
        "OUTPUT_PARAMS"))
    levelmin, nlevelmax = int(amr["levelmin"][0]), int(amr["levelmax"][0])
    nexpand = per_level(amr.get("nexpand", [1]), levelmin, nlevelmax, 1)
    assert len(set(nexpand)) == 1, "the 1D oracle takes one nexpand for all levels"
    hp = HydroParams(gamma=hyd["gamma"][0], riemann=hyd.get("riemann", ["llf"])[0],
                     slope_type=int(hyd.get("slope_type", [1])[0]), courant_factor=hyd.get("courant_factor", [0.5])[0],
                     interpol_var=int(ref.get("interpol_var", [0])[0]),
                     interpol_type=int(ref.get("interpol_type", [1])[0]))
    grads = tuple(ref.get(k, [-1.0])[0] for k in ("err_grad_d", "err_grad_p", "err_grad_u"))
    nreg = int(ini["nregion"][0])
    for k in range(nreg):
        assert ini["region_type(%d)" % (k + 1)][0] == "square"
    regions = [(ini["x_center"][k], ini["length_x"][k], ini["d_region"][k], ini.get("u_region", [0.0] * nreg)[k],
                ini["p_region"][k], ini.get("exp_region", [2.0] * nreg)[k]) for k in range(nreg)]
    boundaries = []
    for i in range(int(bnd.get("nboundary", [0])[0])):
        lo, hi = int(bnd["ibound_min"][i]), int(bnd["ibound_max"][i])
        assert lo == hi and lo in (-1, 1)
        boundaries.append((lo, int(bnd["bound_type"][i])))
    nout = int(outp.get("noutput", [1])[0])
    return oracle.run_1d(hp, grads, levelmin=levelmin, nlevelmax=nlevelmax, ngridmax=int(amr["ngridmax"][0]),
                         tout=outp["tout"][nout - 1], regions=regions, boundaries=boundaries,
                         nsubcycle=per_level(run.get("nsubcycle", [2]), levelmin, nlevelmax, 2),
                         nexpand=nexpand[-1], boxlen=amr.get("boxlen", [1.0])[0])


def snapshot_variables(res, gamma, smallr=1e-10):
    """The hydro file's variables (hydro/output_hydro.f90:80-130): density,
    velocity = rho u / max(rho, smallr), pressure = (gamma-1)(E - (rho u)^2 /
    (2 max(rho, smallr))); and the leaf cells' x, level, dx."""
    u = res["u"]
    d = u[:, 0]
    dd = np.maximum(d, smallr)
    v = u[:, 1] / dd
    e = u[:, 2] - 0.5 * u[:, 1] ** 2 / dd
    p = (gamma - 1.0) * e
    lv = res["level"].astype(np.float64)
    return {"density": d, "velocity_x": v, "pressure": p, "x": res["x"], "level": lv, "dx": 0.5 ** lv}


def checksum(key, a, threshold, min_variance):
    """check_solution's per-variable sum (1D: no vector norms)."""
    av = np.average(a)
    if av != 0.0:
        a = np.where(np.abs(a - av) / abs(av) < min_variance, av, a)
    if key in ("density", "pressure"):
        s = np.log10(np.abs(a))
    else:
        s = np.where(np.abs(a) < threshold, 0.0, np.abs(a))
    return math.fsum(s)


def rel_error(sol, ref):
    if sol == ref == 0.0:
        return 0.0
    if sol == 0.0 or ref == 0.0:
        return math.inf
    return abs(sol - ref) / min(abs(sol), abs(ref))


@pytest.fixture(scope="module")
def sod():
    fx = json.loads((GOLDEN / "sod_tube_regression.json").read_text())
    assert "NDIM=1" in fx["build_flags"] and "SOLVER=hydro" in fx["build_flags"]
    res = run_namelist_1d(fx["namelist"])
    return fx, res


def test_sod_tube_tree_matches_reference(sod):
    """The refinement history: the final tree's leaf count, level sum and
    cell-centre sum are integers or dyadic fractions and match exactly."""
    fx, res = sod
    ref = fx["checksums"]
    assert res["taken"]
    v = snapshot_variables(res, 1.4)
    thr, mv = fx["checker"]["threshold"], fx["checker"]["min_variance"]
    assert len(res["x"]) == ref["ncells"]
    for k in ("level", "x", "dx"):
        assert checksum(k, v[k], thr, mv) == ref[k], k


def test_sod_tube_checksums_within_reference_tolerance(sod):
    """Every checksum of sod-tube-ref.dat within check_solution's 3e-13; the
    time as the info file writes it (E23.15: 15 significant digits)."""
    fx, res = sod
    ref, chk = fx["checksums"], fx["checker"]
    gamma = fx["namelist"]["HYDRO_PARAMS"]["gamma"][0]
    v = snapshot_variables(res, gamma)
    sol = {k: checksum(k, v[k], chk["threshold"], chk["min_variance"]) for k in v}
    sol["ncells"] = float(len(res["x"]))
    sol["time"] = float("%.14e" % res["t"])
    errs = {k: rel_error(sol[k], ref[k]) for k in sol}
    bad = {k: (sol[k], ref[k], e) for k, e in errs.items() if e > chk["tolerance"]}
    assert not bad, bad
    # the sums that do not pass through a threshold agree to the last digit
    assert sol["density"] == ref["density"] and sol["pressure"] == ref["pressure"], errs
    assert sol["time"] == ref["time"]


def test_sod_tube_level_subcycling_remap_matters(sod):
    """Control: without read_params' level remap of nsubcycle (namelist entry
    1 at level 1 instead of levelmin) the run takes other time steps and the
    checksums fail, so the comparison above is sensitive to the run's
    schedule, not only to the hydro arithmetic."""
    fx, _ = sod
    nml = json.loads(json.dumps(fx["namelist"]))
    ns = nml["RUN_PARAMS"]["nsubcycle"]
    nml["RUN_PARAMS"]["nsubcycle"] = ns[2:]  # the first namelist entries would land on levels 1-2
    res = run_namelist_1d(nml)
    assert abs(res["t"] - fx["checksums"]["time"]) > 1e-6
