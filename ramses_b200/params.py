"""Host-side mirror of RAMSES's ``&HYDRO_PARAMS`` / ``&AMR_PARAMS`` knobs that the
hydro step reads (``hydro/hydro_parameters.f90:74-89``, read by
``hydro/read_hydro_params.f90:43-54,138``; ``amr/amr_parameters.f90``).

Defaults are the reference's defaults. Values outside what the CUDA path
implements are rejected when the library is initialised (there is no CPU
fallback), mirroring the reference's ``stop`` on an unknown Riemann solver
(``hydro/umuscl.f90:801-803``) or slope type (``:1474-1476``).
"""
from __future__ import annotations

import dataclasses
import re
from typing import Dict, List

RIEMANN_CODES = {"llf": 1, "hll": 2, "hllc": 3, "acoustic": 4, "exact": 5}
SCHEME_CODES = {"muscl": 0, "plmde": 1}
SLOPE_TYPES = (0, 1, 2, 3, 7, 8)


@dataclasses.dataclass
class HydroParams:
    gamma: float = 1.4
    courant_factor: float = 0.5
    smallr: float = 1e-10
    smallc: float = 1e-10
    slope_type: int = 1
    slope_theta: float = 1.5
    riemann: str = "llf"
    scheme: str = "muscl"
    interpol_var: int = 0
    interpol_type: int = 1
    pressure_fix: bool = False
    difmag: float = 0.0
    beta_fix: float = 0.0
    niter_riemann: int = 10

    @property
    def riemann_code(self) -> int:
        try:
            return RIEMANN_CODES[self.riemann.strip().lower()]
        except KeyError:
            raise ValueError("unknown Riemann solver %r (supported: llf, hll, hllc, acoustic, exact)" % self.riemann)

    @property
    def scheme_code(self) -> int:
        try:
            return SCHEME_CODES[self.scheme.strip().lower()]
        except KeyError:
            raise ValueError("scheme %r not supported (muscl, plmde)" % self.scheme)

    def validate(self) -> None:
        self.riemann_code  # noqa: B018 - raises on unknown solver
        if self.slope_type not in SLOPE_TYPES:
            raise ValueError("Unknown slope type %r" % self.slope_type)
        self.scheme_code  # noqa: B018 - raises on unknown scheme
        if not (self.difmag >= 0.0) or self.difmag == float("inf"):
            raise ValueError("difmag must be finite and >= 0")
        if not (self.beta_fix >= 0.0) or self.beta_fix == float("inf"):
            raise ValueError("beta_fix must be finite and >= 0")
        if self.riemann_code == 5 and self.niter_riemann < 1:
            raise ValueError("niter_riemann must be >= 1 for the exact Riemann solver")
        if self.interpol_var not in (0, 1, 2) or self.interpol_type not in (0, 1, 2, 3, 4):
            raise ValueError("bad interpol_var/interpol_type")
        if self.interpol_type == 4 and self.interpol_var != 2:
            raise ValueError("interpol_type=4 is designed for interpol_var=2")


def parse_namelist(text: str) -> Dict[str, Dict[str, str]]:
    """Minimal Fortran namelist reader: {group: {name: raw value}}."""
    groups: Dict[str, Dict[str, str]] = {}
    for m in re.finditer(r"&(\w+)(.*?)\n\s*/", text, flags=re.S):
        g = m.group(1).upper()
        body = re.sub(r"!.*", "", m.group(2))
        entries: Dict[str, str] = {}
        for line in re.split(r"[\n,](?=\s*[A-Za-z_][\w()]*\s*=)", body):
            if "=" in line:
                k, v = line.split("=", 1)
                entries[k.strip().lower()] = v.strip().rstrip(",")
        groups[g] = entries
    return groups


def _fortran_value(v: str):
    v = v.strip()
    if v.lower() in (".true.", "t"):
        return True
    if v.lower() in (".false.", "f"):
        return False
    if v[:1] in "'\"":
        return v.strip("'\"")
    try:
        return int(v)
    except ValueError:
        return float(v.lower().replace("d", "e"))


def hydro_params_from_namelist(text: str) -> HydroParams:
    g = parse_namelist(text).get("HYDRO_PARAMS", {})
    hp = HydroParams()
    fields = {f.name for f in dataclasses.fields(HydroParams)}
    for k, v in g.items():
        if k in fields:
            setattr(hp, k, _fortran_value(v))
    for k, v in parse_namelist(text).get("REFINE_PARAMS", {}).items():
        if k in ("interpol_var", "interpol_type"):
            setattr(hp, k, _fortran_value(v))
    return hp


@dataclasses.dataclass
class RefineParams:
    """Gradient refinement criterion of &REFINE_PARAMS with the reference's
    defaults (hydro/hydro_parameters.f90:47-52): a negative err_grad_* switches
    that criterion off."""
    err_grad_d: float = -1.0
    err_grad_p: float = -1.0
    err_grad_u: float = -1.0
    floor_d: float = 1e-10
    floor_u: float = 1e-10
    floor_p: float = 1e-10


def refine_params_from_namelist(text: str) -> RefineParams:
    rp = RefineParams()
    fields = {f.name for f in dataclasses.fields(RefineParams)}
    for k, v in parse_namelist(text).get("REFINE_PARAMS", {}).items():
        if k in fields:
            setattr(rp, k, float(_fortran_value(v)))
    return rp


def nsubcycle_from_namelist(text: str, nlevelmax: int) -> List[int]:
    """``nsubcycle`` of ``&RUN_PARAMS`` (default 2 for every level), with
    Fortran repeat counts (``3*1,2``)."""
    out = [2] * (nlevelmax + 1)
    raw = parse_namelist(text).get("RUN_PARAMS", {}).get("nsubcycle")
    if raw:
        vals: List[int] = []
        for tok in raw.replace(" ", "").split(","):
            if "*" in tok:
                r, v = tok.split("*")
                vals += [int(v)] * int(r)
            elif tok:
                vals.append(int(tok))
        for i, v in enumerate(vals):
            if i + 1 <= nlevelmax:
                out[i + 1] = v
    return out
