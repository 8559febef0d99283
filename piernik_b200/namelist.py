"""Reader for the parts of PIERNIK's problem.par that the sweep path uses.

Fortran namelist groups (``$NAME ... /`` or ``&NAME ... /``) are parsed into
dictionaries; ``read_problem_par`` maps BASE_DOMAIN, FLUID_IONIZED,
FLUID_NEUTRAL, FLUID_DUST, NUMERICAL_SETUP and END_CONTROL onto ``Setup``.
A second namelist string, like the reference's ``piernik -n '&GROUP k=v/'``
command-line override (src/IO/dataio_pub.F90:82), is applied after the file.
"""
from __future__ import annotations

import re
from typing import Dict, List, Optional

from .config import BND_NAMES, Setup

def _strip_comments(text: str) -> str:
    out = []
    for line in text.splitlines():
        res, q = [], None
        for ch in line:
            if q:
                res.append(ch)
                if ch == q:
                    q = None
            elif ch in "'\"":
                q = ch
                res.append(ch)
            elif ch == "!":
                break
            else:
                res.append(ch)
        out.append("".join(res))
    return "\n".join(out)


def _value(tok: str):
    t = tok.strip()
    if not t:
        return None
    if t[0] in "'\"":
        return t[1:-1]
    lo = t.lower()
    if lo in (".true.", "t", ".t."):
        return True
    if lo in (".false.", "f", ".f."):
        return False
    try:
        return int(t)
    except ValueError:
        pass
    try:
        return float(lo.replace("d", "e"))
    except ValueError:
        return t


def _split_values(s: str) -> List[str]:
    vals, cur, q = [], [], None
    for ch in s:
        if q:
            cur.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            cur.append(ch)
        elif ch in ",\n":
            vals.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    vals.append("".join(cur))
    return [v for v in (x.strip() for x in vals) if v]


def parse_namelists(text: str) -> Dict[str, Dict[str, object]]:
    """Parse all namelist groups of a file; keys are lower case."""
    text = _strip_comments(text)
    groups: Dict[str, Dict[str, object]] = {}
    pos = 0
    pat = re.compile(r"[$&]\s*([A-Za-z_][A-Za-z0-9_]*)")
    while True:
        m = pat.search(text, pos)
        if not m:
            break
        name = m.group(1).upper()
        body_start = m.end()
        # the group ends at the first '/' outside quotes
        i, q = body_start, None
        while i < len(text):
            ch = text[i]
            if q:
                if ch == q:
                    q = None
            elif ch in "'\"":
                q = ch
            elif ch == "/":
                break
            i += 1
        body = text[body_start:i]
        pos = i + 1
        entries = groups.setdefault(name, {})
        # split "key = values" pairs
        parts = re.split(r"([A-Za-z_][A-Za-z0-9_]*(?:\(\s*\d*\s*:?\s*\d*\s*\))?)\s*=", body)
        for k in range(1, len(parts) - 1, 2):
            key = re.sub(r"\s", "", parts[k]).lower()
            vals = [_value(v) for v in _split_values(parts[k + 1])]
            entries[key] = vals[0] if len(vals) == 1 else vals
    return groups


def read_problem_par(text: str, cmdline: Optional[str] = None, setup: Optional[Setup] = None,
                     fluids: Optional[List[str]] = None, magnetic: Optional[bool] = None) -> Setup:
    """Build a Setup from problem.par text (and an optional override namelist).

    Which fluids exist and whether B is evolved are compile-time choices of the
    reference (IONIZED / NEUTRAL / DUST / MAGNETIC in piernik.def), so they are
    arguments here; their gamma values come from the FLUID_* groups.
    """
    g = parse_namelists(text)
    if cmdline:
        for name, ent in parse_namelists(cmdline).items():
            g.setdefault(name, {}).update(ent)
    s = setup if setup is not None else Setup()
    kw = {}
    dom = g.get("BASE_DOMAIN", {})
    if "n_d" in dom:
        nd = dom["n_d"] if isinstance(dom["n_d"], list) else [dom["n_d"]]
        kw["n"] = tuple(int(x) for x in (list(nd) + [1, 1, 1])[:3])
    if "nb" in dom:
        kw["nb"] = int(dom["nb"])
    lo = list(s.xmin)
    hi = list(s.xmax)
    for d, ax in enumerate("xyz"):
        if f"{ax}min" in dom:
            lo[d] = float(dom[f"{ax}min"])
        if f"{ax}max" in dom:
            hi[d] = float(dom[f"{ax}max"])
    kw["xmin"], kw["xmax"] = tuple(lo), tuple(hi)
    bnd = [list(x) for x in s.bnd]
    for d, ax in enumerate("xyz"):
        for side, sfx in enumerate("lr"):
            key = f"bnd_{ax}{sfx}"
            if key in dom:
                name = str(dom[key]).strip().lower()
                if name not in BND_NAMES:
                    raise ValueError(f"boundary {key}={name!r} is not supported by the sweep path")
                bnd[d][side] = BND_NAMES[name]
    kw["bnd"] = tuple(tuple(x) for x in bnd)
    kinds = fluids if fluids is not None else [k for k, _ in s.fluids]
    groups = {"ion": "FLUID_IONIZED", "neu": "FLUID_NEUTRAL", "dst": "FLUID_DUST"}
    old = dict(s.fluids)
    kw["fluids"] = [(k, float(g.get(groups[k], {}).get("gamma", old.get(k, 5.0 / 3.0)))) for k in kinds]
    if magnetic is not None:
        kw["magnetic"] = bool(magnetic)
    ns = g.get("NUMERICAL_SETUP", {})
    for key in ("cfl", "cfl_glm", "glm_alpha", "smalld", "smallei", "dt_initial", "dt_max_grow", "dt_min",
                "dt_max", "cfl_max", "dt_shrink"):
        if key in ns:
            kw[key] = float(ns[key])
    for key in ("use_smalld", "use_smallei", "disallow_negatives", "ch_grid", "use_eglm"):
        if key in ns:
            kw[key] = bool(ns[key])
    if "limiter" in ns:
        kw["limiter"] = str(ns["limiter"]).strip().lower()
        if "limiter_b" not in ns:
            kw["limiter_b"] = kw["limiter"]
    if "limiter_b" in ns:
        kw["limiter_b"] = str(ns["limiter_b"]).strip().lower()
    if "integration_order" in ns:
        kw["integration_order"] = int(ns["integration_order"])
    if "cflcontrol" in ns:
        kw["cflcontrol"] = str(ns["cflcontrol"]).strip().lower()
    if "max_redostep_attempts" in ns:
        kw["max_redostep_attempts"] = int(ns["max_redostep_attempts"])
    if "skip_sweep" in ns:
        v = ns["skip_sweep"]
        kw["skip_sweep"] = tuple(bool(x) for x in (v if isinstance(v, list) else [v] * 3))
    if "interpol_str" in ns:
        val = str(ns["interpol_str"]).strip().lower()
        names = {"linear": "linear", "lin": "linear", "1": "linear", "weno3": "weno3", "wo3": "weno3", "2": "weno3"}
        if val not in names:
            raise ValueError(f"interpol_str={val!r} is outside the sweep path this library implements")
        kw["interpolation"] = names[val]                  # interpolations.F90:set_interpolations
    if "w_epsilon" in ns:
        kw["w_epsilon"] = float(ns["w_epsilon"])
    for key in ("ord_fluid_prolong", "ord_mag_prolong"):
        if key in ns:
            kw[key] = int(ns[key])
    if "solver_str" in ns:                               # global.F90:423-437
        val = str(ns["solver_str"]).strip().lower()
        if val in ("", "riemann", "riemann_split"):
            kw["solver"] = "split"
        elif val in ("unsplit", "van_leer", "riemann_unsplit"):
            kw["solver"] = "unsplit"
        else:
            raise ValueError(f"solver_str={val!r} is outside the sweep path this library implements")
    if "divb_0" in ns:
        val = str(ns["divb_0"]).strip().lower()
        if val not in ("hdc", "glm", "divergence cleaning"):
            raise ValueError(f"divB_0={val!r} is outside the sweep path this library implements")
    end = g.get("END_CONTROL", {})
    if "tend" in end:
        kw["tend"] = float(end["tend"])
    if "nend" in end:
        kw["nend"] = int(end["nend"])
    out = s.replace(**kw)
    return out
