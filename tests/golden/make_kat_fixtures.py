"""Generate tests/golden/kat_analytic.json from the reference's own analytic test
utilities (ouxsbli/tests/utils/sod_exact.py and oblique_shock.py of the reference
checkout), so that this project's independent restatements (tests/sod_exact.py,
tests/oblique_shock.py) are pinned against them.

Run where a reference checkout is at hand, giving its root (the tests do not need
it: they read only the JSON):

    python tests/golden/make_kat_fixtures.py <path of the reference checkout>
"""
from __future__ import annotations

import importlib.util
import json
import math
import pathlib
import sys

import numpy as np


def _load(path: pathlib.Path, name: str):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main(ref_root: str) -> None:
    utils = pathlib.Path(ref_root) / "ouxsbli" / "tests" / "utils"
    sod = _load(utils / "sod_exact.py", "ref_sod_exact")
    osk = _load(utils / "oblique_shock.py", "ref_oblique_shock")
    out = {"source": "ouxsbli/tests/utils/{sod_exact,oblique_shock}.py of the reference"}
    # Sod profiles: the default problem, a second pair of states, at a few times
    x = np.linspace(0.0, 1.0, 41)
    cases = []
    for states, t in (((1.0, 0.0, 1.0, 0.125, 0.0, 0.1), 0.2), ((1.0, 0.0, 1.0, 0.125, 0.0, 0.1), 0.1),
                      ((2.0, 0.1, 3.0, 0.5, -0.2, 0.4), 0.12)):
        rho, u, p = sod.solve(x, t, *states, gamma=1.4, x0=0.5)
        cases.append({"states": list(states), "t": t, "x": x.tolist(), "rho": np.asarray(rho).tolist(),
                      "u": np.asarray(u).tolist(), "p": np.asarray(p).tolist()})
    out["sod"] = cases
    # oblique shock: free stream, post-shock state, reflected state (the OS test's inputs)
    M0, gamma, R, p_tot, T_tot = 2.0, 1.4, 287.03, 100.0e3, 295.0
    beta, beta_r = math.pi * 37.2 / 180.0, math.pi * 44.1 / 180.0
    u0, p0, T0 = osk.free_stream(M0, gamma, R, p_tot, T_tot)
    rho2, p2, T2 = osk.oblique_shock(M0, p0, T0, beta, gamma, R)
    rho3, ux3, uy3, p3 = osk.reslected_shock(M0, gamma, R, p_tot, T_tot, beta, beta_r)
    out["oblique"] = {"M0": M0, "gamma": gamma, "R": R, "p_tot": p_tot, "T_tot": T_tot, "beta": beta,
                      "beta_r": beta_r, "free_stream": [u0, p0, T0], "post_shock": [rho2, p2, T2],
                      "reflected": [rho3, ux3, uy3, p3],
                      "downstream_mach": float(osk.downstream_mach(M0, 37.2, 8.0, gamma))}
    dst = pathlib.Path(__file__).resolve().parent / "kat_analytic.json"
    dst.write_text(json.dumps(out, indent=1))
    print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_kat_fixtures.py <path of the reference checkout>")
    main(sys.argv[1])
