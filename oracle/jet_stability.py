"""Diagnostic of the reference algorithm itself (not used by the tests): a
pure-hydro RMHD jet (B = 0, v_jet = 0.9, W = 2.29, WENO5 + "hlld", SSPRK3,
CFL 0.35, the reference driver's ghost fills) run by the reference's own Numba
code (core/rmhd_core.py step_ssprk3 :1609, core/boundary.py, core/nozzle.py,
imported read-only from a checkout) and by the C oracle, printing the maximum
density and the total D = rho W of the interior every few steps.

Both grow without bound within ~40 steps at 32^3 (max rho ~1e4, total D x100):
the reference's scheme (componentwise reconstruction of the three-velocity,
v and p caps in prim_to_cons, the hydro fallback of cons_to_prim_rmhd) is not
stable for these relativistic jets, so a 100-step comparison of two runs of it
measures the blow-up, not the precision of either run.

usage: python oracle/jet_stability.py oracle [n] [steps]
       python oracle/jet_stability.py reference <n> <steps> <AstroFD checkout>
"""
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))


def main():
    which = sys.argv[1]
    n = int(sys.argv[2]) if len(sys.argv) > 2 else 32
    K = int(sys.argv[3]) if len(sys.argv) > 3 else 40
    from astrofd_b200.workloads import rmhd_jet, rmhd_jet_config
    ng, d = 3, 1.0 / n
    core, noz, _ = rmhd_jet_config(n, ng, vjet=0.9, sigma_amb=0.0, sigma_jet=0.0)
    core = dict(core, RESISTIVE_ENABLED=False)
    pr = rmhd_jet(n, ng, sigma_amb=0.0)
    dt = core["CFL"] * d
    rng = np.random.default_rng(1234)
    if which == "reference":
        os.environ["PYTHONDONTWRITEBYTECODE"] = "1"
        sys.dont_write_bytecode = True
        if len(sys.argv) < 5:
            sys.exit("reference mode needs the path of an AstroFD checkout (4th argument)")
        sys.path.insert(0, sys.argv[4])
        from core import boundary as B, nozzle as N, rmhd_core as R
        R.configure(core)
        step = lambda a: R.step_ssprk3(a, d, d, d, dt)
        bcs = lambda a: (B.apply_periodic_yz(a, ng), B.apply_outflow_right_x(a, ng),
                         N.apply_nozzle_left_x(a, d, d, d, n, n, 0.5, 0.5, rng, noz))
    else:
        import oracle as O
        P = O.params_from_config("rmhd", dict(core, FLUX_MODE="reference"))
        step = lambda a: O.step(P, a, d, d, d, dt, 3)
        bcs = lambda a: (O.apply_periodic_yz(a, ng), O.apply_outflow_right_x(a, ng),
                         O.apply_nozzle_left_x(a, d, d, d, n, n, 0.5, 0.5, rng, noz))
    i = slice(ng, -ng)
    lorentz = lambda q: 1.0 / np.sqrt(1.0 - (q[1] ** 2 + q[2] ** 2 + q[3] ** 2))
    D0 = float((pr[0] * lorentz(pr))[i, i, i].sum())
    for s in range(K):
        bcs(pr)
        pr = step(pr)
        if (s + 1) % 5 == 0:
            q = pr[:, i, i, i]
            print(json.dumps({"step": s + 1, "rho_max": float(q[0].max()),
                              "D_total_over_initial": float((q[0] * lorentz(q)).sum()) / D0,
                              "v_max": float(np.sqrt((q[1:4] ** 2).sum(0)).max()),
                              "p_max": float(q[4].max())}), flush=True)


if __name__ == "__main__":
    main()
