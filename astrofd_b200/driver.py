"""The reference driver's loop iteration on device blocks, and the accuracy
protocol of the mixed-precision + learned-con2prim path.

``DriverStep`` is one iteration of solvers/srhd3d_mpi_muscl.py's time loop
(:288-326) for the RMHD jet: ghost fills (y/z, +x outflow, nozzle), one
SSPRK3 step, ghost fills again, then the operator-split sources (cooling,
two-temperature).  ``rho_l1_arms`` runs five such loops in lockstep and
reports how far each drifts from plain float64.
"""
import numpy as np


class DriverStep:
    """One reference driver-loop iteration on device tensors."""

    def __init__(self, n, ng, core_cfg, nozzle_cfg, src_cfg, slab=None, halo="step"):
        from .core import boundary, nozzle, rmhd_core, source_terms
        self.B, self.N, self.R, self.S = boundary, nozzle, rmhd_core, source_terms
        self.n, self.ng = n, ng
        self.d = 1.0 / n
        self.dt = core_cfg["CFL"] * self.d
        self.noz, self.src = nozzle_cfg, src_cfg
        self.slab = slab
        self.halo = halo
        self.bufs = None
        self.rng = np.random.default_rng(1234 + (777 * slab.rank if slab else 0))

    def bcs(self, pr):
        if self.noz.get("YZ_BOUNDARY") == "outflow":
            self.B.apply_outflow_yz(pr, self.ng)
        else:
            self.B.apply_periodic_yz(pr, self.ng)
        if self.slab is None or self.slab.last:
            self.B.apply_outflow_right_x(pr, self.ng)
        if self.slab is None or self.slab.first:
            self.N.apply_nozzle_left_x(pr, self.d, self.d, self.d, self.n, self.n, 0.5, 0.5,
                                       self.rng, self.noz)

    def __call__(self, pr, out, profile=False):
        d = self.d
        if self.slab is not None:
            self.slab.exchange(pr)
        self.bcs(pr)
        times = None
        if profile:
            _, times, launches = self.R.engine().step_profiled(pr, d, d, d, self.dt, 3, out)
            times = (times, launches)
        elif self.slab is not None and self.halo == "stage":
            if self.bufs is None:
                self.bufs = [out.new_empty(out.shape) for _ in range(2)]
            self.slab.step_stagewise(
                lambda p0, pk, dst, st: self.R.step_stage(p0, pk, dst, d, d, d, self.dt, 3, st),
                pr, out, self.bufs, 3)
        else:
            self.R.step_ssprk3(pr, d, d, d, self.dt, out=out)
        self.bcs(out)
        self.S.apply_cooling_heating(out, self.dt, self.src)
        self.S.apply_two_temperature(out, self.dt, self.src)
        return out, pr, times



def norms(a, b, ng):
    """Relative L1 and Linf of rho, p and W of state a against state b over
    the interior."""
    import torch
    i = slice(ng, -ng)

    def fields(q):
        q = q[:, i, i, i]
        return {"rho": q[0], "p": q[4],
                "W": 1.0 / torch.sqrt(1.0 - (q[1] ** 2 + q[2] ** 2 + q[3] ** 2))}

    fa, fb = fields(a), fields(b)
    return {k: {"l1": float(((fa[k] - fb[k]).abs().mean() / fb[k].abs().mean()).item()),
                "linf": float(((fa[k] - fb[k]).abs().max() / fb[k].abs().max()).item())}
            for k in fb}



# The stable member of the 256^3 configuration's family: the same scheme and
# sources (RMHD, Gamma 4/3, WENO5 + "hlld", SSPRK3, CFL 0.35, resistivity,
# two-temperature, cooling, outflow boundaries) with an unmagnetised jet at
# the 128^3 RMHD configuration's v = 0.99 (W = 7.09), on which two float64 runs
# 1e-12 apart stay 1e-12 apart for 100 steps at 256^3.  Any magnetic field
# makes the reference scheme's jet chaotic (ambient sigma = 1e-4 at v = 0.9
# already by step 40).
STABLE = dict(jet_v=0.99, sigma_jet=0.0, sigma_amb=0.0)


def rho_l1_arms(n, steps, jet_v, sigma_jet, sigma_amb, boundaries="baseline",
                flux_mode="conservative", net=None, every=10, stage_kernel="split"):
    """Five runs of the same driver loop in lockstep: plain float64 (the
    comparison), mixed + learned (the headline path), float64 with a 1e-12
    relative density perturbation of the initial state (the floor: how far two
    float64 runs drift apart on this flow), and the headline path's two halves
    on their own: float32 faces with the reference's con2prim start, and
    float64 faces with the learned start.  Returns the density L1 of each
    against plain float64 every `every` steps and at the end, the norms of rho,
    p and W of the last step, and the con2prim counts."""
    import torch
    from . import learned_c2p
    from .core import rmhd_core
    from .workloads import rmhd_jet, rmhd_jet_config
    core, noz, src = rmhd_jet_config(n, 3, vjet=jet_v, sigma_amb=sigma_amb,
                                     sigma_jet=sigma_jet, boundaries=boundaries)
    rmhd_core.set_c2p_network(learned_c2p.load(net or learned_c2p.DATA))
    arms = {"fp64": ("fp64", False, 0.0), "mixed_learned": ("mixed", True, 0.0),
            "fp64_perturbed_1e-12": ("fp64", False, 1e-12),
            "mixed_reference_guess": ("mixed", False, 0.0),
            "fp64_learned_guess": ("fp64", True, 0.0)}
    state = {}
    for name, (prec, learned, perturb) in arms.items():
        pr = rmhd_jet(n, 3, sigma_amb=sigma_amb)
        if perturb:
            pr[0] *= 1.0 + perturb * np.random.default_rng(5).standard_normal(pr[0].shape)
        a = torch.from_numpy(pr).cuda()
        state[name] = [a, torch.empty_like(a), DriverStep(n, 3, core, noz, src),
                       {"cells": 0, "learned_fallback": 0, "hydro_fallback": 0,
                        "wait_timeouts": 0}]
    every = max(1, every)
    history = []
    for k in range(1, steps + 1):
        for name, (prec, learned, _) in arms.items():
            rmhd_core.configure(dict(core, PRECISION=prec, FLUX_MODE=flux_mode,
                                     C2P_GUESS="learned" if learned else "reference",
                                     STAGE_KERNEL=stage_kernel))
            st = state[name]
            rmhd_core.c2p_stats(reset=True)
            st[0], st[1], _ = st[2](st[0], st[1])
            for key, v in rmhd_core.c2p_stats(reset=True).items():
                if key in st[3]:
                    st[3][key] += v
        if k % every == 0 or k == steps:
            ref = state["fp64"][0]
            rec = {"step": k}
            for name in arms:
                if name != "fp64":
                    rec[name] = norms(state[name][0], ref, 3)["rho"]["l1"]
            history.append(rec)
    ref = state["fp64"][0]
    out = {"steps": steps, "grid": n, "jet_v": jet_v, "sigma_jet": sigma_jet,
           "sigma_amb": sigma_amb, "boundaries": boundaries, "flux_mode": flux_mode,
           "rho_l1": {name: history[-1][name] for name in arms if name != "fp64"},
           "mixed_learned_vs_fp64": norms(state["mixed_learned"][0], ref, 3),
           "fp64_perturbed_1e-12_vs_fp64": norms(state["fp64_perturbed_1e-12"][0], ref, 3),
           "rho_l1_history": history,
           "c2p_counts": {name: state[name][3] for name in arms}}
    del state
    torch.cuda.empty_cache()
    return out
