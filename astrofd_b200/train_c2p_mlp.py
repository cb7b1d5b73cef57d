"""Train the learned con2prim guess on the GPU and report its quality.

    python -m astrofd_b200.train_c2p_mlp [--samples 4194304] [--steps 6000]

Data: the learned-c2p sampler (astrofd_b200.learned_c2p.sample_primitives)
plus cells harvested from a 128^3 magnetised-jet run of this library.  Labels:
(log(Z / (D + tau + B^2)), log W) of the reference con2prim's solution, kept only where that
solution is a root of the reference's own equation (elsewhere the reference
returns its hydro fallback, which is no function of the inputs to learn).  Weights go to
astrofd_b200/data/c2p_mlp.npz; a JSON report (loss, polish-step count,
fallback rate, the share of states converged after 0, 1 and 2 polish
steps, max relative primitive error against the full FP64 Newton, and the
same figures without the network) is printed.
"""
import argparse
import json
import time

import numpy as np
import torch

from . import learned_c2p as LC


def harvest_jet(n=128, steps=12, per_snapshot=1 << 19, seed=0):
    """Conserved states of a magnetised-jet run (mixed precision), sampled."""
    from .core import boundary, nozzle, rmhd_core, source_terms
    from .workloads import rmhd_jet, rmhd_jet_config
    core, noz, src = rmhd_jet_config(n, 3)
    rmhd_core.configure(dict(core, PRECISION="mixed", FLUX_MODE="conservative",
                             C2P_GUESS="reference"))
    d = 1.0 / n
    dt = core["CFL"] * d
    a = torch.from_numpy(rmhd_jet(n, 3)).cuda()
    b = torch.empty_like(a)
    rng = np.random.default_rng(seed)
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    prims = []
    for s in range(steps):
        boundary.apply_periodic_yz(a, 3)
        boundary.apply_outflow_right_x(a, 3)
        nozzle.apply_nozzle_left_x(a, d, d, d, n, n, 0.5, 0.5, rng, noz)
        rmhd_core.step_ssprk3(a, d, d, d, dt, out=b)
        a, b = b, a
        source_terms.apply_cooling_heating(a, dt, src)
        source_terms.apply_two_temperature(a, dt, src)
        if s % 3 == 2:
            flat = a[:9].reshape(9, -1)
            idx = torch.randint(0, flat.shape[1], (per_snapshot,), device="cuda", generator=g)
            prims.append(flat[:, idx])
    return torch.cat(prims, dim=1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--samples", type=int, default=1 << 22)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--eval", type=int, default=1 << 20)
    ap.add_argument("--out", default=LC.DATA)
    ap.add_argument("--no-harvest", action="store_true")
    a = ap.parse_args()
    t0 = time.time()
    e = LC.c2p_engine()
    X, T, _ = LC.make_dataset(LC.sample_primitives(a.samples, 11), e, valid_only=True)
    if not a.no_harvest:
        Xj, Tj, _ = LC.make_dataset(harvest_jet(), e, valid_only=True)
        X, T = torch.cat([X, Xj]), torch.cat([T, Tj])
    xmu, xsd, ymu, ysd = LC.normalisation(X, T)
    tr = LC.Trainer(LC.init_params(0, xmu, xsd, ymu, ysd))
    losses = tr.train(X, T, steps=a.steps, batch=a.batch, lr=3e-3, lr_end=5e-5,
                      log_every=max(a.steps // 10, 1))
    t_train = time.time() - t0
    # evaluation on fresh samples (the C4 batch) and on held-out jet cells
    report = {"samples": int(X.shape[0]), "steps": a.steps, "batch": a.batch,
              "train_seconds": round(t_train, 1), "loss": losses}
    sets = {"sampler": LC.sample_primitives(a.eval, 99),
            "sampler_valid": LC.sample_primitives(a.eval, 98)}
    if not a.no_harvest:
        sets["jet128"] = harvest_jet(steps=9, per_snapshot=a.eval // 3, seed=1)
    for name, prim in sets.items():
        Xe, Te, Ue = LC.make_dataset(prim, e, valid_only=(name == "sampler_valid"))
        ref = e.c2p_array(Ue)
        out = {}
        for label, params in (("network", tr.params), ("no_network", None)):
            q, st = LC.c2p_learned(e, Ue, params, max_polish=2)
            rel = ((q - ref).abs() / ref.abs().clamp_min(1e-300))[:5].max(dim=0).values
            n = max(st["cells"], 1)
            hist = [LC.c2p_learned(e, Ue, params, max_polish=k)[1]["learned_polish"] / n
                    for k in (0, 1)] + [st["learned_polish"] / n]
            out[label] = {"cells": st["cells"],
                          "converged_within_0_1_2_polish": hist,
                          "converged_within_2_polish": st["learned_polish"] / n,
                          "fallback_rate": st["learned_fallback"] / n,
                          "mean_polish_steps": st["polish_steps"] / n,
                          "bisection": st["bisection"], "hydro_fallback": st["hydro_fallback"],
                          "max_rel_primitive_error_vs_full_newton": float(rel.max().item()),
                          "frac_rel_error_above_1e-6": float((rel > 1e-6).float().mean().item())}
        Y = tr.forward(Xe)
        out["guess_abs_err_median_logZ_logW"] = (Y - Te).abs().median(dim=0).values.tolist()
        report[name] = out
    LC.save(tr.params.cpu().numpy(), a.out, report=json.dumps(report))
    print(json.dumps(report))


if __name__ == "__main__":
    main()
