"""The MLP oracle's analytic gradients against central finite differences
(BF16 rounding switched off, float64 throughout), so the oracle that judges
the tensor-core backward kernels is itself pinned."""
import numpy as np

import mlp_oracle as MO


def test_oracle_gradients_match_finite_differences(monkeypatch):
    monkeypatch.setattr(MO, "bf16", lambda a: np.asarray(a, dtype=np.float64))
    rng = np.random.default_rng(0)
    P = {"W1": rng.normal(0, 0.5, (64, 5)), "b1": rng.normal(0, 0.1, 64),
         "W2": rng.normal(0, 0.15, (64, 64)), "b2": rng.normal(0, 0.1, 64),
         "W3": rng.normal(0, 0.15, (64, 64)), "b3": rng.normal(0, 0.1, 64),
         "W4": rng.normal(0, 0.15, (2, 64)), "b4": rng.normal(0, 0.1, 2),
         "xmu": np.zeros(5), "xsd": np.ones(5), "ymu": np.zeros(2), "ysd": np.ones(2)}
    P = {k: np.asarray(v, dtype=np.float64) for k, v in P.items()}
    X = rng.normal(size=(17, 5))
    T = rng.normal(size=(17, 2))
    # the oracle casts features/targets to float32 like the kernels; use
    # float32-representable data so the finite differences see the same inputs
    X = X.astype(np.float32).astype(np.float64)
    T = T.astype(np.float32).astype(np.float64)
    _, g = MO.loss_and_grads(P, X, T)
    h = 1e-6
    for name in ("W1", "b1", "W3", "W4", "b4"):
        flat = P[name].reshape(-1)
        for idx in rng.choice(flat.size, size=min(6, flat.size), replace=False):
            old = flat[idx]
            flat[idx] = old + h
            lp, _ = MO.loss_and_grads(P, X, T)
            flat[idx] = old - h
            lm, _ = MO.loss_and_grads(P, X, T)
            flat[idx] = old
            fd = (lp - lm) / (2 * h)
            an = g[name].reshape(-1)[idx]
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(fd)), (name, idx, fd, an)
