"""Learned con2prim initial guess: data, training and evaluation on the GPU.

The network (5 -> 64 -> 64 -> 64 -> 2, ReLU) maps the invariants of a
conserved RMHD state to log(Z / (D + tau + B^2)) and log W of the primitive
state that the reference's full Newton con2prim (core/rmhd_core.py:249)
recovers from it: Z = rho h W^2 is the variable of the reference's Newton
iteration and D + tau + B^2 its second starting point, so a network that
outputs 0 reproduces that start.  log W is an auxiliary target; the solver
uses the first output only.
Everything runs through libastrofd_b200.so: samples are converted with the
library's prim_to_cons, labelled with its reference con2prim, featurised, and
the weights are trained with its tensor-core forward/backward kernels and an
Adam kernel.  There is no counterpart in the reference.

Parameter block (float32, astro_mlp_param_bytes() bytes): the trainable
prefix W1 b1 W2 b2 W3 b3 W4 b4, then xmu[5] xsd[5] ymu[2] ysd[2].
"""
import ctypes as C
import math
import os

import numpy as np
import torch

from . import _lib, runtime as rt

NIN, H, NOUT = 5, 64, 2
_SHAPES = [("W1", (H, NIN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)),
           ("b3", (H,)), ("W4", (NOUT, H)), ("b4", (NOUT,)), ("xmu", (NIN,)), ("xsd", (NIN,)),
           ("ymu", (NOUT,)), ("ysd", (NOUT,))]
DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "c2p_mlp.npz")


def offsets():
    off, o = {}, 0
    for name, shp in _SHAPES:
        n = int(np.prod(shp))
        off[name] = (o, shp)
        o += n
    return off, o


def n_trainable():
    return _lib.load().astro_mlp_trainable()


def init_params(seed=0, xmu=None, xsd=None, ymu=None, ysd=None):
    """He-style init of the float32 parameter block (numpy)."""
    rng = np.random.default_rng(seed)
    off, total = offsets()
    assert total * 4 == _lib.load().astro_mlp_param_bytes()
    flat = np.zeros(total, np.float32)

    def put(name, arr):
        o, shp = off[name]
        flat[o:o + int(np.prod(shp))] = np.asarray(arr, np.float32).reshape(-1)

    for name, fan_in in (("W1", NIN), ("W2", H), ("W3", H), ("W4", H)):
        o, shp = off[name]
        put(name, rng.normal(0.0, math.sqrt(1.0 / fan_in), shp))
    put("xmu", np.zeros(NIN) if xmu is None else xmu)
    put("xsd", np.ones(NIN) if xsd is None else xsd)
    put("ymu", np.zeros(NOUT) if ymu is None else ymu)
    put("ysd", np.ones(NOUT) if ysd is None else ysd)
    return flat


def unpack(flat):
    off, _ = offsets()
    return {k: np.asarray(flat[o:o + int(np.prod(s))]).reshape(s) for k, (o, s) in off.items()}


def sample_primitives(count, seed, gamma=4.0 / 3.0):
    """The learned-c2p sampler: rho log-uniform [1e-4, 10], p [1e-6, 10],
    W [1, 50], isotropic v and B directions, |B| from a log-uniform
    magnetisation sigma = B^2 / (rho h) in [1e-3, 10]."""
    rng = np.random.default_rng(seed)
    rho = 10.0 ** rng.uniform(-4.0, 1.0, count)
    p = 10.0 ** rng.uniform(-6.0, 1.0, count)
    W = 10.0 ** rng.uniform(0.0, math.log10(50.0), count)
    v = np.sqrt(1.0 - 1.0 / W ** 2)

    def iso():
        x = rng.normal(size=(3, count))
        return x / np.linalg.norm(x, axis=0)

    h = 1.0 + gamma / (gamma - 1.0) * p / rho
    sigma = 10.0 ** rng.uniform(-3.0, 1.0, count)
    pr = np.zeros((9, count))
    pr[0] = rho
    pr[1:4] = v * iso()
    pr[4] = p
    pr[5:8] = np.sqrt(sigma * rho * h) * iso()
    return pr


def c2p_engine(gamma=4.0 / 3.0, p_max=1e3, v_max=0.9999):
    from .core._engine import Engine
    e = Engine(_lib.RMHD)
    e.configure(dict(GAMMA=gamma, P_MAX=p_max, V_MAX=v_max))
    return e


def residual(U, q, gamma, p_max, v_max):
    """|f(Z)| / max(1, tau) of the reference's con2prim equation
    (rmhd_f_of_Z, core/rmhd_core.py:229) at Z = rho h W^2 of primitives q.
    Labels whose residual is large come from the reference's hydro fallback,
    not from a root of its equation."""
    SM = 1e-12
    D, tau = U[0], U[4]
    B2 = (U[5:8] ** 2).sum(0)
    SB = (U[1:4] * U[5:8]).sum(0)
    S2 = (U[1:4] ** 2).sum(0)
    v2q = (q[1:4] ** 2).sum(0)
    Z = (q[0] + gamma / (gamma - 1.0) * q[4]) / (1.0 - v2q)
    dZ = Z.clamp_min(SM)
    vb = SB / dZ
    v2 = (S2 + SB * SB * (2.0 * Z + B2) / (dZ * dZ)) / ((Z + B2) ** 2 + SM)
    v2 = torch.where(v2 >= v_max * v_max, torch.full_like(v2, v_max * v_max - 1e-14), v2)
    W2 = 1.0 / (1.0 - v2)
    rho = D / W2.sqrt().clamp_min(SM)
    h = Z / (rho * W2).clamp_min(SM)
    p = ((h - 1.0) * rho * (gamma - 1.0) / gamma).clamp(SM, p_max)
    b2 = B2 / W2 + vb * vb
    f = Z - p + 0.5 * B2 + 0.5 * b2 - D - tau
    return f.abs() / tau.clamp_min(1.0)


def make_dataset(prim, engine, valid_only=False, tol=1e-8):
    """(features [n,5], targets [n,2] = (log(Z / (D + tau + B^2)), log W) of
    the reference con2prim solution, conserved [9,n]) on the device.
    valid_only keeps the states whose reference solution is a root of its
    equation."""
    L = _lib.load()
    q = torch.as_tensor(prim, dtype=torch.float64, device="cuda").contiguous()
    U = engine.p2c_array(q)
    sol = engine.c2p_array(U)
    n = U.shape[1]
    X = torch.empty((n, NIN), dtype=torch.float32, device="cuda")
    _lib.check(L.astro_c2p_features(rt.ptr(U), rt.ptr(X), n, rt.stream_handle()), "features")
    v2 = (sol[1:4] ** 2).sum(0)
    g = engine.p.gamma
    Z = (sol[0] + g / (g - 1.0) * sol[4]) / (1.0 - v2)
    Za = (U[0] + U[4] + (U[5:8] ** 2).sum(0)).clamp_min(1e-12)
    T = torch.stack([torch.log(Z / Za), -0.5 * torch.log1p(-v2)], dim=1).float()
    ok = torch.isfinite(X).all(1) & torch.isfinite(T).all(1)
    if valid_only:
        p = engine.p
        ok &= residual(U, sol, p.gamma, p.p_max, p.v_max) < tol
    return X[ok].contiguous(), T[ok].contiguous(), U[:, ok].contiguous()


def normalisation(X, T):
    return (X.mean(0).cpu().numpy(), X.std(0).clamp_min(1e-6).cpu().numpy(),
            T.mean(0).cpu().numpy(), T.std(0).clamp_min(1e-6).cpu().numpy())


class Trainer:
    """Adam on the device through astro_mlp_train_grad / astro_mlp_adam."""

    def __init__(self, flat_params):
        self.L = _lib.load()
        self.nt = self.L.astro_mlp_trainable()
        self.params = torch.as_tensor(flat_params, dtype=torch.float32).cuda().contiguous()
        self.grad = torch.zeros(self.nt, dtype=torch.float32, device="cuda")
        self.m = torch.zeros_like(self.grad)
        self.v = torch.zeros_like(self.grad)
        self.loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        self.status = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.step_no = 0

    def grad_of(self, X, T):
        self.grad.zero_()
        self.loss.zero_()
        _lib.check(self.L.astro_mlp_train_grad(rt.ptr(self.params), rt.ptr(X), rt.ptr(T), X.shape[0],
                                               rt.ptr(self.grad), rt.ptr(self.loss),
                                               rt.ptr(self.status), rt.stream_handle()),
                   "astro_mlp_train_grad")
        return self.grad, self.loss

    def step(self, X, T, lr):
        self.L.astro_mlp_train_grad(rt.ptr(self.params), rt.ptr(X), rt.ptr(T), X.shape[0],
                                    rt.ptr(self.grad), rt.ptr(self.loss), rt.ptr(self.status),
                                    rt.stream_handle())
        self.step_no += 1
        _lib.check(self.L.astro_mlp_adam(rt.ptr(self.params), rt.ptr(self.grad), rt.ptr(self.m),
                                         rt.ptr(self.v), C.c_float(lr), C.c_float(0.9),
                                         C.c_float(0.999), C.c_float(1e-8), self.step_no,
                                         rt.stream_handle()), "astro_mlp_adam")

    def train(self, X, T, steps, batch=8192, lr=3e-3, lr_end=1e-4, seed=0, log_every=0):
        n = X.shape[0]
        g = torch.Generator(device="cuda")
        g.manual_seed(seed)
        losses = []
        for s in range(steps):
            lr_s = lr * (lr_end / lr) ** (s / max(steps - 1, 1))
            idx = torch.randint(0, n, (batch,), device="cuda", generator=g)
            self.loss.zero_()
            self.step(X[idx].contiguous(), T[idx].contiguous(), lr_s)
            if log_every and (s % log_every == 0 or s == steps - 1):
                losses.append((s, float(self.loss.item())))
        if int(self.status.item()) != 0:
            raise _lib.AstroError("tensor-core wait timed out during training")
        return losses

    def forward(self, X):
        Y = torch.empty((X.shape[0], NOUT), dtype=torch.float32, device="cuda")
        _lib.check(self.L.astro_mlp_forward(rt.ptr(self.params), rt.ptr(X), rt.ptr(Y), X.shape[0],
                                            rt.ptr(self.status), rt.stream_handle()),
                   "astro_mlp_forward")
        return Y


def c2p_learned(engine, U, params, max_polish=2, listed=True, out=None):
    """Batch con2prim with the learned guess (params=None: Z = D + tau + B^2
    start).  listed: solve the states whose polish fails in a second kernel
    (else inline).  out: an optional preallocated [9,n] result.  Returns
    (primitives [9,n], stats dict)."""
    L = _lib.load()
    p = _lib.AstroParams()
    C.memmove(C.byref(p), C.byref(engine.p), C.sizeof(p))
    p.mlp = None if params is None else params.data_ptr()
    if out is None:
        out = torch.empty_like(U)
    stats = torch.zeros(8, dtype=torch.int64, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    nb = L.astro_c2p_learned_workspace_bytes(U.shape[1]) if listed else 0
    w = rt.workspace(nb, U.device) if listed else None
    _lib.check(L.astro_c2p_learned(C.byref(p), rt.ptr(U), rt.ptr(out), U.shape[1], int(max_polish),
                                   rt.ptr(w) if listed else None, nb, rt.ptr(stats),
                                   rt.ptr(status), rt.stream_handle()),
               "astro_c2p_learned")
    names = [f for f, _ in _lib.AstroC2PStats._fields_]
    st = dict(zip(names, stats.cpu().tolist()))
    st["status"] = int(status.item())
    return out, st


def save(flat, path=DATA, **meta):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez(path, params=np.asarray(flat, np.float32), **meta)


def load(path=DATA):
    d = np.load(path)
    return d["params"]
