"""Shared implementation behind the drop-in srhd_core / rmhd_core modules.

``Engine`` holds the configured parameters of one physics module (the
reference keeps them as Numba-frozen module globals, core/srhd_core.py:18-41,
core/rmhd_core.py:21-50; here they are a POD struct passed by value to every
kernel, so re-configuring takes effect immediately) and forwards array calls
to libastrofd_b200.so.
"""
import ctypes as C

import numpy as np
import torch

from .. import _lib, runtime as rt


class Engine:
    def __init__(self, physics):
        self.physics = physics
        self.nm = 5 if physics == _lib.SRHD else 9
        self.p = _lib.AstroParams()
        self.p.physics = physics
        self.p.gamma = 5.0 / 3.0
        self.p.srhd_gamma = 5.0 / 3.0
        self.p.p_max = 1.0
        self.p.v_max = 0.999
        self.p.glm_ch = 1.0
        self.p.glm_cp = 0.1
        self.p.passive_offset = 5 if physics == _lib.SRHD else 9
        self.p.flux_mode = _lib.FLUX_REFERENCE
        self.p.precision = _lib.PREC_FP64
        self.p.c2p_guess = _lib.GUESS_REFERENCE
        self.p.mlp = None
        self.net = None
        self.stats = None

    # -- learned con2prim network ------------------------------------------
    def set_network(self, params):
        """Device parameter block of the learned con2prim guess (float32,
        astro_mlp_param_bytes() bytes), or None."""
        if params is None:
            self.net, self.p.mlp = None, None
            return
        t = torch.as_tensor(params, dtype=torch.float32)
        if not t.is_cuda:
            t = t.cuda()
        t = t.contiguous()
        if t.numel() * 4 != _lib.load().astro_mlp_param_bytes():
            raise _lib.AstroError("network parameter block has the wrong size")
        self.net = t
        self.p.mlp = t.data_ptr()

    def _require_network(self):
        if self.p.c2p_guess == _lib.GUESS_LEARNED and self.net is None:
            from .. import learned_c2p
            import os
            if not os.path.exists(learned_c2p.DATA):
                raise _lib.AstroError("C2P_GUESS='learned' needs a trained network: "
                                      "set_c2p_network(...) or python -m astrofd_b200.train_c2p_mlp")
            self.set_network(learned_c2p.load())

    # -- configure() ------------------------------------------------------
    def configure(self, params):
        p = self.p
        g = lambda k, d: params.get(k, d)
        p.gamma = float(g("GAMMA", p.gamma))
        p.p_max = float(g("P_MAX", p.p_max))
        p.v_max = float(g("V_MAX", p.v_max))
        p.limiter = _lib.LIMITER.get(str(g("LIMITER", "mc")).lower(), 0)
        p.recon = _lib.RECON.get(str(g("RECON", "muscl")).lower(), 0)
        r = str(g("RIEMANN", "hlle")).lower()
        if self.physics == _lib.SRHD:
            p.riemann = 1 if r == "hllc" else 0
            # the reference's SRHD kernels take gamma as a default argument
            # bound at import (srhd_core.py:47,62,134): always 5/3 unless the
            # caller opts in to honouring GAMMA
            p.srhd_gamma = p.gamma if g("SRHD_HONOUR_GAMMA", False) else 5.0 / 3.0
        else:
            p.riemann = 2 if r == "hlld_full" else (1 if r == "hlld" else 0)
            p.glm_ch = float(g("GLM_CH", p.glm_ch))
            p.glm_cp = float(g("GLM_CP", p.glm_cp))
            p.resistive = 1 if g("RESISTIVE_ENABLED", bool(p.resistive)) else 0
            p.resistivity = float(g("RESISTIVITY", p.resistivity))
        p.n_passive = int(g("N_PASSIVE", p.n_passive))
        p.passive_offset = int(g("PASSIVE_OFFSET", p.passive_offset))
        fm = str(g("FLUX_MODE", "reference")).lower()
        p.flux_mode = _lib.FLUX_CONSERVATIVE if fm == "conservative" else _lib.FLUX_REFERENCE
        pm = str(g("PRECISION", "fp64")).lower()
        p.precision = _lib.PREC_MIXED if pm == "mixed" else _lib.PREC_FP64
        cg = str(g("C2P_GUESS", "reference")).lower()
        p.c2p_guess = _lib.GUESS_LEARNED if cg == "learned" else _lib.GUESS_REFERENCE
        # STAGE_KERNEL (no reference counterpart): "split" (per-direction face
        # passes + update, the default) or "fused" (one kernel per stage)
        sk = str(g("STAGE_KERNEL", "fused" if p.fused_stage else "split")).lower()
        p.fused_stage = 1 if sk == "fused" else 0

    # -- right-hand side --------------------------------------------------
    def rhs(self, pr, nx, ny, nz, dx, dy, dz):
        L = _lib.load()
        t, was_np = rt.to_device(pr)
        if tuple(t.shape[1:]) != (nx, ny, nz):
            raise _lib.AstroError("nx, ny, nz must be the ghost-inclusive block extents")
        grid = rt.grid_of(t, dx, dy, dz)
        out = torch.empty((self.nm + self.p.n_passive, nx, ny, nz), dtype=torch.float64,
                          device=t.device)
        nb = L.astro_rhs_workspace_bytes(C.byref(self.p), C.byref(grid))
        if nb == 0:
            _lib.check(-2 if t.shape[0] < self.nm else -4, "astro_rhs (configuration)")
        w = rt.workspace(nb, t.device)
        _lib.check(L.astro_rhs(C.byref(self.p), C.byref(grid), rt.ptr(t), rt.ptr(out),
                               rt.ptr(w), nb, rt.stream_handle(t.device)), "astro_rhs")
        return out.cpu().numpy() if was_np else out

    # -- one SSPRK step ---------------------------------------------------
    def step(self, pr, dx, dy, dz, dt, rk_order, out=None):
        L = _lib.load()
        t, was_np = rt.to_device(pr)
        grid = rt.grid_of(t, dx, dy, dz)
        if out is None:
            out = torch.empty_like(t)
        nb = L.astro_step_workspace_bytes(C.byref(self.p), C.byref(grid))
        if nb == 0:
            _lib.check(-4, "astro_step (configuration)")
        self._require_network()
        w = rt.workspace(nb, t.device)
        stats = self._stats_buffer(t.device)
        _lib.check(L.astro_step(C.byref(self.p), C.byref(grid), rt.ptr(t), rt.ptr(out),
                                float(dt), int(rk_order), rt.ptr(w), nb, rt.ptr(stats),
                                rt.stream_handle(t.device)), "astro_step")
        return out.cpu().numpy() if was_np else out

    # -- fixed-metric GR wrappers -------------------------------------------
    def rhs_gr(self, gr, pr, dx, dy, dz):
        L = _lib.load()
        t, was_np = rt.to_device(pr)
        grid = rt.grid_of(t, dx, dy, dz)
        nx, ny, nz = t.shape[1:]
        out = torch.empty((self.nm + self.p.n_passive, nx, ny, nz), dtype=torch.float64,
                          device=t.device)
        nb = L.astro_gr_workspace_bytes(C.byref(self.p), C.byref(grid), C.byref(gr), 0)
        if nb == 0:
            _lib.check(-4, "astro_rhs_gr (configuration)")
        w = rt.workspace(nb, t.device)
        _lib.check(L.astro_rhs_gr(C.byref(self.p), C.byref(grid), C.byref(gr), rt.ptr(t),
                                  rt.ptr(out), rt.ptr(w), nb, rt.stream_handle(t.device)),
                   "astro_rhs_gr")
        return out.cpu().numpy() if was_np else out

    def step_gr(self, gr, pr, dx, dy, dz, dt, rk_order, out=None):
        L = _lib.load()
        t, was_np = rt.to_device(pr)
        grid = rt.grid_of(t, dx, dy, dz)
        if out is None:
            out = torch.empty_like(t)
        nb = L.astro_gr_workspace_bytes(C.byref(self.p), C.byref(grid), C.byref(gr), 1)
        if nb == 0:
            _lib.check(-4, "astro_step_gr (configuration)")
        self._require_network()
        w = rt.workspace(nb, t.device)
        stats = self._stats_buffer(t.device)
        _lib.check(L.astro_step_gr(C.byref(self.p), C.byref(grid), C.byref(gr), rt.ptr(t),
                                   rt.ptr(out), float(dt), int(rk_order), rt.ptr(w), nb,
                                   rt.ptr(stats), rt.stream_handle(t.device)), "astro_step_gr")
        return out.cpu().numpy() if was_np else out

    def step_stage(self, pr_in, pr_stage, out, dx, dy, dz, dt, rk_order, stage):
        """Stage `stage` of the SSPRK step from pr_in (astro_step_stage): CUDA
        tensors only; the stages of one step run in order with no other step
        on this device in between (the conserved state stays in the cached
        workspace)."""
        L = _lib.load()
        for t in (pr_in, pr_stage, out):
            if not (isinstance(t, torch.Tensor) and t.is_cuda and t.is_contiguous()):
                raise _lib.AstroError("step_stage takes contiguous CUDA tensors")
        grid = rt.grid_of(pr_in, dx, dy, dz)
        nb = L.astro_step_workspace_bytes(C.byref(self.p), C.byref(grid))
        if nb == 0:
            _lib.check(-4, "astro_step_stage (configuration)")
        self._require_network()
        w = rt.workspace(nb, pr_in.device)
        stats = self._stats_buffer(pr_in.device)
        _lib.check(L.astro_step_stage(C.byref(self.p), C.byref(grid), rt.ptr(pr_in),
                                      rt.ptr(pr_stage), rt.ptr(out), float(dt), int(rk_order),
                                      int(stage), rt.ptr(w), nb, rt.ptr(stats),
                                      rt.stream_handle(pr_in.device)), "astro_step_stage")
        return out

    def step_profiled(self, pr, dx, dy, dz, dt, rk_order, out):
        """One step with per-kernel-class CUDA-event times (synchronises)."""
        L = _lib.load()
        grid = rt.grid_of(pr, dx, dy, dz)
        nb = L.astro_step_workspace_bytes(C.byref(self.p), C.byref(grid))
        self._require_network()
        w = rt.workspace(nb, pr.device)
        stats = self._stats_buffer(pr.device)
        times = _lib.AstroKernelTimes()
        _lib.check(L.astro_step_profiled(C.byref(self.p), C.byref(grid), rt.ptr(pr), rt.ptr(out),
                                         float(dt), int(rk_order), rt.ptr(w), nb, rt.ptr(stats),
                                         rt.stream_handle(pr.device), C.byref(times)),
                   "astro_step_profiled")
        return out, [times.ms[i] for i in range(5)], [times.launches[i] for i in range(5)]

    def _stats_buffer(self, device):
        if self.stats is None or self.stats.device != torch.device(device):
            self.stats = torch.zeros(8, dtype=torch.int64, device=device)
        return self.stats

    def c2p_stats(self, reset=False):
        """con2prim outcome counters accumulated since the last reset."""
        if self.stats is None:
            return {}
        v = self.stats.cpu().tolist()
        names = [f for f, _ in _lib.AstroC2PStats._fields_]
        if reset:
            self.stats.zero_()
        return dict(zip(names, v))

    # -- CFL ---------------------------------------------------------------
    def max_char_speed(self, pr, nx, ny, nz):
        L = _lib.load()
        t, _ = rt.to_device(pr)
        grid = rt.grid_of(t)
        out = torch.empty(1, dtype=torch.float64, device=t.device)
        _lib.check(L.astro_max_char_speed(C.byref(self.p), C.byref(grid), rt.ptr(t), rt.ptr(out),
                                          None, 0, rt.stream_handle(t.device)),
                   "astro_max_char_speed")
        return out

    # -- pointwise conversions ----------------------------------------------
    def p2c_array(self, q):
        L = _lib.load()
        t, was_np = rt.to_device(q)
        t = t.reshape(self.nm, t.numel() // self.nm).contiguous()
        out = torch.empty_like(t)
        _lib.check(L.astro_p2c(C.byref(self.p), rt.ptr(t), rt.ptr(out), t.shape[1],
                               rt.stream_handle(t.device)), "astro_p2c")
        return out.cpu().numpy() if was_np else out

    def c2p_array(self, U):
        L = _lib.load()
        t, was_np = rt.to_device(U)
        t = t.reshape(self.nm, t.numel() // self.nm).contiguous()
        out = torch.empty_like(t)
        stats = self._stats_buffer(t.device)
        _lib.check(L.astro_c2p(C.byref(self.p), rt.ptr(t), rt.ptr(out), t.shape[1],
                               rt.ptr(stats), rt.stream_handle(t.device)), "astro_c2p")
        return out.cpu().numpy() if was_np else out

    def scalar_convert(self, fn, values):
        """Scalar call (the reference's per-cell helpers): routed through the
        same device kernels on a one-element batch."""
        a = np.asarray(values, dtype=np.float64).reshape(self.nm, -1)
        if a.shape[1] != 1:
            return fn(a)
        res = fn(a)
        res = res.cpu().numpy() if isinstance(res, torch.Tensor) else res
        return tuple(float(x) for x in res[:, 0])
