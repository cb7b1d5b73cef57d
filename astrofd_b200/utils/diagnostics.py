"""Drop-in replacement of AstroFD's utils/diagnostics.py: run diagnostics
of a primitive block on the device.

``compute_diagnostics_and_write`` (utils/diagnostics.py:5): max Lorentz
factor over the interior (v^2 >= 1 taken as 1 - 1e-14) and the inlet flux
sum dy dz S_x over the first interior x layer, S_x from prim_to_cons.
``compute_centerline_and_write`` (utils/diagnostics.py:59): Gamma, rho, p and
v_x along x at the middle interior y and z (v capped at V_MAX as the
reference does).  ``compute_divb_and_write`` (utils/diagnostics.py:128):
max, rms and mean of the central-difference div B over the interior.  Same
arguments, return values and CSV files (diagnostics.csv, centerline.csv,
divb.csv, appended, header on creation) as the reference.

The reductions are one device kernel (astro_diagnostics) and one 48-byte
copy back; the centreline is 5 x nx values copied back.  ``pr`` is a float64
CUDA tensor (a numpy block is copied to the device first).

``comm`` is the reference's mpi4py communicator (the driver passes
MPI.COMM_WORLD; reductions then use MPI.MAX / MPI.SUM, as
utils/diagnostics.py:28,44 do), None for one process, or any other object
with ``allreduce(value, op)`` (op ``MAX`` or ``SUM`` of this module) and
``gather(obj, root=0)``; ``TorchComm`` is that object over
torch.distributed.  As in the reference, only rank 0 adds the inlet
plane (it holds the x = 0 slab) and writes the files.

The reference calls prim_to_cons without an adiabatic index, so the module
default 5/3 of core/srhd_core.py:47 and core/rmhd_core.py:138 applies
whatever GAMMA is configured; that is kept (``INLET_GAMMA``).  The V_MAX and
P_MAX caps of the RMHD prim_to_cons are the configured ones (the
rmhd_core engine's).
"""
import math
import os

import numpy as np
import torch

from .. import _lib, runtime as rt

MAX, SUM = "max", "sum"
INLET_GAMMA = 5.0 / 3.0


class TorchComm:
    """The allreduce / gather subset of an mpi4py communicator over a
    torch.distributed process group (any backend; values travel as float64
    host tensors for gloo, device tensors for nccl)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)

    def _device(self):
        if self.dist.get_backend(self.group) == "nccl":
            return torch.device("cuda", torch.cuda.current_device())
        return torch.device("cpu")

    def allreduce(self, value, op=SUM):
        t = torch.tensor([float(value)], dtype=torch.float64, device=self._device())
        rop = self.dist.ReduceOp.MAX if op == MAX else self.dist.ReduceOp.SUM
        self.dist.all_reduce(t, op=rop, group=self.group)
        return float(t.item())

    def gather(self, obj, root=0):
        out = [None] * self.size
        self.dist.all_gather_object(out, obj, group=self.group)
        return out if self.rank == root else None


def _comm_op(comm, op):
    """``op`` in the communicator's own vocabulary: mpi4py's MPI.MAX /
    MPI.SUM for an mpi4py communicator, this module's strings otherwise."""
    if type(comm).__module__.split(".")[0] == "mpi4py":
        import sys
        mpi = sys.modules.get("mpi4py.MPI")
        if mpi is None:
            from mpi4py import MPI as mpi
        return mpi.MAX if op == MAX else mpi.SUM
    return op


def _allreduce(comm, value, op):
    return value if comm is None else comm.allreduce(value, op=_comm_op(comm, op))


def _gather(comm, obj):
    return [obj] if comm is None else comm.gather(obj, root=0)


def _block(pr):
    if isinstance(pr, torch.Tensor):
        t, _ = rt.to_device(pr)
        if not t.is_contiguous():
            raise _lib.AstroError("primitive tensor must be contiguous")
        return t
    return rt.to_device(pr)[0]


def device_reductions(pr, dx, dy, dz, NG, is_rmhd, gamma=INLET_GAMMA):
    """One launch of astro_diagnostics: dict with max_gamma, inlet_sx (sum
    of S_x over the first interior x layer, without dy dz), divb_max,
    divb_sum, divb_sumsq and divb_n (zero when the block has < 8 variables)."""
    from ..core import rmhd_core, srhd_core
    L = _lib.load()
    t = _block(pr)
    eng = (rmhd_core if is_rmhd else srhd_core).engine()
    p = _lib.AstroParams.from_buffer_copy(eng.p)
    p.physics = _lib.RMHD if is_rmhd else _lib.SRHD
    out = torch.empty(6, dtype=torch.float64, device=t.device)
    g = rt.grid_of(t, dx, dy, dz)
    _lib.check(L.astro_diagnostics(p, g, int(NG), rt.ptr(t), float(gamma), rt.ptr(out),
                                   rt.stream_handle(t.device)), "astro_diagnostics")
    v = out.cpu().numpy()
    return dict(max_gamma=float(v[0]), inlet_sx=float(v[1]), divb_max=float(v[2]),
                divb_sum=float(v[3]), divb_sumsq=float(v[4]), divb_n=int(round(v[5])))


def _append(path, header, lines):
    new = not os.path.exists(path)
    with open(path, "a") as f:
        if new:
            f.write(header)
        f.writelines(lines)


def compute_diagnostics_and_write(pr, dx, dy, dz, offs_x, counts, comm, rank, step, t, dt,
                                  amax, run_dir, prim_to_cons, NG, is_rmhd=False):
    """Global max Gamma and inlet flux; appends a row to diagnostics.csv on
    rank 0 and returns (max Gamma, signed flux, |flux|).  ``prim_to_cons``
    is accepted for the reference's signature; the device computes S_x with
    the SRHD or RMHD prim_to_cons by ``is_rmhd``, adiabatic index 5/3."""
    r = device_reductions(pr, dx, dy, dz, NG, is_rmhd)
    global_maxG = _allreduce(comm, r["max_gamma"], MAX)
    inlet_flux = r["inlet_sx"] * dy * dz if rank == 0 else 0.0
    total = _allreduce(comm, inlet_flux, SUM)
    signed_flux, abs_flux = total, abs(total)
    if rank == 0:
        _append(os.path.join(run_dir, "diagnostics.csv"),
                "step,time,dt,amax,maxGamma,inletFlux_signed,inletFlux_abs\n",
                [f"{step},{t:.8e},{dt:.8e},{amax:.6e},{global_maxG:.6e},"
                 f"{signed_flux:.6e},{abs_flux:.6e}\n"])
    return global_maxG, signed_flux, abs_flux


def centerline(pr, V_MAX, NG):
    """(Gamma, rho, p, vx) along the interior x at the middle interior y, z
    of this block (utils/diagnostics.py:72-99)."""
    t = _block(pr)
    nx, ny, nz = (int(s) - 2 * NG for s in t.shape[1:])
    j, k = NG + ny // 2, NG + nz // 2
    line = t[:5, NG:NG + nx, j, k].cpu().numpy()
    rho, vx, vy, vz, p = (line[v].copy() for v in range(5))
    v2 = vx * vx + vy * vy + vz * vz
    vmax2 = V_MAX * V_MAX
    mask = v2 >= vmax2
    if np.any(mask):
        fac = V_MAX / np.sqrt(v2[mask] + 1e-32)
        vx[mask] *= fac
        vy[mask] *= fac
        vz[mask] *= fac
        v2[mask] = vmax2 - 1e-14
    G = 1.0 / np.sqrt(1.0 - np.clip(v2, 0, 1 - 1e-14))
    return G, rho, p, vx


def compute_centerline_and_write(pr, dx, dy, dz, offs_x, counts, comm, rank, step, t, run_dir,
                                 V_MAX, NG):
    """Appends the gathered centreline (rank order) to centerline.csv on
    rank 0; i runs from 0 over the gathered cells and x = (i + 1/2) dx, as
    in the reference."""
    G, rho, p, vx = centerline(pr, V_MAX, NG)
    parts = _gather(comm, (G, rho, p, vx))
    if rank != 0 or parts is None:
        return
    G, rho, p, vx = (np.concatenate([q[m] for q in parts]) for m in range(4))
    lines = []
    for ii in range(G.size):
        x = (ii + 0.5) * dx
        lines.append(f"{step},{t:.8e},{ii},{x:.8e},{G[ii]:.8e},{rho[ii]:.8e},"
                     f"{p[ii]:.8e},{vx[ii]:.8e}\n")
    _append(os.path.join(run_dir, "centerline.csv"), "step,time,i,x,Gamma,rho,p,vx\n", lines)


def compute_divb_and_write(pr, dx, dy, dz, offs_x, counts, comm, rank, step, t, run_dir, NG):
    """(max |div B|, rms, mean) over all ranks' interiors, appended to
    divb.csv on rank 0; (None, None, None) for blocks of fewer than 8
    variables."""
    if pr.shape[0] < 8:
        return None, None, None
    r = device_reductions(pr, dx, dy, dz, NG, pr.shape[0] >= 9)
    gmax = _allreduce(comm, r["divb_max"], MAX)
    gsum = _allreduce(comm, r["divb_sum"], SUM)
    gsq = _allreduce(comm, r["divb_sumsq"], SUM)
    gn = _allreduce(comm, r["divb_n"], SUM)
    if gn > 0:
        mean, rms = gsum / gn, math.sqrt(gsq / gn)
    else:
        mean = rms = 0.0
    if rank == 0:
        _append(os.path.join(run_dir, "divb.csv"), "step,time,divB_max,divB_rms,divB_mean\n",
                [f"{step},{t:.8e},{gmax:.6e},{rms:.6e},{mean:.6e}\n"])
    return gmax, rms, mean
