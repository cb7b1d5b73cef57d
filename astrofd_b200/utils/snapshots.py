"""NPZ snapshots and checkpoints of primitive blocks in the reference
driver's format, written from device blocks without stalling the step loop.

Formats (solvers/srhd3d_mpi_muscl.py):
* snapshot ``jet3d_rank{rank:04d}_step{step:06d}.npz`` (:332-389): rho, vx,
  vy, vz, p; for hydro/GRHD blocks with TRACER_OFFSET > 5 also the
  Israel-Stewart fields pi, pixx, piyy, pizz, pixy, pixz, piyz, qx, qy, qz;
  for RMHD/GRMHD Bx, By, Bz, psi; then the tracers by TRACER_NAMES (and
  ``tracer_names`` as an object array), Te and Ti, the chemistry fractions by
  CHEM_NAMES; ``meta`` = [dx, dy, dz, t] and a ``comment`` string.  Whole
  blocks, ghosts included.
* checkpoint ``checkpoint_rank{rank:04d}_step{step:06d}.npz`` (:420-428):
  ``prim`` (the block), ``meta`` = [dx, dy, dz, t, step], ``comment``.
* ``load_checkpoint`` (:192-200): (pr, t, step), (pr, 0.0, 0) when meta is
  missing or short.

Field offsets follow utils/settings.py:246-256 (TRACER_OFFSET, THERMO_OFFSET,
CHEM_OFFSET) with the driver's defaults (solvers/srhd3d_mpi_muscl.py:77-85).

``SnapshotWriter`` takes CUDA tensors: the block is copied device to device
into a staging buffer in HBM on the caller's stream (a 1.6 GB 256^3 RMHD
block in well under a millisecond), then to pinned host memory on a side
stream, and a background thread writes the file; the caller's stream only
orders the staging copy, so the following steps overlap the host copy and
the file write.  ``wait()`` returns when every file is on disk.  numpy
blocks are written directly.
"""
import os
import threading

import numpy as np
import torch

IS_FIELDS = ("pi", "pixx", "piyy", "pizz", "pixy", "pixz", "piyz", "qx", "qy", "qz")
CHEM_NAMES = ["xHII", "xHeII", "xHeIII"]


def _layout(settings):
    s = settings or {}
    n_tr = int(s.get("N_TRACERS", 0))
    tr_off = int(s.get("TRACER_OFFSET", 5))
    n_th = int(s.get("N_THERMO", 0))
    th_off = int(s.get("THERMO_OFFSET", tr_off + n_tr))
    n_ch = int(s.get("N_CHEM", 0))
    ch_off = int(s.get("CHEM_OFFSET", th_off + n_th))
    return dict(n_tr=n_tr, tr_off=tr_off, names=list(s.get("TRACER_NAMES", None) or []),
                n_th=n_th, th_off=th_off, n_ch=n_ch, ch_off=ch_off,
                ch_names=list(s.get("CHEM_NAMES", CHEM_NAMES)),
                physics=str(s.get("PHYSICS", "hydro")).lower())


def snapshot_fields(pr, dx, dy, dz, t, settings):
    """The arrays of one snapshot file, in the driver's order (views of the
    host block ``pr``)."""
    L = _layout(settings)
    out = dict(rho=pr[0], vx=pr[1], vy=pr[2], vz=pr[3], p=pr[4])
    hydro = L["physics"] in ("hydro", "grhd")
    if hydro and L["tr_off"] > 5:
        out.update({name: pr[5 + m] for m, name in enumerate(IS_FIELDS)})
    elif not hydro:
        out.update(Bx=pr[5], By=pr[6], Bz=pr[7], psi=pr[8])
    if L["n_tr"] > 0:
        for ti in range(L["n_tr"]):
            name = L["names"][ti] if ti < len(L["names"]) else f"tracer{ti}"
            out[name] = pr[L["tr_off"] + ti]
        out["tracer_names"] = np.array(L["names"], dtype=object)
    if L["n_th"] > 0:
        out["Te"] = pr[L["th_off"]]
        out["Ti"] = pr[L["th_off"] + 1]
    if L["n_ch"] > 0:
        for ci in range(L["n_ch"]):
            name = L["ch_names"][ci] if ci < len(L["ch_names"]) else f"chem{ci}"
            out[name] = pr[L["ch_off"] + ci]
    out["meta"] = np.array([dx, dy, dz, t], dtype=np.float64)
    out["comment"] = ("3D SRHD/GRHD block (with ghosts)." if hydro
                      else "3D RMHD/GRMHD block (with ghosts).")
    return out


def snapshot_path(run_dir, rank, step):
    return os.path.join(run_dir, f"jet3d_rank{rank:04d}_step{step:06d}.npz")


def checkpoint_path(run_dir, rank, step):
    return os.path.join(run_dir, f"checkpoint_rank{rank:04d}_step{step:06d}.npz")


def _save_snapshot(host, path, dx, dy, dz, t, settings):
    np.savez(path, **snapshot_fields(host, dx, dy, dz, t, settings))


def _save_checkpoint(host, path, dx, dy, dz, t, step):
    np.savez(path, prim=host, meta=np.array([dx, dy, dz, t, step], dtype=np.float64),
             comment="Checkpoint (with ghosts).")


def _host(pr):
    if isinstance(pr, torch.Tensor):
        return pr.detach().cpu().numpy()
    return np.asarray(pr)


def write_snapshot(pr, run_dir, rank, step, dx, dy, dz, t, settings):
    """Synchronous snapshot of a numpy block or CUDA tensor; returns the path."""
    path = snapshot_path(run_dir, rank, step)
    _save_snapshot(_host(pr), path, dx, dy, dz, t, settings)
    return path


def write_checkpoint(pr, run_dir, rank, step, dx, dy, dz, t):
    path = checkpoint_path(run_dir, rank, step)
    _save_checkpoint(_host(pr), path, dx, dy, dz, t, step)
    return path


def load_checkpoint(path, device=None):
    """(pr, t, step) as the driver's load_checkpoint; ``device`` (e.g.
    "cuda") returns the block as a float64 tensor there."""
    data = np.load(path)
    pr = data["prim"]
    meta = data["meta"] if "meta" in data.files else None
    if device is not None:
        pr = torch.from_numpy(np.ascontiguousarray(pr, dtype=np.float64)).to(device)
    if meta is None or len(meta) < 5:
        return pr, 0.0, 0
    return pr, float(meta[3]), int(meta[4])


class SnapshotWriter:
    """Snapshots and checkpoints of CUDA blocks overlapped with the steps
    that follow (one file in flight; a second request waits for the first)."""

    def __init__(self, device=None):
        self.device = (torch.device("cuda", torch.cuda.current_device()) if device is None
                       else torch.device(device))
        self.side = torch.cuda.Stream(self.device)
        self.stage = None
        self.pinned = None
        self.thread = None
        self.error = None

    def _buffers(self, t):
        if self.stage is None or self.stage.shape != t.shape:
            self.stage = torch.empty_like(t)
            self.pinned = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
        return self.stage, self.pinned

    def _submit(self, pr, save, *args):
        if not isinstance(pr, torch.Tensor) or not pr.is_cuda:
            save(np.asarray(_host(pr)), *args)
            return
        self.wait()
        stage, pinned = self._buffers(pr)
        main = torch.cuda.current_stream(pr.device)
        stage.copy_(pr)                       # ordered on the caller's stream
        self.side.wait_stream(main)
        with torch.cuda.stream(self.side):
            pinned.copy_(stage, non_blocking=True)
            done = torch.cuda.Event()
            done.record(self.side)

        def work():
            try:
                done.synchronize()
                save(pinned.numpy(), *args)
            except BaseException as e:  # reported by wait()
                self.error = e

        self.thread = threading.Thread(target=work, daemon=True)
        self.thread.start()

    def snapshot(self, pr, run_dir, rank, step, dx, dy, dz, t, settings):
        path = snapshot_path(run_dir, rank, step)
        self._submit(pr, _save_snapshot, path, dx, dy, dz, t, settings)
        return path

    def checkpoint(self, pr, run_dir, rank, step, dx, dy, dz, t):
        path = checkpoint_path(run_dir, rank, step)
        self._submit(pr, _save_checkpoint, path, dx, dy, dz, t, step)
        return path

    def wait(self):
        if self.thread is not None:
            self.thread.join()
            self.thread = None
        if self.error is not None:
            e, self.error = self.error, None
            raise e
