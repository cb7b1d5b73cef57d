"""Device plumbing shared by the drop-in modules: host/device dispatch, the
caller-owned workspace cache and stream handles.

Arrays handed to the public API may be numpy float64 blocks (the reference's
own type) or torch float64 CUDA tensors.  numpy inputs are uploaded, computed
on the GPU and copied back, so a reference driver keeps working unchanged;
torch CUDA tensors stay resident and the call is stream-ordered.  Nothing here
computes on the CPU.
"""
import ctypes as C

import numpy as np
import torch

from . import _lib

_work = {}


def require_cuda():
    if not torch.cuda.is_available():
        raise _lib.AstroError("astrofd_b200 needs a CUDA device (B200); no CPU fallback")


def stream_handle(device=None):
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def workspace(nbytes, device):
    """A cached uint8 device buffer of at least nbytes on device."""
    key = torch.device(device).index
    buf = _work.get(key)
    if buf is None or buf.numel() < nbytes:
        buf = torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)
        _work[key] = buf
    return buf


def to_device(a):
    """(tensor on GPU, was_numpy).  float64, C-contiguous."""
    if isinstance(a, torch.Tensor):
        if not a.is_cuda:
            raise _lib.AstroError("torch tensors must be on a CUDA device")
        if a.dtype != torch.float64:
            raise _lib.AstroError("primitive blocks are float64")
        return a.contiguous(), False
    require_cuda()
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    return torch.from_numpy(arr).to("cuda", non_blocking=False), True


def ptr(t):
    return C.c_void_p(t.data_ptr())


def grid_of(t, dx=1.0, dy=1.0, dz=1.0):
    nv, nx, ny, nz = (int(s) for s in t.shape)
    return _lib.AstroGrid(nv, nx, ny, nz, float(dx), float(dy), float(dz))
