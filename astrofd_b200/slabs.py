"""x-slab decomposition of a jet block over ranks, one process per GPU.

``decompose_x`` restates solvers/srhd3d_mpi_muscl.py:92-97 (near-equal
slabs, the first nx % size ranks one layer wider).  ``SlabDomain.exchange``
does what exchange_halos (solvers/srhd3d_mpi_muscl.py:103-123) does: the NG
ghost layers on each x side of a slab receive the neighbour's NG interior
layers next to it.  The reference's two blocking Sendrecv phases become one
batched isend/irecv round over torch.distributed (NCCL between GPUs, gloo
for CPU tensors); the result is the same.  The slabs are packed into
contiguous buffers in HBM (x is the outermost index, so each variable's
layers are one contiguous run) and unpacked into the ghosts after the round;
all of it is ordered on the caller's stream.

The driver exchanges once per step, before the boundary fills
(solvers/srhd3d_mpi_muscl.py:286-292): the ranks' later RK stages read ghost
values of the previous step, so a multi-rank run differs from a one-block
run near the slab faces, as the reference's does.  Only the first rank
applies the nozzle and only the last the +x outflow.  ``step_stagewise``
also exchanges the output of every RK stage but the last before the next
stage reads it; the ranks then compute exactly what one block would.
"""
import torch


def decompose_x(nx_glob, size, rank):
    """(count, offset, counts, offsets) of ``rank``'s slab of nx_glob cells."""
    counts = [nx_glob // size] * size
    for r in range(nx_glob % size):
        counts[r] += 1
    offsets = [0] * size
    for r in range(1, size):
        offsets[r] = offsets[r - 1] + counts[r - 1]
    return counts[rank], offsets[rank], counts, offsets


class SlabDomain:
    def __init__(self, nx_glob, ng, rank=None, size=None, group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        live = dist.is_available() and dist.is_initialized()
        self.rank = rank if rank is not None else (dist.get_rank(group) if live else 0)
        self.size = size if size is not None else (dist.get_world_size(group) if live else 1)
        self.ng = int(ng)
        self.nx, self.offset, self.counts, self.offsets = decompose_x(nx_glob, self.size,
                                                                      self.rank)
        self.left = self.rank - 1 if self.rank > 0 else None
        self.right = self.rank + 1 if self.rank + 1 < self.size else None
        self._bufs = None
        if self.size > 1 and self.nx < self.ng:
            raise ValueError(f"slab of {self.nx} cells is thinner than {self.ng} ghost layers")

    @property
    def first(self):
        return self.left is None

    @property
    def last(self):
        return self.right is None

    def _peer(self, r):
        return r if self.group is None else self.dist.get_global_rank(self.group, r)

    def _buffers(self, pr):
        shape = (pr.shape[0], self.ng) + tuple(pr.shape[2:])
        key = (shape, pr.dtype, pr.device)
        if self._bufs is None or self._bufs[0] != key:
            self._bufs = (key, [torch.empty(shape, dtype=pr.dtype, device=pr.device)
                                for _ in range(4)])
        return self._bufs[1]

    def step_stagewise(self, stage_fn, pr, out, bufs, rk_order):
        """One SSPRK step with a halo exchange after every stage but the last:
        stage_fn(pr, pr_stage, dst, stage) runs one stage (e.g. the drop-in
        cores' step_stage); bufs: two blocks like pr for the intermediate
        stages.  Returns out."""
        cur = pr
        for st in range(rk_order):
            dst = out if st == rk_order - 1 else bufs[st % 2]
            stage_fn(pr, cur, dst, st)
            if st < rk_order - 1:
                self.exchange(dst)
            cur = dst
        return out

    def exchange(self, pr):
        """Fill the x ghost layers of ``pr`` (in place) from the neighbours."""
        if self.left is None and self.right is None:
            return pr
        ng = self.ng
        sendL, recvL, sendR, recvR = self._buffers(pr)
        ops = []
        P2P = self.dist.P2POp
        if self.left is not None:
            sendL.copy_(pr[:, ng:2 * ng])
            ops += [P2P(self.dist.isend, sendL, self._peer(self.left), self.group),
                    P2P(self.dist.irecv, recvL, self._peer(self.left), self.group)]
        if self.right is not None:
            sendR.copy_(pr[:, -2 * ng:-ng])
            ops += [P2P(self.dist.isend, sendR, self._peer(self.right), self.group),
                    P2P(self.dist.irecv, recvR, self._peer(self.right), self.group)]
        for req in self.dist.batch_isend_irecv(ops):
            req.wait()
        if self.left is not None:
            pr[:, :ng].copy_(recvL)
        if self.right is not None:
            pr[:, -ng:].copy_(recvR)
        return pr
