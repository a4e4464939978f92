"""CPU collectives for ViewParallelTrainer over a torch.distributed gloo group
(test infrastructure: the product exchange is multiview.CudaCollectives over
NCCL).  Buffers are float32 CPU tensors, which the oracle backend reads as
numpy arrays."""
from __future__ import annotations

import torch
import torch.distributed as dist


class TorchCollectives:
    def __init__(self, group=None):
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)

    def alloc(self, numel):
        return torch.zeros(int(numel), dtype=torch.float32)

    def view(self, buf, offset, numel):
        return buf[offset:offset + numel]

    def zero(self, buf):
        buf.zero_()

    def copy(self, dst, src):
        dst.copy_(src)

    def reduce_scatter(self, out, inp):
        dist.reduce_scatter_tensor(out, inp, op=dist.ReduceOp.SUM, group=self.group)

    def all_gather(self, out, inp):
        dist.all_gather_into_tensor(out, inp, group=self.group)

    def all_reduce_scalar(self, x):
        t = torch.tensor([x], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        return float(t.item())
