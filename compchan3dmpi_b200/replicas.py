"""One process per GPU, independent replicas ("replicas only").

Every rank integrates its own copy of the workload on its own GPU.  No
field data crosses GPUs: the only collectives are a barrier around the
timed region and a max-over-ranks of the device time.  The reference's 3D
MPI decomposition (v1.9/codes/main_v1.9.f90:84-137) is not reproduced,
because a production grid fits in one B200.

Works with the ``gloo`` backend on CPU (tests) and ``nccl`` on GPUs.
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from datetime import timedelta


@dataclass
class Ranks:
    rank: int = 0
    world: int = 1
    local_rank: int = 0
    backend: str | None = None

    @property
    def is_root(self) -> bool:
        return self.rank == 0


def from_env() -> Ranks:
    return Ranks(rank=int(os.environ.get("RANK", "0")), world=int(os.environ.get("WORLD_SIZE", "1")),
                 local_rank=int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: float = 120.0) -> Ranks:
    """Join the process group when WORLD_SIZE > 1 (addresses from the env)."""
    r = from_env()
    if r.world > 1:
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        if backend == "nccl":
            import torch
            torch.cuda.set_device(r.local_rank)
            dist.init_process_group("nccl", timeout=timedelta(seconds=timeout_s),
                                    device_id=torch.device("cuda", r.local_rank))
        else:
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
        r.backend = backend
    return r


def barrier(r: Ranks):
    if r.world > 1:
        import torch.distributed as dist
        if r.backend == "nccl":
            import torch
            dist.barrier(device_ids=[r.local_rank])
        else:
            dist.barrier()


def max_over_ranks(r: Ranks, x: float) -> float:
    return _reduce(r, x, "max")


def sum_over_ranks(r: Ranks, x: float) -> float:
    return _reduce(r, x, "sum")


def _reduce(r: Ranks, x: float, op: str) -> float:
    if r.world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    dev = torch.device("cuda", r.local_rank) if r.backend == "nccl" else torch.device("cpu")
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def finalize(r: Ranks):
    if r.world > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
