"""Replica parallelism across GPUs: one process per GPU, whole frame pairs (or whole requests) per
GPU, nothing exchanged on the data path.

Frame pairs are independent (multipass.rs:136-192 analyses one pair from its two frames alone),
so a run shards by pairs: a sequence of pairs is cut into contiguous ranges, one per rank, and a
request stream is dispatched to the least-loaded device. torch.distributed (NCCL on GPUs, gloo on
CPU) is used only to agree on timing (the maximum over ranks) and to gather run statistics.
"""
import os
from datetime import timedelta

__all__ = ["pair_range", "Ranks", "least_loaded", "MultiDeviceServer"]


def pair_range(n_pairs, rank, world):
    """Contiguous, balanced [start, stop) of `n_pairs` pairs for `rank` of `world` ranks; the first
    n_pairs % world ranks take one pair more. A stream of K+1 frames has K sequential pairs
    (i, i+1); the rank owning [start, stop) needs frames start .. stop inclusive."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError(f"rank {rank} of world {world}")
    if n_pairs < 0:
        raise ValueError("negative pair count")
    base, extra = divmod(n_pairs, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


class Ranks:
    """This process's place in a torchrun job (RANK, LOCAL_RANK, WORLD_SIZE, MASTER_* from the
    environment) with the few collectives a replica job needs. A single process (no WORLD_SIZE, or
    1) needs no process group and every collective is the identity."""

    def __init__(self, backend=None, timeout_s=300, device=None):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self._dist = None
        self._dev = device
        if self.world > 1:
            import torch.distributed as dist
            if not dist.is_initialized():
                kw = {"timeout": timedelta(seconds=timeout_s)}
                if backend == "nccl" and device is not None:
                    kw["device_id"] = device
                dist.init_process_group(backend or "gloo", **kw)
            self._dist = dist

    def _tensor(self, v):
        import torch
        dev = self._dev if (self._dev is not None and self._dist.get_backend() == "nccl") else "cpu"
        return torch.tensor([float(v)], dtype=torch.float64, device=dev)

    def barrier(self):
        if self._dist:
            self._dist.barrier()

    def max(self, v):
        """Maximum of `v` over ranks (a time: the job takes as long as its slowest rank)."""
        if not self._dist:
            return float(v)
        t = self._tensor(v)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v):
        if not self._dist:
            return float(v)
        t = self._tensor(v)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM)
        return float(t.item())

    def gather(self, obj):
        """Every rank's `obj`, in rank order (run statistics; small objects only)."""
        if not self._dist:
            return [obj]
        out = [None] * self.world
        self._dist.all_gather_object(out, obj)
        return out

    def close(self):
        if self._dist and self._dist.is_initialized():
            self._dist.barrier()
            self._dist.destroy_process_group()
        self._dist = None


def least_loaded(loads):
    """Index of the smallest load, the lowest index on ties."""
    if not loads:
        raise ValueError("no devices")
    best = 0
    for i, v in enumerate(loads):
        if v < loads[best]:
            best = i
    return best


class MultiDeviceServer:
    """One serving engine per device; each request goes whole to the device with the fewest bytes
    of input outstanding (least-loaded admission), so requests never cross devices.

    `make_server(device)` builds the per-device engine (PivServer by default); engines need
    submit(a, b, cfg, pre) -> ticket and wait(ticket) -> result."""

    def __init__(self, devices, make_server=None, **server_kw):
        if not devices:
            raise ValueError("no devices")
        if make_server is None:
            from .api import PivServer

            def make_server(d):
                return PivServer(device=d, **server_kw)
        self.devices = list(devices)
        self.servers = [make_server(d) for d in self.devices]
        self.load = [0] * len(self.devices)
        self._tickets = {}
        self._next = 1

    def submit(self, a, b, cfg=None, pre=None):
        i = least_loaded(self.load)
        cost = int(getattr(a, "nbytes", 0)) + int(getattr(b, "nbytes", 0))
        t = self.servers[i].submit(a, b, cfg, pre)
        self.load[i] += cost
        tid = self._next
        self._next += 1
        self._tickets[tid] = (i, t, cost)
        return tid

    def device_of(self, ticket):
        return self.devices[self._tickets[ticket][0]]

    def wait(self, ticket):
        i, t, cost = self._tickets.pop(ticket)
        try:
            return self.servers[i].wait(t)
        finally:
            self.load[i] -= cost

    def reserve(self, nbytes):
        """Grows every device's request pool by nbytes ahead of the load (PivServer.reserve);
        returns the bytes each pool holds afterwards, in device order."""
        return [s.reserve(nbytes) for s in self.servers]

    def close(self):
        for s in self.servers:
            close = getattr(s, "close", None)
            if close:
                close()
