"""One answer sharded across GPUs by sub-database.

The first dimension of the answer is independent per sub-database k < r
(reference twosteps.cpp:1527-1579: scan of sub-database k, then its giant
steps; then externalProduct per k, test-pir.cpp:113-114); only the packing tree
(packingRLWEs, answer.cpp:800-835) needs all r results.  So with G ranks (G a
power of two dividing r), rank g holds sub-databases [g r/G, (g+1) r/G),
repeats the query's baby steps (cheap, and it saves broadcasting the 8 MiB
rotated-query buffer), answers its sub-databases up to the external products,
and the r external products (64 KiB each, coefficient form) are gathered to
rank 0 -- the one collective of the path -- which runs the packing tree.

The compute backend is pluggable: :class:`GpuShard` runs on this process's
GPU through the C ABI; tests drive the same orchestration with other
backends.
"""
from __future__ import annotations

import numpy as np

from .native import N, Context


def shard_range(r: int, world: int, rank: int) -> tuple[int, int]:
    """Sub-databases [lo, hi) of `rank` among `world` ranks."""
    if world < 1 or r % world or (world & (world - 1)):
        raise ValueError("world must be a power of two dividing r")
    per = r // world
    return rank * per, (rank + 1) * per


class GpuShard:
    """A rank's share on its GPU: a context with the rank's sub-databases (for
    the first dimension and the external products) and, on rank 0, one with all
    r for the packing tree."""

    def __init__(self, datacrt, r: int, N1: int, world: int, rank: int, perms, keys: dict, device: int = 0):
        lo, hi = shard_range(r, world, rank)
        words = N * N // 2
        self.r, self.rank, self.local = r, rank, hi - lo
        self.ctx = Context(self.local, N1, device=device)
        self.ctx.upload_db(np.ascontiguousarray(datacrt[lo * words:hi * words]))
        self.ctx.upload_perms(perms)
        lv_local = self.local.bit_length() - 1
        self.ctx.upload_client(0, keys["baby"], keys["giant"], keys["packing"][:lv_local * 4 * 2 * N], keys["rgsw"])
        self.pack_ctx = None
        if rank == 0:
            self.pack_ctx = Context(r, N1, device=device)
            self.pack_ctx.upload_client(0, keys["baby"], keys["giant"], keys["packing"], keys["rgsw"])

    def local_ext(self, query) -> np.ndarray:
        """External products of this rank's sub-databases, [local][2][N] words."""
        first, _ = self.ctx.matrix_vector_mul(0, query)
        ext, _ = self.ctx.external_product(0, np.zeros_like(first), first)
        return ext.reshape(self.local, 2 * N)

    def pack(self, ext_all) -> np.ndarray:
        return self.pack_ctx.packing(0, np.ascontiguousarray(ext_all).reshape(-1))

    def close(self):
        self.ctx.close()
        if self.pack_ctx:
            self.pack_ctx.close()


class ShardedAnswer:
    """Orchestration: local share, one gather to rank 0, packing on rank 0.

    `gather(local) -> list of every rank's local array (rank order) on rank 0,
    None elsewhere` is the collective; `gather_torch` builds it from a
    torch.distributed process group."""

    def __init__(self, backend, r: int, world: int, rank: int, gather):
        self.backend, self.r, self.world, self.rank, self.gather = backend, r, world, rank, gather

    def answer(self, query):
        parts = self.gather(self.backend.local_ext(query))
        if self.rank != 0:
            return None
        ext_all = np.concatenate([np.asarray(p).reshape(-1, 2 * N) for p in parts])
        if ext_all.shape[0] != self.r:
            raise RuntimeError(f"gathered {ext_all.shape[0]} external products, expected {self.r}")
        return self.backend.pack(ext_all)


def gather_torch(group=None, device=None):
    """A gather to rank 0 over torch.distributed (gloo: CPU tensors; nccl: GPU)."""
    import torch
    import torch.distributed as dist

    def gather(local: np.ndarray):
        t = torch.from_numpy(np.ascontiguousarray(local).view(np.int64))
        if device is not None:
            t = t.to(device)
        rank, world = dist.get_rank(group), dist.get_world_size(group)
        out = [torch.empty_like(t) for _ in range(world)] if rank == 0 else None
        dist.gather(t, out, dst=0, group=group)
        if rank != 0:
            return None
        return [o.cpu().numpy().view(np.uint64) for o in out]
    return gather
