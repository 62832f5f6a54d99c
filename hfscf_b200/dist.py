"""Multi-process plumbing for the bench, the batched mode and the partitioned build (one
process per GPU).

Two ways to spread the two-electron path over ranks:
  * replicas: independent molecules (a batch) split across ranks with no data-path
    collective; only the max-over-ranks of the timed region is reduced;
  * one molecule partitioned (hfgpu_set_partition): every rank computes every world-th
    quartet of each class list, and the partial two-electron terms are summed with one
    all-reduce per build (n^2 doubles: G = 2J - K), per gradient (natoms x 3) or per
    two-electron Hessian (3 natoms x 3 natoms), the
    exchange step of the multi-GPU Fock build (the reference's build is one OpenMP loop on
    one host, hfscf_hf_solver.cpp:254-286).
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist


def _initialized() -> bool:
    return dist.is_available() and dist.is_initialized()


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a float over all ranks (identity without a process group)."""
    if not _initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(n_items: int, rank: int, world: int) -> list[int]:
    """Items of this rank when n_items independent objects are dealt round-robin."""
    return list(range(rank, n_items, world))


def allreduce_sum_(t: torch.Tensor) -> torch.Tensor:
    """In-place sum over ranks (identity without a process group).  The tensor must live where
    the backend wants it: on the rank's GPU for NCCL, on the host for gloo."""
    if _initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t


def rank_world() -> tuple[int, int]:
    if not _initialized():
        return 0, 1
    return dist.get_rank(), dist.get_world_size()


class ShardedFock:
    """RHF Fock build of one molecule partitioned over the ranks of the process group.

    ``engine`` computes this rank's share of J and K (its handle set to part = rank of
    nparts = world); ``__call__(D, H)`` returns F = H + sum over ranks of (2 J_r - K_r), the
    same matrix as the unpartitioned build up to FP64 summation order, on every rank.  The sum
    runs on ``device`` (the rank's GPU for NCCL; None = host tensors, for gloo)."""

    def __init__(self, engine, device=None, precision=None):
        self.engine = engine
        self.device = device
        self.precision = precision
        self.rank, self.world = rank_world()
        engine.set_partition(self.rank, self.world)

    def two_electron(self, D: np.ndarray) -> np.ndarray:
        kw = {} if self.precision is None else {"precision": self.precision}
        J, K = self.engine.jk(D, [D], **kw)
        G = torch.from_numpy(np.ascontiguousarray(2.0 * J - K[0]))
        if self.device is not None:
            G = G.to(self.device)
        return allreduce_sum_(G).cpu().numpy()

    def __call__(self, D: np.ndarray, H: np.ndarray) -> np.ndarray:
        return H + self.two_electron(D)

    def grad2e(self, D: np.ndarray, scale: float = 1.0) -> np.ndarray:
        """Two-electron RHF gradient, summed over the ranks' parts."""
        kw = {} if self.precision is None else {"precision": self.precision}
        g = torch.from_numpy(np.ascontiguousarray(self.engine.grad2e(D, scale, **kw)))
        if self.device is not None:
            g = g.to(self.device)
        return allreduce_sum_(g).cpu().numpy()

    def hess2e(self, D: np.ndarray, scale: float = 1.0) -> np.ndarray:
        """Two-electron RHF Hessian (3 natoms x 3 natoms), summed over the ranks' parts: one
        all-reduce of 9 natoms^2 doubles."""
        Hm = torch.from_numpy(np.ascontiguousarray(self.engine.hess2e(D, scale)))
        if self.device is not None:
            Hm = Hm.to(self.device)
        return allreduce_sum_(Hm).cpu().numpy()

    def close(self):
        self.engine.set_partition(0, 1)


def sharded_rhf_gradient(basis, res, fock: ShardedFock) -> np.ndarray:
    """Full RHF gradient with the two-electron term summed over the ranks' parts; the one-electron
    and nuclear terms are computed once per rank (every rank returns the same gradient)."""
    from .basis import nuclear_repulsion_gradient
    D, F = res.D, res.F
    Q = D @ F @ D
    g = fock.grad2e(D, 1.0)
    g += fock.engine.one_electron_grad(D, Q, 2.0, -2.0)
    g += nuclear_repulsion_gradient(basis.Z, basis.coords)
    return g
