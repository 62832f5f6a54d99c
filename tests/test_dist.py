"""Two-rank gloo tests (CPU) of the multi-process plumbing."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from hfscf_b200 import dist as D


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = D.max_over_ranks(1.5 + rank)
        items = D.shard(11, rank, world)
        q.put((rank, m, items))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_replica_shards_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    maxes = {r: m for r, m, _ in out}
    assert maxes == {0: 2.5, 1: 2.5}
    items = sorted(i for _, _, its in out for i in its)
    assert items == list(range(11))


def test_without_process_group_is_identity():
    assert D.max_over_ranks(3.25) == 3.25
    assert D.shard(5, 0, 1) == [0, 1, 2, 3, 4]


class _PartEngine:
    """Stand-in for a partitioned engine on the host: part p of nparts returns the oracle's
    J, K and two-electron gradient times the mask of the packed-index entries dealt to it, so
    that only the sum over the parts is the whole."""

    def __init__(self, bs):
        import numpy as np
        import oracle
        self.bs = bs
        self.eri = oracle.eri_packed(bs)
        self.part, self.nparts = 0, 1
        n = bs.nbf
        self.idx = (np.arange(n)[:, None] * 7 + np.arange(n)[None, :] * 3) % 5

    def set_partition(self, part, nparts):
        self.part, self.nparts = part, nparts

    def _mask(self, shape):
        import numpy as np
        m = (self.idx % self.nparts) == self.part
        return np.broadcast_to(m, shape)

    def jk(self, DJ, DKs, precision=None):
        import numpy as np
        import oracle
        J, K = oracle.jk(self.eri, DJ)
        return J * self._mask(J.shape), np.stack([K * self._mask(K.shape)])

    def grad2e(self, D, scale=1.0, precision=None):
        import numpy as np
        import oracle
        g = scale * oracle.grad2e_rhf(self.bs, D)
        w = (np.arange(g.size).reshape(g.shape) % self.nparts) == self.part
        return g * w

    def hess2e(self, D, scale=1.0):
        import numpy as np
        import oracle
        hc, he = oracle.ref_hess2e(self.bs, D)
        Hm = scale * (hc + he)
        w = (np.arange(Hm.size).reshape(Hm.shape) % self.nparts) == self.part
        return Hm * w

    def one_electron_grad(self, D, Q, cD, cQ):
        import oracle
        return oracle.ref_onee_grad(self.bs, D, Q, cD, cQ)


def _sharded_worker(rank, world, port, q):
    import numpy as np
    import torch.distributed as dist
    import oracle
    from hfscf_b200 import basis as B
    from hfscf_b200 import molecules as M
    from hfscf_b200 import scf
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        Z, x, name, pure = M.workload(1)
        bs = B.build_basis(name, Z, x, pure=pure)
        S, T, V = oracle.ref_onee(bs)
        fk = D.ShardedFock(_PartEngine(bs))
        res = scf.rhf(bs, fock=fk, H=T + V, S=S)
        g = D.sharded_rhf_gradient(bs, res, fk)
        h = fk.hess2e(res.D)
        q.put((rank, res.energy, res.iterations, g, h))
    finally:
        dist.destroy_process_group()


def test_partitioned_scf_and_gradient_sum_the_parts_over_two_gloo_ranks():
    """One molecule's Fock build, two-electron gradient and two-electron Hessian split over two
    ranks (each rank's engine returns only its part), summed by ShardedFock's all-reduce: both
    ranks run the same SCF and get the energy, gradient and Hessian of the unpartitioned oracle
    run."""
    import numpy as np
    import oracle
    from hfscf_b200 import basis as B
    from hfscf_b200 import molecules as M
    from hfscf_b200 import scf
    if not oracle.ref_available():
        pytest.skip("reference library not built here")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    Z, x, name, pure = M.workload(1)
    bs = B.build_basis(name, Z, x, pure=pure)
    S, T, V = oracle.ref_onee(bs)
    whole = _PartEngine(bs)
    ref = scf.rhf(bs, fock=lambda Dm, H: H + 2.0 * whole.jk(Dm, [Dm])[0] - whole.jk(Dm, [Dm])[1][0], H=T + V, S=S)
    gref = scf.rhf_gradient(bs, ref, whole)
    href = whole.hess2e(ref.D)
    for _, e, it, g, h in out:
        assert abs(e - ref.energy) < 1e-10
        assert it == ref.iterations
        assert np.max(np.abs(g - gref)) < 1e-10
        assert np.max(np.abs(h - href)) < 1e-10  # the two-electron Hessian's parts summed too
