"""The device J/K build enqueues without host synchronisation, so it captures in a CUDA graph.

With density screening on, how much of every quartet-list segment a build launches depends on
the density (its largest |D| decides which Schwarz-bound decades can survive).  Those counts
are computed on the device by the build itself, so a graph captured once serves any later
density: the replays below take a density whose screened prefix differs from the captured one
and must match eager builds of it (FP64, to 1e-11: the atomics add in a different order).
"""
import numpy as np
import pytest

from hfscf_b200 import basis as B
from hfscf_b200 import engine as E
from hfscf_b200 import molecules as M

pytestmark = pytest.mark.gpu


def _sym(rng, n, scale):
    A = rng.normal(size=(n, n))
    return scale * (A + A.T) / n


@pytest.mark.parametrize("form", [0, 2], ids=["thread-form", "staged-form"])
@pytest.mark.parametrize("precision", [E.FP64, E.MIXED], ids=["fp64", "mixed"])
def test_jk_device_replays_from_a_cuda_graph(precision, form):
    import torch
    Z, x = M.water_cluster(3, 2.9, np.random.default_rng(8), 0.1)
    bs = B.build_basis("6-31g*", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=False)
    n = bs.nbf
    rng = np.random.default_rng(9)
    dev = torch.device("cuda", 0)
    densities = [torch.from_numpy(_sym(rng, n, s)).to(dev) for s in (1.0, 1e-3, 1e-6)]
    stream = torch.cuda.Stream(dev)
    tol = 1e-11 if precision == E.FP64 else 1e-9
    with E.Engine(bs, device=0) as eng:
        sched = eng.get_schedule()
        sched[:, 3] = form
        eng.set_schedule(sched)
        eng.set_stream(stream.cuda_stream)
        Din = torch.zeros((n, n), dtype=torch.float64, device=dev)
        J = torch.zeros_like(Din)
        K = torch.zeros_like(Din)
        eager = []
        with torch.cuda.stream(stream):
            for D in densities:
                Din.copy_(D)
                eng.jk_device(Din.data_ptr(), 1, Din.data_ptr(), J.data_ptr(), K.data_ptr(), precision)
                eager.append((J.clone(), K.clone()))
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            eng.jk_device(Din.data_ptr(), 1, Din.data_ptr(), J.data_ptr(), K.data_ptr(), precision)
        for rep in range(2):
            for D, (J0, K0) in zip(densities, eager):
                with torch.cuda.stream(stream):
                    Din.copy_(D)
                    J.zero_()
                    K.zero_()
                    g.replay()
                torch.cuda.synchronize()
                scale = float(J0.abs().max())
                assert float((J - J0).abs().max()) <= tol * max(scale, 1.0)
                assert float((K - K0).abs().max()) <= tol * max(scale, 1.0)
        del g
        eng.set_stream(None)
