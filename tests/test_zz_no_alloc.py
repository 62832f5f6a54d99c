"""The scratch-free gradient entry point (hfgpu_grad2e_device_noalloc).

It exists for callers that cannot allocate device memory while they run -- a
driver whose own pool allocator owns the device, or an optimisation/dynamics
loop that forbids allocation after start-up.  It must give the same two-electron
gradient as the allocating entry point, hfgpu_grad2e_device, call after call,
although every call reuses the same fixed scratch array left over from the
previous one.  This file is collected last so that a run stopping at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10  # the FP64 two-electron gradient tolerance used by the other parity tests
TOL_MIXED = 1e-6  # the mixed-precision gradient tolerance of the launch-form tests


def _case(workload, pure=None):
    from hfscf_b200 import basis as B
    from hfscf_b200 import molecules as M
    if workload == "ch4":
        Z, x = M.methane()
        x = np.asarray(x) * B.ANGSTROM_TO_BOHR + np.random.default_rng(3).normal(scale=0.05, size=(5, 3))
        return B.build_basis("cc-pvdz", Z, x, pure=True)
    Z, x, name, p = M.workload(workload)
    return B.build_basis(name, Z, x, pure=p if pure is None else pure)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", ["water-octamer-6-31g*", "methane-cc-pvdz"])
def test_noalloc_gradient_matches_allocating_entry_point_on_two_calls(case, precision):
    """Two calls in a row against hfgpu_grad2e_device at the same precision.  In mixed
    precision the FP32 part of every table-mode class reuses the same array as floats."""
    import torch

    from hfscf_b200 import engine as E
    bs = _case(4) if case.startswith("water") else _case("ch4")
    prec, tol = (E.FP64, TOL) if precision == "fp64" else (E.MIXED, TOL_MIXED)
    n = bs.nbf
    rng = np.random.default_rng(21)
    A = rng.normal(size=(n, n))
    D = (A + A.T) / n
    lib = E.lib()
    lib.hfgpu_noalloc_scratch_bytes.restype = ctypes.c_longlong
    assert lib.hfgpu_noalloc_scratch_bytes() == 32 << 20
    with E.Engine(bs, device=0) as eng:
        dev = torch.device("cuda", 0)
        Dd = torch.from_numpy(D).to(dev)
        ref = torch.zeros((bs.natoms, 3), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        eng.grad2e_device(Dd.data_ptr(), 2.0, 1, Dd.data_ptr(), 1.0, ref.data_ptr(), prec)
        torch.cuda.synchronize()
        g_ref = ref.cpu().numpy()
        for _ in range(2):
            out = torch.zeros((bs.natoms, 3), dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            rc = lib.hfgpu_grad2e_device_noalloc(eng.h, ctypes.c_void_p(Dd.data_ptr()), ctypes.c_double(2.0),
                                                 ctypes.c_int(1), ctypes.c_void_p(Dd.data_ptr()),
                                                 ctypes.c_double(1.0), ctypes.c_void_p(out.data_ptr()),
                                                 ctypes.c_int(prec))
            assert rc == 0, lib.hfgpu_last_error(eng.h)
            torch.cuda.synchronize()
            assert np.max(np.abs(out.cpu().numpy() - g_ref)) < tol
        assert torch.cuda.current_device() == 0


def test_noalloc_gradient_of_a_batched_handle():
    """A batched handle (one water hexamer and two single waters) through the scratch-free
    entry point: every molecule's block of the concatenated density is read at its own
    offset, as in hfgpu_batch_grad2e_device."""
    import torch

    from hfscf_b200 import basis as B
    from hfscf_b200 import batch
    from hfscf_b200 import engine as E
    from hfscf_b200 import molecules as M
    rng = np.random.default_rng(5)
    mols = []
    for k in (6, 1, 1):
        Z, x = M.water_cluster(k, 3.0, rng, 0.05)
        mols.append((np.asarray(Z), np.asarray(x) * B.ANGSTROM_TO_BOHR, "6-31g*", False))
    bases = batch.batch_bases(mols)
    be = batch.BatchEngine(bases)
    dev = torch.device("cuda", 0)
    blocks = []
    for b in bases:
        A = rng.normal(size=(b.nbf, b.nbf))
        blocks.append(((A + A.T) / b.nbf).ravel())
    D = torch.from_numpy(np.concatenate(blocks)).to(dev)
    natoms = sum(b.natoms for b in bases)
    ref = torch.zeros((natoms, 3), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    be.grad2e_device(D, ref)
    torch.cuda.synchronize()
    lib = E.lib()
    for _ in range(2):
        out = torch.zeros_like(ref)
        torch.cuda.synchronize()
        rc = lib.hfgpu_grad2e_device_noalloc(be.h, ctypes.c_void_p(D.data_ptr()), ctypes.c_double(2.0),
                                             ctypes.c_int(1), ctypes.c_void_p(D.data_ptr()), ctypes.c_double(1.0),
                                             ctypes.c_void_p(out.data_ptr()), ctypes.c_int(E.FP64))
        assert rc == 0, lib.hfgpu_last_error(be.h)
        torch.cuda.synchronize()
        assert np.max(np.abs(out.cpu().numpy() - ref.cpu().numpy())) < TOL
    be.close()
