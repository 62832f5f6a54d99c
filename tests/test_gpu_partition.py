"""One molecule's J/K build and two-electron gradient split into parts (hfgpu_set_partition):
the parts run one after another on one GPU and their outputs are summed, as the all-reduce of a
multi-GPU build sums them.  The sum equals the unpartitioned output up to FP64 summation order
(1e-11) and the oracle (J/K 1e-10, gradient 1e-10), with and without density screening, in
mixed precision (each part computes the same quartets in FP32 as the whole build does) and with
each J/K kernel form forced; the Fock entry points, which add H, are refused on a partitioned
handle; the scratch-free gradient entry point honours the partition too."""
import ctypes

import numpy as np
import pytest

import oracle
from hfscf_b200 import basis as B
from hfscf_b200 import engine as E
from hfscf_b200 import molecules as M

pytestmark = pytest.mark.gpu

TOL_SUM = 1e-11
TOL_ORACLE = 1e-10


def _water4(pure=False, name="6-31g*"):
    Z, x = M.water_cluster(4, 2.9, np.random.default_rng(17), 0.1)
    return B.build_basis(name, Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=pure)


def _density(bs, seed=4):
    """A converged-looking density: the core guess, so that density screening has work to skip."""
    S, T, V = E.one_electron(bs)
    w, U = np.linalg.eigh(S)
    X = (U / np.sqrt(w)) @ U.T
    _, Cp = np.linalg.eigh(X.T @ (T + V) @ X)
    C = X @ Cp
    nocc = int(np.sum(bs.Z)) // 2
    D = C[:, :nocc] @ C[:, :nocc].T
    rng = np.random.default_rng(seed)
    A = rng.normal(scale=1e-3, size=D.shape)
    return D + (A + A.T)


def _parts_jk(eng, D, nparts, precision=E.FP64):
    J = np.zeros_like(D)
    K = np.zeros_like(D)
    for p in range(nparts):
        eng.set_partition(p, nparts)
        Jp, Kp = eng.jk(D, [D], precision)
        J += Jp
        K += Kp[0]
    eng.set_partition(0, 1)
    return J, K


@pytest.mark.parametrize("nparts", [2, 3, 7])
@pytest.mark.parametrize("density_tol", [0.0, 1e-12])
def test_partitioned_jk_sums_to_the_whole_build(nparts, density_tol):
    bs = _water4()
    D = _density(bs)
    eri = oracle.eri_packed(bs)
    J0, K0 = oracle.jk(eri, D)
    with E.Engine(bs, density_tol=density_tol) as eng:
        Jw, Kw = eng.jk(D, [D])
        J, K = _parts_jk(eng, D, nparts)
    assert np.max(np.abs(J - Jw)) < TOL_SUM
    assert np.max(np.abs(K - Kw[0])) < TOL_SUM
    assert np.max(np.abs(J - J0)) < TOL_ORACLE
    assert np.max(np.abs(K - K0)) < TOL_ORACLE


def test_partitioned_jk_in_a_pure_basis_and_mixed_precision():
    bs = _water4(pure=True, name="cc-pvdz")
    D = _density(bs)
    with E.Engine(bs) as eng:
        for prec in (E.FP64, E.MIXED):
            Jw, Kw = eng.jk(D, [D], prec)
            J, K = _parts_jk(eng, D, 4, prec)
            assert np.max(np.abs(J - Jw)) < TOL_SUM
            assert np.max(np.abs(K - Kw[0])) < TOL_SUM


# Schedules forcing one J/K form for every class that has it: thread form (plain), the
# primitive-split form with 8 lanes, the warp-per-quartet and block-per-quartet forms, the staged
# persistent form and the low-residency form (the grids of all of them are sized from the part's
# share).
FORCED = {"thread": (64, 0, 0, 0), "primwarp8": (128, 8, 0, 0), "warp": (64, 0, 1, 0), "block": (64, 0, 2, 0),
          "staged": (64, 0, 0, 2), "lowres": (128, 0, 0, 3)}


@pytest.mark.parametrize("form", list(FORCED))
def test_partitioned_jk_under_every_kernel_form(form):
    bs = _water4()
    D = _density(bs)
    with E.Engine(bs) as eng:
        sched = np.tile(np.array(FORCED[form], dtype=np.int32), (E.NUM_CLASSES, 1))
        eng.set_schedule(sched)
        Jw, Kw = eng.jk(D, [D])
        J, K = _parts_jk(eng, D, 3)
    assert np.max(np.abs(J - Jw)) < TOL_SUM
    assert np.max(np.abs(K - Kw[0])) < TOL_SUM


@pytest.mark.parametrize("forms", ["thread", "warp", "split", "block"])
def test_partitioned_gradient_sums_to_the_whole(forms):
    bs = _water4()
    D = _density(bs)
    g0 = oracle.grad2e_rhf(bs, D)
    with E.Engine(bs) as eng:
        eng.set_grad_forms({"thread": 0, "warp": 1, "split": 2, "block": 4}[forms])
        gw = eng.grad2e(D, 1.0)
        g = np.zeros_like(gw)
        for p in range(3):
            eng.set_partition(p, 3)
            g += eng.grad2e(D, 1.0)
        eng.set_partition(0, 1)
    assert np.max(np.abs(g - gw)) < TOL_SUM
    assert np.max(np.abs(g - g0)) < TOL_ORACLE


def test_partitioned_noalloc_gradient_sums_to_the_whole():
    import torch
    bs = _water4()
    D = _density(bs)
    lib = E.lib()
    with E.Engine(bs) as eng:
        gw = eng.grad2e(D, 1.0)
        dev = torch.device("cuda", 0)
        Dd = torch.from_numpy(D).to(dev)
        tot = torch.zeros((bs.natoms, 3), dtype=torch.float64, device=dev)
        for p in range(2):
            eng.set_partition(p, 2)
            rc = lib.hfgpu_grad2e_device_noalloc(eng.h, ctypes.c_void_p(Dd.data_ptr()), ctypes.c_double(2.0),
                                                 ctypes.c_int(1), ctypes.c_void_p(Dd.data_ptr()),
                                                 ctypes.c_double(1.0), ctypes.c_void_p(tot.data_ptr()),
                                                 ctypes.c_int(E.FP64))
            assert rc == 0, lib.hfgpu_last_error(eng.h)
        torch.cuda.synchronize()
        eng.set_partition(0, 1)
    # grad2e(D, 1) is the RHF two-electron gradient; the device entry point with cJ = 2, cK = 1
    # accumulates the same quantity
    assert np.max(np.abs(tot.cpu().numpy() - gw)) < TOL_SUM


def test_fock_entry_points_are_refused_on_a_partitioned_handle_and_bad_partitions_rejected():
    bs = _water4()
    D = _density(bs)
    S, T, V = E.one_electron(bs)
    H = T + V
    with E.Engine(bs) as eng:
        eng.set_partition(1, 2)
        with pytest.raises(E.HfgpuError) as ei:
            eng.fock_rhf(D, H)
        assert ei.value.code == 4
        with pytest.raises(E.HfgpuError) as ei:
            eng.fock_delta(D, H)
        assert ei.value.code == 4
        for part, nparts in ((2, 2), (-1, 2), (0, 0)):
            with pytest.raises(E.HfgpuError) as ei:
                eng.set_partition(part, nparts)
            assert ei.value.code == 1
        eng.set_partition(0, 1)
        F = eng.fock_rhf(D, H)  # usable again, whole build
        J, K = oracle.jk(oracle.eri_packed(bs), D)
        assert np.max(np.abs(F - (H + 2.0 * J - K))) < TOL_ORACLE


@pytest.mark.parametrize("form", [-1, 0, 1, 2, 3], ids=["default", "thread", "block", "warp", "line"])
def test_partitioned_hessian_sums_to_the_whole(form):
    """The two-electron Hessian honours the partition: its parts, summed as an all-reduce of the
    3 natoms x 3 natoms blocks would sum them, equal the whole Hessian (1e-11) in every form."""
    Z, x = M.water_cluster(2, 2.9, np.random.default_rng(17), 0.1)
    bs = B.build_basis("6-31g*", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=False)
    D = _density(bs)
    with E.Engine(bs, density_tol=0.0) as eng:
        eng.set_hess_form(form)
        H = eng.hess2e(D)
        Hs = np.zeros_like(H)
        for p in range(3):
            eng.set_partition(p, 3)
            Hs += eng.hess2e(D)
        eng.set_partition(0, 1)
    assert np.max(np.abs(Hs - H)) < TOL_SUM
    assert np.max(np.abs(H)) > 1e-3
