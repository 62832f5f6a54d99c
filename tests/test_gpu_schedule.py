"""Launch schedule and autotuner: every launch form of every quartet class gives the
oracle's ERIs, J and K, and an autotuned schedule changes nothing but speed.

Tolerances as in test_gpu_parity: ERIs 1e-11, J/K 1e-10 absolute (FP64).
"""
import numpy as np
import pytest

import oracle
from hfscf_b200 import basis as B
from hfscf_b200 import engine as E
from hfscf_b200 import molecules as M

pytestmark = pytest.mark.gpu

ERI_TOL = 1e-11
MAT_TOL = 1e-10


def _sym(rng, n):
    A = rng.normal(size=(n, n))
    return (A + A.T) / n


def _molecules():
    rng = np.random.default_rng(23)
    Z, x = M.water(rng)
    h2o = B.build_basis("6-31g**", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=False)
    Z, x = M.methane()
    x = np.asarray(x) * B.ANGSTROM_TO_BOHR + rng.normal(scale=0.05, size=(5, 3))
    ch4 = B.build_basis("cc-pvdz", Z, x, pure=True)
    return [("h2o-631gss-cart", h2o), ("ch4-ccpvdz-pure", ch4)]


MOLS = _molecules()
# (block, primwarp, warp, capped) applied to every class
# capped = 2: the persistent form with the Boys table staged in shared memory (classes of L <= 4)
FORMS = [(32, 0, 0, 0), (64, 1, 0, 1), (128, 0, 1, 0), (64, 1, 1, 0), (64, 4, 0, 1), (32, 8, 1, 1), (128, 16, 0, 0),
         (64, 0, 0, 2), (128, 4, 0, 2), (32, 0, 1, 2), (64, 0, 0, 3), (128, 0, -1, 3), (64, 0, 2, 0), (64, 8, 2, 0)]


@pytest.mark.parametrize("form", FORMS, ids=[f"b{f[0]}-pw{f[1]}-w{f[2]}-c{f[3]}" for f in FORMS])
@pytest.mark.parametrize("name,bs", MOLS, ids=[m[0] for m in MOLS])
def test_every_launch_form_matches_oracle(name, bs, form):
    rng = np.random.default_rng(29)
    D = _sym(rng, bs.nbf)
    eri0 = oracle.eri_packed(bs)
    J0, K0 = oracle.jk(eri0, D)
    with E.Engine(bs, density_tol=0.0) as eng:
        eng.set_schedule(np.tile(np.array(form, dtype=np.int32), (E.NUM_CLASSES, 1)))
        assert (eng.get_schedule() == np.array(form)).all()
        eri = eng.eri_packed()
        J, K = eng.jk(D, [D])
    assert np.max(np.abs(eri - eri0)) < ERI_TOL
    assert np.max(np.abs(J - J0)) < MAT_TOL and np.max(np.abs(K[0] - K0)) < MAT_TOL


def test_schwarz_factors_under_the_block_form():
    """The Schwarz pass of set_geometry runs the large classes through the scheduled form too; in
    the block-per-quartet form its per-pair maximum is reduced over the block's warps."""
    bs = MOLS[1][1]
    with E.Engine(bs) as eng0:
        q0 = eng0.schwarz()
    with E.Engine(bs) as eng:
        eng.set_schedule(np.tile(np.array((64, 0, 2, 0), dtype=np.int32), (E.NUM_CLASSES, 1)))
        eng.set_geometry(bs.coords)
        q1 = eng.schwarz()
    assert np.max(np.abs(q1 - q0)) < 1e-12


def test_set_schedule_rejects_bad_entries():
    bs = MOLS[0][1]
    with E.Engine(bs) as eng:
        before = eng.get_schedule()
        bad = before.copy()
        bad[3, 0] = 48
        with pytest.raises(E.HfgpuError):
            eng.set_schedule(bad)
        assert (eng.get_schedule() == before).all()


def test_autotuned_schedule_gives_the_same_fock_build():
    Z, x = M.water_cluster(2, 2.9, np.random.default_rng(31), 0.1)
    bs = B.build_basis("6-31g*", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=False)
    rng = np.random.default_rng(37)
    D = _sym(rng, bs.nbf)
    H = _sym(rng, bs.nbf)
    with E.Engine(bs) as eng:
        F0 = eng.fock_rhf(D, H)
        Fm0 = eng.fock_rhf(D, H, E.MIXED)
        sched = eng.autotune(D, repeats=2)
        assert sched.shape == (E.NUM_CLASSES, 4)
        assert set(np.unique(sched[:, 0])) <= {32, 64, 128}
        assert set(np.unique(sched[:, 1])) <= {0, 1, 4, 8, 16, 32} and set(np.unique(sched[:, 2])) <= {-1, 0, 1, 2}
        assert set(np.unique(sched[:, 3])) <= {0, 1, 2, 3}
        assert (eng.get_schedule() == sched).all()
        F1 = eng.fock_rhf(D, H)
        Fm1 = eng.fock_rhf(D, H, E.MIXED)
    assert np.max(np.abs(F1 - F0)) < 1e-11
    assert np.max(np.abs(Fm1 - Fm0)) < 1e-6


@pytest.mark.parametrize("gmax", [0, 48], ids=["thread-per-quartet", "block-per-quartet"])
@pytest.mark.parametrize("name,bs", MOLS, ids=[m[0] for m in MOLS])
def test_gradient_launch_forms_match_oracle(name, bs, gmax):
    """The default gradient form of the large classes under opts.grad_warp_max_waves: one thread
    per quartet (0) or one block of four warps per quartet (> 0), each in turn (FP64, tolerance
    1e-10 as in test_gpu_parity)."""
    rng = np.random.default_rng(31)
    D = _sym(rng, bs.nbf)
    g0 = oracle.grad2e_rhf(bs, D)
    with E.Engine(bs, grad_warp_max_waves=gmax) as eng:
        g = eng.grad2e(D)
        gm = eng.grad2e(D, precision=E.MIXED)
    assert np.max(np.abs(g - g0)) < 1e-10
    assert np.max(np.abs(gm - g0)) < 1e-6


@pytest.mark.parametrize("precision", [E.FP64, E.MIXED], ids=["fp64", "mixed"])
def test_staged_form_with_density_screening_matches_plain_form(precision):
    """The staged persistent form under density screening (the counts of its launches come
    from the device) gives the plain form's J and K."""
    Z, x = M.water_cluster(3, 2.9, np.random.default_rng(33), 0.1)
    bs = B.build_basis("6-31g*", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=False)
    rng = np.random.default_rng(35)
    D = 1e-3 * _sym(rng, bs.nbf)
    with E.Engine(bs) as eng:
        J0, K0 = eng.jk(D, [D], precision)
        sched = eng.get_schedule()
        sched[:, 3] = 2
        sched[:, 1] = 0
        eng.set_schedule(sched)
        J1, K1 = eng.jk(D, [D], precision)
    tol = 1e-12 if precision == E.FP64 else 1e-9
    assert np.max(np.abs(J1 - J0)) < tol and np.max(np.abs(K1[0] - K0[0])) < tol


def test_staging_wait_runs_out_and_reports():
    """Bounded wait of the shared-memory staging: with the barrier armed and no copy issued
    (the engine's wait test), every staged block gives up after its poll limit, records
    status 2 and skips its quartets; the host-pointer build fails with HFGPU_ERR_CUDA, the
    device build reports the status through hfgpu_device_status, and the context stays
    usable for a normal engine afterwards.  No fault, no hang."""
    import torch
    rng = np.random.default_rng(37)
    Z, x = M.water(rng)
    bs = B.build_basis("6-31g*", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=False)
    D = _sym(rng, bs.nbf)
    staged = np.tile(np.array((64, 0, 0, 2), dtype=np.int32), (E.NUM_CLASSES, 1))
    with E.Engine(bs, stage_wait_test=True) as eng:
        eng.set_schedule(staged)
        with pytest.raises(E.HfgpuError) as err:
            eng.jk(D, [D])
        assert err.value.code == 3 and "staging wait ran out" in str(err.value)
        assert eng.device_status() == 0  # the failing call read and cleared it
        dev = torch.device("cuda", 0)
        Dd = torch.from_numpy(D).to(dev)
        J = torch.zeros_like(Dd)
        K = torch.zeros_like(Dd)
        torch.cuda.synchronize()
        eng.jk_device(Dd.data_ptr(), 1, Dd.data_ptr(), J.data_ptr(), K.data_ptr())
        assert eng.device_status() == 2
        assert eng.device_status() == 0
    eri0 = oracle.eri_packed(bs)
    J0, K0 = oracle.jk(eri0, D)
    with E.Engine(bs, density_tol=0.0) as eng:
        eng.set_schedule(staged)
        J, K = eng.jk(D, [D])
        assert eng.device_status() == 0
    assert np.max(np.abs(J - J0)) < MAT_TOL and np.max(np.abs(K[0] - K0)) < MAT_TOL


def test_host_abort_flag_stops_persistent_builds():
    """hfgpu_request_abort: with the flag set, the persistent launches stop at their first chunk
    and record status 3 (the host-pointer build then fails with HFGPU_ERR_STATE, a device
    build reports it through hfgpu_device_status); after the flag is reset the same handle
    builds the full J and K again."""
    import torch
    Z, x = M.water_cluster(3, 2.9, np.random.default_rng(39), 0.1)
    bs = B.build_basis("6-31g*", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=False)
    rng = np.random.default_rng(41)
    D = _sym(rng, bs.nbf)
    staged = np.tile(np.array((64, 0, 0, 2), dtype=np.int32), (E.NUM_CLASSES, 1))
    with E.Engine(bs) as eng:
        eng.set_schedule(staged)
        J0, K0 = eng.jk(D, [D])
        eng.request_abort(True)
        with pytest.raises(E.HfgpuError) as err:
            eng.jk(D, [D])
        assert err.value.code == 4 and "hfgpu_request_abort" in str(err.value)
        dev = torch.device("cuda", 0)
        Dd = torch.from_numpy(D).to(dev)
        J = torch.zeros_like(Dd)
        K = torch.zeros_like(Dd)
        torch.cuda.synchronize()
        eng.jk_device(Dd.data_ptr(), 1, Dd.data_ptr(), J.data_ptr(), K.data_ptr())
        assert eng.device_status() == 3
        eng.request_abort(False)
        J1, K1 = eng.jk(D, [D])
        assert eng.device_status() == 0
    assert np.max(np.abs(J1 - J0)) < 1e-12 and np.max(np.abs(K1[0] - K0[0])) < 1e-12


def test_gradient_form_autotuner_keeps_the_gradient():
    """hfgpu_autotune_grad picks, per op-table class, thread, warp or block form; the gradient
    after tuning equals the oracle's (FP64, 1e-10)."""
    rng = np.random.default_rng(43)
    bs = MOLS[1][1]  # methane cc-pVDZ: d shells, every op-table class present
    D = _sym(rng, bs.nbf)
    g0 = oracle.grad2e_rhf(bs, D)
    with E.Engine(bs) as eng:
        forms = eng.autotune_grad(D, repeats=1)
        assert set(np.unique(forms)) <= {-1, 0, 1, 2, 3, 4, 5, 6} and (forms >= 0).any()
        g = eng.grad2e(D)
    assert np.max(np.abs(g - g0)) < 1e-10


@pytest.mark.parametrize("form", [0, 1, 2, 3, 4, 5, 6],
                         ids=["thread", "warp", "warp-split-per-set", "block", "block-split-per-set",
                              "block8", "block8-split-per-set"])
@pytest.mark.parametrize("name,bs", MOLS, ids=[m[0] for m in MOLS])
def test_every_gradient_form_matches_oracle(name, bs, form):
    """Each gradient form of the op-table classes forced in turn: one thread per quartet, one
    warp per quartet, the warp form split into four launches of one accumulator set each, and
    the same two with a block of four or eight warps per quartet (FP64 1e-10, mixed 1e-6
    against the oracle)."""
    rng = np.random.default_rng(47)
    D = _sym(rng, bs.nbf)
    g0 = oracle.grad2e_rhf(bs, D)
    with E.Engine(bs) as eng:
        eng.set_grad_forms(form)
        g = eng.grad2e(D)
        gm = eng.grad2e(D, precision=E.MIXED)
    assert np.max(np.abs(g - g0)) < 1e-10
    assert np.max(np.abs(gm - g0)) < 1e-6
