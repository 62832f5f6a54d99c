"""One case of the hot path, bracketed for a profiler.

    python -m hfscf_b200.profile_case jk   --workload 2 [--precision mixed] [--repeat 3]
    python -m hfscf_b200.profile_case grad --workload 3 [--repeat 1]
    python -m hfscf_b200.profile_case hess --workload 4 [--repeat 1] [--hess-form 0|1|2|3]
    python -m hfscf_b200.profile_case jk   --workload 2 --variant 2   (every class in the staged form)

Builds the named workload's basis (``molecules.workload``: 1 = H2O/cc-pVDZ,
2 = n-octane/6-31G**, 3 = anthracene/cc-pVDZ, 4 = (H2O)8/6-31G*), forms the
core-guess density (and with ``--autotune`` tunes the J/K launch schedule or the gradient
forms on it),
runs one untimed warm-up of the operation and then
``--repeat`` timed ones between ``cudaProfilerStart``/``cudaProfilerStop`` (so
``ncu --profile-from-start off`` sees exactly those launches).  Prints one JSON
line with the per-call device time and the kernel count of each call.
"""
from __future__ import annotations

import argparse
import json

import numpy as np
import torch

from . import basis as B
from . import engine as E
from . import molecules as M
from . import scf


def core_guess_density(bs, S, H):
    X = scf.sym_orth(S)
    _, Cp = np.linalg.eigh(X.T @ H @ X)
    C = X @ Cp
    nocc = int(np.sum(bs.Z)) // 2
    return C[:, :nocc] @ C[:, :nocc].T


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("op", choices=("jk", "grad", "hess"))
    ap.add_argument("--workload", type=int, default=2)
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="fp64")
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--autotune", action="store_true",
                    help="hfgpu_autotune (jk) or hfgpu_autotune_grad (grad) first, as bench.py does")
    ap.add_argument("--variant", type=int, choices=(0, 1, 2), default=None,
                    help="thread-form variant for every class (schedule column 3: 0 plain, 1 capped, "
                         "2 staged persistent)")
    ap.add_argument("--hess-form", type=int, choices=(-1, 0, 1, 2, 3), default=-1,
                    help="hess: -1 default per class, 0 one thread, 1 one block, 2 one warp per quartet")
    a = ap.parse_args(argv)
    if not torch.cuda.is_available():
        raise SystemExit("profile_case needs a CUDA device")
    Z, x, name, pure = M.workload(a.workload)
    bs = B.build_basis(name, Z, x, pure=pure)
    S, T, V = E.one_electron(bs)
    D = core_guess_density(bs, S, T + V)
    prec = E.MIXED if a.precision == "mixed" else E.FP64
    dev = torch.device("cuda", a.device)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    with E.Engine(bs, device=a.device) as eng:
        eng.set_stream(stream.cuda_stream)
        Dd = torch.from_numpy(np.ascontiguousarray(D)).to(dev)
        if a.autotune:
            if a.op == "jk":
                eng.autotune(Dd, E.FP64, 3)
            else:
                eng.autotune_grad(Dd, prec, 3)
        if a.variant is not None:
            sched = eng.get_schedule()
            sched[:, 3] = a.variant
            eng.set_schedule(sched)
        n = bs.nbf
        J = torch.empty((n, n), dtype=torch.float64, device=dev)
        K = torch.empty((n, n), dtype=torch.float64, device=dev)
        g = torch.zeros((bs.natoms, 3), dtype=torch.float64, device=dev)
        Hs = torch.zeros((3 * bs.natoms, 3 * bs.natoms), dtype=torch.float64, device=dev)
        if a.op == "hess":
            eng.set_hess_form(a.hess_form)

        def once():
            if a.op == "jk":
                eng.jk_device(Dd.data_ptr(), 1, Dd.data_ptr(), J.data_ptr(), K.data_ptr(), prec)
            elif a.op == "hess":
                # two-electron Hessian of sum D (2J - K) at fixed D (RHF weights, as hfgpu_hess2e)
                eng.hess2e_device(Dd.data_ptr(), 2.0, 1, Dd.data_ptr(), 1.0, Hs.data_ptr())
            else:
                # RHF two-electron gradient of sum D (2J - K): cJ = 2, cK = 1 (as hfgpu_grad2e_backward)
                eng.grad2e_device(Dd.data_ptr(), 2.0, 1, Dd.data_ptr(), 1.0, g.data_ptr(), prec)
            return eng.last_launches()

        once()
        torch.cuda.synchronize()
        times, launches = [], []
        torch.cuda.profiler.start()
        for _ in range(a.repeat):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            launches.append(once())
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        torch.cuda.profiler.stop()
        print(json.dumps({"op": a.op, "workload": name, "nbf": n, "precision": a.precision,
                          "ms": [round(t, 3) for t in times], "kernels": launches}))


if __name__ == "__main__":
    main()
