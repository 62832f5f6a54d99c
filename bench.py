"""Benchmark: direct RHF Fock builds/s on one B200 (per GPU, replicas for N > 1).

Workload (the headline configuration): n-octane C8H18, RHF/6-31G** with
Cartesian d (210 basis functions), FP64 direct Fock builds, Schwarz 1e-12,
density screening 1e-12, at the converged SCF density.  Geometry: idealised
all-trans chain rotated by a seeded quaternion (synthetic; no dataset).

A step is one full Fock build F = H + 2J[D] - K[D] over every screened shell
quartet.  `value` times the device-resident build (CUDA events on the engine's
stream, L2 flushed between steps); `e2e` times the reference-facing C ABI call
hfgpu_fock_rhf with pinned host D, H and F (copies inside the timed region).

`--impl reference` times the reference's own CPU code for the same build
(oracle/_ref: the reference's integral translation units compiled in place) on a
bounded sample, with all host threads.

Launch: python bench.py [--gpus N --steps K --warmup W] (torchrun for N > 1).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = ("n-octane C8H18 RHF/6-31G** (Cartesian d, 210 basis functions), FP64 direct Fock build, "
            "Schwarz 1e-12, density screening 1e-12, converged SCF density")
METRIC = "direct RHF Fock builds/s"
UNIT = "Fock builds/s"
N_ITER_AMORTISE = 15  # SCF iterations the reference's one-off ERI generation is spread over


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the 512-molecule batched section")
    ap.add_argument("--no-configs", action="store_true", help="skip the H2O, anthracene and (H2O)8 sections")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch schedule")
    return ap.parse_args()


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def workload_basis():
    from hfscf_b200 import basis as B, molecules as M
    Z, x, name, pure = M.workload(2)
    return B.build_basis(name, Z, x, pure=pure)


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own code on a bounded sample
# ---------------------------------------------------------------------------
def reference_fock_build_seconds(bs, eri_stride=1, fock_rows=10):
    """The reference's Fock build on this host's cores: its ERI generation (every unique shell
    quartet with eri_stride = 1, else every eri_stride-th scaled to all, with its default
    Schwarz screening) amortised over N_ITER_AMORTISE SCF iterations, plus one
    update_fock_matrix contraction (rows 0..fock_rows-1, scaled to all N(N+1)/2 rows)."""
    import oracle
    if not oracle.ref_available():
        return None
    L = oracle.ref()
    L.hfref_time_eri_sample.restype = ctypes.c_double
    L.hfref_time_fock_sample.restype = ctypes.c_double
    args, keep = oracle._flat(bs)
    s, t, fixed = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_double()
    sec = L.hfref_time_eri_sample(*args, ctypes.c_double(1e-14), ctypes.c_longlong(eri_stride), ctypes.byref(s),
                                  ctypes.byref(t), ctypes.byref(fixed))
    # sampled quartets scaled to all; the once-per-geometry part (first touch of the ERI
    # vector, screen matrix) added once
    t_eri = sec * t.value / max(s.value, 1) + fixed.value
    c = ctypes.c_double()
    n = bs.nbf
    sec2 = L.hfref_time_fock_sample(ctypes.c_longlong(n), ctypes.c_longlong(fock_rows), ctypes.byref(c))
    frac = sum(n - i for i in range(fock_rows)) / (n * (n + 1) / 2)
    t_con = sec2 / frac
    build = t_eri / N_ITER_AMORTISE + t_con
    what = "every unique shell quartet" if eri_stride == 1 else \
        f"every {eri_stride}th unique shell quartet ({s.value} of {t.value}) scaled to all"
    sample = (f"reference Erios over {what}, plus the screen matrix and first touch of the ERI vector; "
              f"update_fock_matrix contraction over rows 0..{fock_rows - 1} scaled to N(N+1)/2 rows; "
              f"build = t_eri/{N_ITER_AMORTISE} + t_contract")
    return {"seconds_per_build": build, "t_eri_s": t_eri, "t_contract_s": t_con, "sample": sample,
            "sample_wall_s": sec + sec2 + fixed.value}


def reference_gradient_seconds(bs, stride=20, rows=4):
    """The reference's RHF gradient, two-electron part (the dominant one): its derivative
    integrals over every stride-th unique quartet scaled to all, plus 3 natoms x (one dV/dX
    assembly pass + one dG/dX contraction, rows 0..rows-1 scaled to all)."""
    import oracle
    if not oracle.ref_available():
        return None
    L = oracle.ref()
    args, keep = oracle._flat(bs)
    td, tf, ta, tc, ck = (ctypes.c_double() for _ in range(5))
    t = time.perf_counter()
    rc = L.hfref_time_grad_sample(*args, ctypes.c_double(1e-14), ctypes.c_longlong(stride), ctypes.c_longlong(rows),
                                  ctypes.byref(td), ctypes.byref(tf), ctypes.byref(ta), ctypes.byref(tc),
                                  ctypes.byref(ck))
    wall = time.perf_counter() - t
    if rc != 0:
        return None
    per_coord = ta.value + tc.value
    total = td.value + tf.value + 3 * bs.natoms * per_coord
    return {"t_grad_s": total, "t_deriv_s": td.value, "t_tensor_alloc_s": tf.value,
            "t_assemble_per_coordinate_s": ta.value, "t_contract_per_coordinate_s": tc.value,
            "sample": f"Erios deriv1 over every {stride}th unique shell quartet scaled to all; "
                      f"dV/dX assembly timed for one coordinate and the dG/dX contraction over {rows} rows "
                      f"scaled to N(N+1)/2, both x 3 natoms = {3 * bs.natoms}",
            "sample_wall_s": wall}


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    import oracle
    bs = workload_basis()
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref/libhfref.so not built"}))
        return 0
    # warm-up and timed steps: each step is one bounded sample of a reference Fock build
    for _ in range(args.warmup):
        reference_fock_build_seconds(bs, eri_stride=200, fock_rows=1)
    times = []
    last = None
    t0 = time.perf_counter()
    for _ in range(args.steps):
        last = reference_fock_build_seconds(bs, eri_stride=20, fock_rows=4)
        times.append(last["seconds_per_build"])
    wall = time.perf_counter() - t0
    per = statistics.mean(times)
    v = 1.0 / per
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "nbf": bs.nbf, "amortised_over_scf_iterations": N_ITER_AMORTISE},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "reference", "sample": last["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "sample_wall_s": wall}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples of SM clock, power and throttle reasons every 20 ms, started before the
    timed region (stop() keeps the samples whose timestamps fall inside it, or, when the region is
    shorter than the sampling interval, the samples nearest to it)."""
    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index, interval_ms=20):
        self.index = index
        self.interval_ms = interval_ms
        self.proc = None
        self.path = None
        self.t0 = self.t1 = None

    def start(self):
        """Starts sampling and waits (at most 5 s) until the first sample has arrived."""
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.interval_ms)],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        deadline = time.time() + 5.0
        while time.time() < deadline and os.path.getsize(self.path) == 0:
            time.sleep(0.02)

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()
        time.sleep(2.5 * self.interval_ms / 1e3)  # let a sample after the region arrive

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 10:
                continue
            try:
                date, _, frac = p[0].partition(".")
                ts = time.mktime(time.strptime(date, "%Y/%m/%d %H:%M:%S")) + (float("0." + frac) if frac else 0.0)
                rows.append((ts, float(p[2]), float(p[3]), p[4], [p[6 + k] for k in range(4)]))
            except (ValueError, IndexError):
                continue
        os.unlink(self.path)
        if not rows:
            return None
        window = "timed region"
        sel = [r for r in rows if self.t0 is not None and self.t0 - 0.05 <= r[0] <= self.t1 + 0.05]
        if not sel and self.t0 is not None:
            mid = 0.5 * (self.t0 + self.t1)
            sel = sorted(rows, key=lambda r: abs(r[0] - mid))[:3]
            window = "3 samples nearest the timed region (it is shorter than the sampling interval)"
        if not sel:
            sel, window = rows, "whole run"
        reasons = sorted({self.REASONS[k] for r in sel for k in range(4) if r[4][k].lower() == "active"})
        return {"sm_mhz": statistics.median(r[1] for r in sel), "sm_max_mhz": max(r[2] for r in sel),
                "reasons": reasons, "samples": len(sel), "window": window,
                "interval_ms": self.interval_ms}


def config_oracle():
    """Oracle energies and gradients of the single-molecule configurations (committed fixture
    made from the reference's own integrals by tests/golden/make_config_refs.py), or None."""
    path = os.path.join(ROOT, "tests", "golden", "config_oracle.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f)["configs"]


CONFIG_NAMES = {1: "H2O RHF/cc-pVDZ (pure d, 24 functions)",
                2: "n-octane C8H18 RHF/6-31G** (Cartesian d, 210 functions)",
                3: "anthracene C14H10 RHF/cc-pVDZ (pure d, 246 functions)",
                4: "(H2O)8 RHF/6-31G* (Cartesian d, 152 functions)"}


def time_to_solution(bs, eng, torch):
    """SCF from the SAD guess + RHF gradient, FP64 and mixed precision (incremental Delta-D
    builds), each run twice with the second pass kept so neither pays a first launch."""
    from hfscf_b200 import engine as E
    from hfscf_b200 import scf
    out = {}
    for _pass in range(2):
        for mode, prec in (("fp64", E.FP64), ("mixed", E.MIXED)):
            torch.cuda.synchronize()
            t = time.perf_counter()
            res = scf.rhf(bs, engine=eng, guess="sad", precision=prec, incremental=prec == E.MIXED)
            scf_s = time.perf_counter() - t
            t = time.perf_counter()
            grad = scf.rhf_gradient(bs, res, eng, prec)
            grad_s = time.perf_counter() - t
            out[mode] = {"res": res, "grad": grad, "scf_s": scf_s, "grad_s": grad_s}
    return out


def device_build_ms(eng, D, reps, torch, flush):
    """Mean CUDA-event time of `reps` device-resident J/K builds (L2 flushed before each)."""
    n = D.shape[0]
    J = torch.empty_like(D)
    K = torch.empty_like(D)
    st = torch.cuda.current_stream()
    eng.jk_device(D.data_ptr(), 1, D.data_ptr(), J.data_ptr(), K.data_ptr())
    tot = 0.0
    for k in range(reps):
        flush.fill_(float(k))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        eng.jk_device(D.data_ptr(), 1, D.data_ptr(), J.data_ptr(), K.data_ptr())
        b.record(st)
        b.synchronize()
        tot += a.elapsed_time(b)
    del n
    return tot / reps


def tune_best_of(eng, D0, trials, torch, flush, device):
    """hfgpu_autotune run `trials` times on the core-guess density D0 (each run starts from the
    schedule the previous one left); the schedule whose flushed builds on D0 were fastest (median
    of 7) is kept.  One tuner run chooses among forms whose times differ by less than the
    run-to-run spread of a whole build, so its result varies; the best of a few is stable."""
    import numpy as np
    from hfscf_b200 import engine as E
    Dd = torch.from_numpy(np.ascontiguousarray(D0)).to(device)
    best = None
    for _ in range(trials):
        sched = eng.autotune(D0, E.FP64, 3)
        ms = sorted(device_build_ms(eng, Dd, 1, torch, flush) for _ in range(7))[3]
        if best is None or ms < best[0]:
            best = (ms, sched)
    eng.set_schedule(best[1])
    return best


def other_configs(local, stream, flush, oracle_refs, autotune):
    """Configurations 1, 3 and 4: Fock build time, SCF + gradient time to solution in FP64 and
    mixed precision, and their errors against the oracle's energies and gradients."""
    import torch
    from hfscf_b200 import basis as B, molecules as M
    from hfscf_b200 import engine as E
    from hfscf_b200.profile_case import core_guess_density
    out = {}
    for idx in (1, 3, 4):
        Z, x, name, pure = M.workload(idx)
        bs = B.build_basis(name, Z, x, pure=pure)
        t = time.perf_counter()
        eng = E.Engine(bs, device=local)
        eng.set_stream(stream.cuda_stream)
        setup_s = time.perf_counter() - t
        if autotune:
            S0, T0, V0 = E.one_electron(bs)
            D0 = core_guess_density(bs, S0, T0 + V0)
            eng.autotune(D0, E.FP64, 3)
            eng.autotune_grad(D0, E.FP64, 2)
        tts = time_to_solution(bs, eng, torch)
        D = torch.from_numpy(np.ascontiguousarray(tts["fp64"]["res"].D)).to(torch.device("cuda", local))
        build_ms = device_build_ms(eng, D, 10, torch, flush)
        ent = {"workload": CONFIG_NAMES[idx], "nbf": bs.nbf, "handle_setup_s": setup_s,
               "fock_build_ms": build_ms, "fock_builds_per_s": 1e3 / build_ms}
        ref = (oracle_refs or {}).get(str(idx))
        for mode in ("fp64", "mixed"):
            r = tts[mode]
            e = {"energy": r["res"].energy, "iterations": r["res"].iterations, "converged": r["res"].converged,
                 "scf_s": r["scf_s"], "grad_s": r["grad_s"], "scf_plus_grad_s": r["scf_s"] + r["grad_s"]}
            if ref is not None:
                e["dE_vs_oracle"] = r["res"].energy - ref["energy"]
                if "gradient" in ref:
                    e["max_abs_dgrad_vs_oracle"] = float(np.max(np.abs(r["grad"] - np.array(ref["gradient"]))))
            ent[mode] = e
        ent["time_to_solution_ratio_fp64_over_mixed"] = ent["fp64"]["scf_plus_grad_s"] / ent["mixed"]["scf_plus_grad_s"]
        out[str(idx)] = ent
        eng.close()
        torch.cuda.set_stream(stream)
    return out


HESS_WORKLOADS = (("(H2O)4 RHF/6-31G* (Cartesian d, 76 functions)", "w4"),
                  (CONFIG_NAMES[4], 4), (CONFIG_NAMES[2], 2))


def hessian_basis(key):
    """Basis of a Hessian workload: the (H2O)8 and octane configurations, and a water tetramer
    built like the octamer (first four lattice sites, the octamer's seed)."""
    from hfscf_b200 import basis as B, molecules as M
    if key == "w4":
        rng = np.random.default_rng(M.SEED_BASE + 4)
        Z, x = M.water_cluster(4, 2.9, rng, 0.1)
        return B.build_basis("6-31g*", Z, np.asarray(x) * M.A2B, pure=False)
    Z, x, name, pure = M.workload(key)
    return B.build_basis(name, Z, x, pure=pure)


def hessian_section(local, stream, flush):
    """Two-electron part of the RHF Hessian at the converged density (hfgpu_hess2e_device, the
    adjoint second-derivative kernels): device time per Hessian (CUDA events on the engine's
    stream, L2 flushed before each, median of 3 after one warm-up)."""
    import torch
    from hfscf_b200 import engine as E
    from hfscf_b200 import scf
    out = {}
    dev = torch.device("cuda", local)
    for name, key in HESS_WORKLOADS:
        bs = hessian_basis(key)
        eng = E.Engine(bs, device=local)
        eng.set_stream(stream.cuda_stream)
        res = scf.rhf(bs, engine=eng, guess="core")
        D = torch.from_numpy(np.ascontiguousarray(res.D)).to(dev)
        n3 = 3 * bs.natoms
        H = torch.zeros((n3, n3), dtype=torch.float64, device=dev)
        times = []
        for k in range(4):
            H.zero_()
            flush.fill_(float(k))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            eng.hess2e_device(D.data_ptr(), 2.0, 1, D.data_ptr(), 1.0, H.data_ptr())
            b.record(stream)
            b.synchronize()
            if k:
                times.append(a.elapsed_time(b))
        Hh = H.cpu().numpy()
        ms = float(np.median(times))
        out[str(key)] = {"workload": name, "nbf": bs.nbf, "natoms": bs.natoms, "hess2e_ms": ms,
                         "hessians_per_s": 1e3 / ms, "max_abs_asymmetry": float(np.max(np.abs(Hh - Hh.T))),
                         "max_abs_translational_residual": float(np.max(np.abs(Hh.reshape(n3, -1, 3).sum(axis=1))))}
        eng.close()
        torch.cuda.set_stream(stream)
    return out


def sharded_build(eng, D, Hd, J, K, F, flush, stream, args, pg, rank, world):
    """One molecule's Fock build partitioned over the ranks (hfgpu_set_partition(rank, world):
    every world-th quartet of each class list) and the partial G = 2J - K summed with one NCCL
    all-reduce per build, F = H + G on every rank.  Device time of the timed steps with CUDA
    events on the build's stream, max over ranks; total work fixed as the ranks grow (strong)."""
    import torch
    F_whole = F.clone()
    G = torch.empty_like(F)
    eng.set_partition(rank, world)

    def step():
        eng.jk_device(D.data_ptr(), 1, D.data_ptr(), J.data_ptr(), K.data_ptr())
        torch.sub(J, K, alpha=0.5, out=G)
        G.mul_(2.0)
        pg.all_reduce(G)
        torch.add(Hd, G, out=F)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    pg.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.fill_(float(k))
        ev[k][0].record(stream)
        step()
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    pg.barrier()
    tot = torch.tensor([sum(a.elapsed_time(b) for a, b in ev) / 1e3], dtype=torch.float64, device=F.device)
    pg.all_reduce(tot, op=pg.ReduceOp.MAX)
    total_s = float(tot.item())
    err = float((F - F_whole).abs().max().item())
    eng.set_partition(0, 1)
    return {"builds_per_s": args.steps / total_s, "ms_per_build": 1e3 * total_s / args.steps,
            "scaling": "strong", "parts": world,
            "collective": "one NCCL all-reduce of G = 2J - K (n^2 doubles) per build",
            "max_abs_F_vs_whole_build": err}


def run_ours(args, world, rank, local):
    import torch
    from hfscf_b200 import engine as E
    from hfscf_b200 import flopmodel, scf
    from hfscf_b200.basis import nuclear_repulsion

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    bs = workload_basis()
    n = bs.nbf
    # one dedicated stream shared by torch and the engine, so the CUDA events
    # below bracket the engine's kernels (the legacy default stream has handle 0)
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    eng = E.Engine(bs, device=local)
    eng.set_stream(stream.cuda_stream)
    # --- untimed set-up: launch schedule, converged SCF (FP64), gradient, mixed-precision SCF ---
    dev = torch.device("cuda", local)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # 256 MiB > 126 MB L2
    tune_s = None
    tuned_ms, tuned_sched = None, None
    if not args.no_autotune:
        from hfscf_b200.profile_case import core_guess_density
        S0, T0, V0 = E.one_electron(bs)
        t = time.perf_counter()
        D0 = core_guess_density(bs, S0, T0 + V0)
        tuned_ms, tuned_sched = tune_best_of(eng, D0, 3, torch, flush, torch.device("cuda", local))
        eng.autotune_grad(D0, E.FP64, 2)
        tune_s = time.perf_counter() - t
    # SCF + gradient time-to-solution, FP64 and mixed, each from the SAD guess (the
    # reference's default); the second of two passes is kept.
    tts = time_to_solution(bs, eng, torch)
    res, grad, scf_wall, grad_wall = (tts["fp64"][k] for k in ("res", "grad", "scf_s", "grad_s"))
    res_mx, grad_mx, mixed_wall, grad_mx_wall = (tts["mixed"][k] for k in ("res", "grad", "scf_s", "grad_s"))
    S, T, V = E.one_electron(bs)
    H = T + V
    D = torch.from_numpy(np.ascontiguousarray(res.D)).to(dev)
    Hd = torch.from_numpy(np.ascontiguousarray(H)).to(dev)
    J = torch.empty((n, n), dtype=torch.float64, device=dev)
    K = torch.empty((n, n), dtype=torch.float64, device=dev)
    F = torch.empty((n, n), dtype=torch.float64, device=dev)

    def step():
        eng.jk_device(D.data_ptr(), 1, D.data_ptr(), J.data_ptr(), K.data_ptr())
        torch.add(Hd, J, alpha=2.0, out=F)
        F.sub_(K)

    for _ in range(args.warmup):
        step()
    eng.set_timing(True)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    class_ms = np.zeros(E.NUM_CLASSES)
    class_work = [None] * E.NUM_CLASSES
    launches = 0
    torch.cuda.synchronize()
    clocks.mark_start()
    torch.cuda.profiler.start()  # ncu --profile-from-start off captures only the timed steps
    for k in range(args.steps):
        flush.fill_(float(k))
        starts[k].record(stream)
        step()
        ends[k].record(stream)
        launches += eng.last_launches() + 2  # + the two elementwise ops of F
        for c in range(E.NUM_CLASSES):
            class_ms[c] += eng.class_time_ms(c)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    clocks.mark_end()
    if pg:
        pg.barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    clk = clocks.stop()
    eng.set_timing(False)
    for c in range(E.NUM_CLASSES):
        class_work[c] = eng.class_stats(c)
    total_s = sum(step_ms) / 1e3
    if pg:
        tt = torch.tensor([total_s], device=dev, dtype=torch.float64)
        pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        total_s = float(tt.item())
    value = world * args.steps / total_s
    # the same molecule's build split over the ranks (only with more than one rank)
    sharded = sharded_build(eng, D, Hd, J, K, F, flush, stream, args, pg, rank, world) if pg else None

    # --- end to end through the reference-facing C ABI, pinned host buffers -----------------
    Dh = torch.from_numpy(np.ascontiguousarray(res.D)).pin_memory()
    Hh = torch.from_numpy(np.ascontiguousarray(H)).pin_memory()
    Fh = torch.empty((n, n), dtype=torch.float64).pin_memory()
    for _ in range(2):
        eng.fock_rhf_ptr(Dh.data_ptr(), Hh.data_ptr(), Fh.data_ptr())
    e2e_s = 0.0
    for k in range(args.steps):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        t = time.perf_counter()
        eng.fock_rhf_ptr(Dh.data_ptr(), Hh.data_ptr(), Fh.data_ptr())
        torch.cuda.synchronize()
        e2e_s += time.perf_counter() - t
    if pg:
        tt = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
        pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        e2e_s = float(tt.item())
    e2e = {"value": world * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 2 * n * n * 8,
           "d2h_bytes_per_step": n * n * 8, "api": "hfgpu_fock_rhf (host D, H -> host F)"}
    err_f = float(np.max(np.abs(Fh.numpy() - F.cpu().numpy())))

    # --- roofline -------------------------------------------------------------------------------
    # The unit is one Fock build: 21 class kernels launched concurrently on six streams
    # between a fork and a join event, so per-class event times overlap; the build's
    # achieved FP64 rate is its algorithmic FLOPs over its event-timed duration.
    peak = E.fp64_peak_tflops(local)
    flops_c = [flopmodel.class_flops(c, class_work[c]["computed"], class_work[c]["prim_quartets"], bs.pure)
               for c in range(E.NUM_CLASSES)]
    total_flops = sum(flops_c)
    gen_flops = sum(flopmodel.generated_class_flops(c, class_work[c]["computed"], class_work[c]["prim_quartets"],
                                                    bs.pure) for c in range(E.NUM_CLASSES))
    build_ms = sum(step_ms) / args.steps
    achieved = total_flops / (build_ms * 1e-3) / 1e12
    dom = int(np.argmax(flops_c))
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get("octane_6-31gss_fock_build_dram_bytes")
    roof = {"bound": "fp64", "kernel": "Fock build = 21 quartet-class kernels, concurrent (fork/join)",
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
            "peak_source": "measured in this run: register-only FP64 FMA kernel (hfgpu_fp64_peak); "
                           "MEASURED_PEAKS.json has no FP64 figure",
            "flops_per_build": total_flops,
            "flop_model": "frozen Head-Gordon-Pople count per class (hfscf_b200/flopmodel.py), independent of "
                          "the generated kernels",
            "generated_code_flops_per_build": gen_flops, "build_ms": build_ms,
            "dominant_class": {"class": flopmodel.class_name(dom), "flop_share": flops_c[dom] / total_flops,
                               "event_ms_overlapped": class_ms[dom] / args.steps}}
    # The two-electron gradient on the converged density (RHF weights cJ = 2, cK = 1), device
    # time with CUDA events, L2 flushed before each; its frozen-model FLOPs (derivative classes,
    # every Schwarz-screened quartet) against the same FP64 peak.
    g2 = torch.zeros((bs.natoms, 3), dtype=torch.float64, device=dev)
    for _ in range(2):
        eng.grad2e_device(D.data_ptr(), 2.0, 1, D.data_ptr(), 1.0, g2.data_ptr())
    g_ms = []
    for k in range(3):
        flush.fill_(float(k))
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        eng.grad2e_device(D.data_ptr(), 2.0, 1, D.data_ptr(), 1.0, g2.data_ptr())
        g1.record(stream)
        g1.synchronize()
        g_ms.append(g0.elapsed_time(g1))
    gwork = [eng.class_work(c) for c in range(E.NUM_CLASSES)]
    gflops = sum(flopmodel.grad_class_flops(c, gwork[c]["quartets"], gwork[c]["prim_quartets"], bs.pure)
                 for c in range(E.NUM_CLASSES))
    grad_ms = float(np.median(g_ms))
    g_ach = gflops / (grad_ms * 1e-3) / 1e12
    roof["gradient"] = {"kernel": "two-electron gradient = 21 derivative-class kernels, concurrent",
                        "device_ms": grad_ms, "ms_samples": [round(t, 3) for t in g_ms],
                        "flops": gflops, "achieved": g_ach, "frac": g_ach / peak,
                        "ms_over_build_ms": grad_ms / build_ms,
                        "flops_over_build_flops": gflops / total_flops,
                        "flop_model": "frozen count of the derivative classes (flopmodel.grad_class_flops)"}
    eris_per_build = sum(flopmodel.class_integrals(c, class_work[c]["computed"], bs.pure) for c in range(E.NUM_CLASSES))
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sum(step_ms) / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded geometry)",
            "config": {"workload": WORKLOAD, "nbf": n, "parallelism": f"replicas x{world}",
                       "l2": "flushed between steps (256 MiB write)",
                       "schedule": ("default" if tune_s is None else
                                    f"best of three hfgpu_autotune runs, and hfgpu_autotune_grad, on the "
                                    f"core-guess density ({tune_s:.2f} s, untimed)"),
                       "schedule_table": None if tuned_sched is None else tuned_sched.tolist(),
                       "quartets_screened": int(sum(class_work[c]["screened"] for c in range(E.NUM_CLASSES))),
                       "quartets_computed_last_build": int(sum(class_work[c]["computed"] for c in range(E.NUM_CLASSES)))},
            "roofline": roof, "e2e": e2e, "gpu_launches": launches, "clocks": clk, "sharded": sharded,
            "scf": {"guess": "SAD", "energy": res.energy, "iterations": res.iterations, "converged": res.converged,
                    "mixed_iterations": res_mx.iterations,
                    "wall_s": scf_wall, "grad_wall_s": grad_wall, "grad_max": float(np.max(np.abs(grad))),
                    "mixed_incremental_energy": res_mx.energy, "mixed_dE": res_mx.energy - res.energy,
                    "mixed_wall_s": mixed_wall, "e_nuc": nuclear_repulsion(bs.Z, bs.coords),
                    "fp64_fock_ms": [round(1e3 * t, 3) for t in res.fock_times],
                    "mixed_incremental_fock_ms": [round(1e3 * t, 3) for t in res_mx.fock_times],
                    "time_to_solution_ratio_fp64_over_mixed": scf_wall / mixed_wall,
                    "fock_time_ratio_fp64_over_mixed": sum(res.fock_times) / sum(res_mx.fock_times),
                    "mixed_grad_wall_s": grad_mx_wall,
                    "mixed_grad_max_abs_diff": float(np.max(np.abs(grad_mx - grad))),
                    "scf_plus_grad_ratio_fp64_over_mixed": (scf_wall + grad_wall) / (mixed_wall + grad_mx_wall)},
            "check": {"max_abs_F_device_vs_api": err_f},
            # model-independent rates: contracted integrals (blocks x block size) per second of the
            # timed builds, and whole RHF gradients (two-electron + one-electron + nuclear) per second
            "throughput": {"eris_per_build": eris_per_build,
                           "eris_per_s": eris_per_build / (build_ms * 1e-3),
                           "gradients_per_s": 1.0 / grad_wall,
                           "mixed_gradients_per_s": 1.0 / grad_mx_wall}}
    # Accounting of the mixed-precision speed-up: the FP32 share of the build's frozen-model
    # flops (quartets below the Schwarz bound 1e-4, by class), the per-build bound that share
    # allows at the FP32:FP64 issue ratio of 2:1, and the time of the SCF outside the Fock builds,
    # which mixed precision does not touch.
    f32_flops = 0.0
    per_class = {}
    for c in range(E.NUM_CLASSES):
        w = class_work[c]
        if w["screened"] > 0:
            share = (w["screened"] - w["high_bound"]) / w["screened"]
            f32_flops += flops_c[c] * share
            per_class["".join("spd"[w[k]] for k in ("la", "lb", "lc", "ld"))] = {
                "flop_share_of_build": round(flops_c[c] / total_flops, 4),
                "fp32_quartet_share": round(share, 4),
                "bound_fp64_over_mixed": round(1.0 / ((1.0 - share) + 0.5 * share), 3)}
    f32 = f32_flops / total_flops
    t_build64 = sum(res.fock_times)
    t_buildmx = sum(res_mx.fock_times)
    line["mixed_accounting"] = {
        "fp32_flop_share_of_build": f32,
        "per_class": per_class,
        "per_build_bound_fp64_over_mixed": 1.0 / ((1.0 - f32) + 0.5 * f32),
        "fp64_scf_builds_s": t_build64, "fp64_scf_other_s": scf_wall - t_build64,
        "mixed_scf_builds_s": t_buildmx, "mixed_scf_other_s": mixed_wall - t_buildmx,
        "ratio_bound_if_mixed_builds_took_no_time":
            (scf_wall + grad_wall) / max(mixed_wall - t_buildmx + grad_mx_wall, 1e-12),
        "note": "FP32:FP64 issue ratio 2:1 on the non-tensor pipes; the SCF's time outside the builds "
                "(DIIS, diagonalisation, guess) is the same in both modes"}
    refs = config_oracle()
    if refs is not None and "2" in refs:
        r2 = refs["2"]
        line["scf"]["oracle"] = "tests/golden/config_oracle.json (oracle RHF on the reference's own integrals)"
        line["scf"]["dE_vs_oracle"] = res.energy - r2["energy"]
        line["scf"]["mixed_dE_vs_oracle"] = res_mx.energy - r2["energy"]
        if "gradient" in r2:
            g0 = np.array(r2["gradient"])
            line["scf"]["max_abs_dgrad_vs_oracle"] = float(np.max(np.abs(grad - g0)))
            line["scf"]["mixed_max_abs_dgrad_vs_oracle"] = float(np.max(np.abs(grad_mx - g0)))
    if not args.no_configs and world == 1:
        line["configs"] = other_configs(local, stream, flush, refs, not args.no_autotune)
        line["hessian"] = hessian_section(local, stream, flush)
    if not args.no_batch:
        # batched-mode workload: 512 seeded small molecules, SCF + gradient each, in one batched handle
        from hfscf_b200 import batch as BT
        from hfscf_b200 import molecules as MM
        from hfscf_b200 import dist as DI
        allm = MM.batch_molecules(512)
        bb = BT.batch_bases([allm[i] for i in DI.shard(len(allm), rank, world)])  # replicas: molecules split
        # the launch schedule from the autotuner, tuned once on the batch in an untimed run (as the
        # octane schedule is); the timed runs below take it as given
        t_tune = time.perf_counter()
        tuned_sched = BT.batch_rhf(bb, device=local, autotune=True, gradient=False, max_iter=2)["schedule"]
        t_tune = time.perf_counter() - t_tune
        torch.cuda.set_stream(stream)

        def timed_batch(**kw):
            """Three whole runs (set-up, SCF, gradients; each wall-clock, max over ranks); the run of
            median wall time is reported, with all three walls (a run's host-side set-up varied
            from 0.4 to 1.2 s between otherwise equal runs)."""
            runs = []
            for _ in range(3):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                r = BT.batch_rhf(bb, device=local, schedule=tuned_sched, **kw)
                runs.append((DI.max_over_ranks(time.perf_counter() - t0, dev), r))
                torch.cuda.set_stream(stream)
            runs.sort(key=lambda x: x[0])
            return runs[1][0], runs[1][1], [round(w, 4) for w, _ in runs]

        wall, rb, walls = timed_batch()
        line["batch"] = {"workload": "512 seeded molecules ((H2O)1-6, CH4, C2H6, NH3; STO-3G or 6-31G*), "
                                     "RHF to convergence + RHF gradient each, one batched handle",
                         "molecules_per_s": 512 / wall, "wall_s": wall, "setup_s": rb["setup_s"],
                         "setup_stages_s": {k: round(v, 4) for k, v in rb["setup_stages_s"].items()},
                         "scf_s": rb["scf_s"], "grad_s": rb["grad_s"], "final_s": rb["final_s"],
                         "close_s": rb["close_s"], "iterations": rb["iterations"],
                         "converged": int(rb["converged"].sum()), "cuda_graph": rb["graph"], "autotuned": rb["autotuned"],
                         "schedule": f"hfgpu_autotune on the batch, untimed ({t_tune:.2f} s incl. its set-up)",
                         "jk_build_ms": rb["build_ms_mean"], "nbf_total": int(sum(b.nbf for b in bb)),
                         "density_step": rb["density"], "diag_fallback_iterations": rb["diag_fallbacks"],
                         "runs": "median of three whole runs", "walls_s": walls}
        # the same batch in mixed precision (FP32 quartets below the Schwarz bound 1e-4)
        wall_m, rbm, walls_m = timed_batch(precision=E.MIXED)
        line["batch"]["mixed"] = {"molecules_per_s": 512 / wall_m, "wall_s": wall_m, "walls_s": walls_m,
                                  "setup_s": rbm["setup_s"],
                                  "scf_s": rbm["scf_s"], "grad_s": rbm["grad_s"], "iterations": rbm["iterations"],
                                  "converged": int(rbm["converged"].sum()),
                                  "max_abs_dE_vs_fp64": float(np.max(np.abs(rbm["energies"] - rb["energies"])))}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
        ref = reference_fock_build_seconds(bs)
        if ref is not None:
            cb = {"value": 1.0 / ref["seconds_per_build"], "unit": UNIT, "cores": os.cpu_count(),
                  "kind": "reference", "sample": ref["sample"], "t_eri_s": ref["t_eri_s"],
                  "t_contract_s": ref["t_contract_s"]}
            # the reference's SCF (ERIs once, one contraction per iteration; the iteration count of
            # the engine's FP64 SCF from the same SAD guess) and its RHF gradient
            cb["t_scf_s"] = ref["t_eri_s"] + res.iterations * ref["t_contract_s"]
            gref = reference_gradient_seconds(bs)
            if gref is not None:
                cb["gradient"] = gref
                cb["t_grad_s"] = gref["t_grad_s"]
                cb["t_scf_plus_grad_s"] = cb["t_scf_s"] + gref["t_grad_s"]
                cb["scf_plus_grad_ratio_reference_over_fp64"] = cb["t_scf_plus_grad_s"] / (scf_wall + grad_wall)
            # the reference's Hessian two-electron part on the water tetramer (sampled; the larger
            # workloads need tens of GB of derivative tensors and hours of its per-atom-pair loops)
            try:
                import oracle
                if oracle.ref_available() and "hessian" in line:
                    rh = oracle.ref_time_hess_sample(hessian_basis("w4"), stride=20)
                    rh["sample"] = ("second-derivative shell routines over every 20th quartet of one xx and one xy "
                                    "loop, scaled; assembly + contraction of one atom pair of each kind, scaled to "
                                    "all pairs and direction pairs (hfscf_hessian_ints.cpp:20-303)")
                    rh["workload"] = HESS_WORKLOADS[0][0]
                    rh["ratio_reference_over_ours"] = rh["t_hess2e_s"] / (line["hessian"]["w4"]["hess2e_ms"] / 1e3)
                    cb["hessian"] = rh
            except Exception as exc:  # the Fock-build baseline stands without it
                cb["hessian"] = {"error": repr(exc)}
            line["cpu_baseline"] = cb
    if rank == 0:
        print(json.dumps(line))
    eng.close()
    if pg:
        pg.destroy_process_group()
    return 0


def main():
    args = parse()
    world, rank, local = dist_init()
    if args.impl == "reference":
        return run_reference(args, world, rank)
    return run_ours(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
