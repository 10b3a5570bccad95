"""Benchmark of the B200 R-matrix solver on the production workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one collision-matrix solve (`rmatrix`) of the production workload: 128
channels x 200 Lagrange mesh points (N = 25600, 128 surface right-hand sides) at
E = 10 MeV -- device assembly of C(E), the mixed-precision LU (3xTF32 tcgen05 trailing
updates), triangular solves, FP64 FGMRES refinement to the FP64 residual floor, R
extraction and the collision matrix.  Inputs are synthetic (seeded; see
hprmat_b200/workloads.py).  `value` is solves/s with the potential already in HBM; `e2e`
is the same through the host C ABI call with the pinned host potential copied in and U
copied out every step.  With N > 1 (torchrun) every rank solves its own copy of the
workload (independent solves; no collective on the data path) and the throughput is the
sum over ranks, timed as the max over ranks.

`--impl reference` times the reference's own algorithm on the host cores instead: the
FP64 restatement of HPRMAT's Type 1 path (assembly, LAPACK zgesv through OpenBLAS on all
host cores, R, U) on the same N = 25600 workload, after the reference's own warm-up of the
BLAS thread pool (a 512 x 512 zgetrf, examples/Ex0/benchmark_large.f90:84-98).  One such solve
takes about a minute on 16 cores, so the arm times as many whole solves as fit in
--ref-budget-s (at least one) and reports that count with the reason.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_FULL = 25600
METRIC = "solves/s"
UNIT = "solves/s"
FLOPS_PER_SOLVE = 8.0 * N_FULL ** 3 / 3.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-comparators", action="store_true", help="skip the FP64 device-LU comparators")
    ap.add_argument("--solves-only", action="store_true",
                    help="only the device-resident timed solves (for profiler launch lists)")
    ap.add_argument("--nch", type=int, default=128, help="channels of the production generator (N = 200 nch)")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed",
                    help="production with --solves-only: the path of the timed solves (fp64: this library's plain "
                         "FP64 LU with the DMMA GEMM, for profiler launch lists of its kernels)")
    ap.add_argument("--workload", choices=["production", "scan", "adjoint", "sweep"], default="production",
                    help="production: one N = 25600 solve per step (the headline); scan: the batched energy "
                         "scan, 12 J-pi blocks x 256 energies (3072 solves) per step; adjoint: loss and gradients "
                         "over 64 energies at N = 3200 per step; sweep: the precision sweep, N = 4000 .. 51200 "
                         "with closed channels at 40 MeV, each size against the device FP64 LU")
    ap.add_argument("--workers", type=int, default=8,
                    help="worker contexts (host thread + stream each) of the batched scan and the adjoint")
    ap.add_argument("--reuse", type=int, default=-1,
                    help="scan/adjoint: keep a block's factorisation across energies as the refinement's "
                         "preconditioner (opts.reuse_factors); default off (measured faster that way for "
                         "both workloads)")
    ap.add_argument("--scan-method", choices=["lu", "shifted"], default="shifted",
                    help="scan: lu (every energy by its own mixed LU on concurrent worker streams) or shifted (one "
                         "Hessenberg reduction per J-pi block, O(N^2 nch) FP64 work per energy, "
                         "hprmat_b200_rmatrix_scan_shifted)")
    ap.add_argument("--scan-blocks", type=int, default=0,
                    help="scan: only the first K J-pi blocks (0: all 12; the first is the largest, N = 3180), for "
                         "profiler runs of one block")
    ap.add_argument("--scan-energies", type=int, default=0,
                    help="scan: only the first K energies of each block (0: all 256), for profiler runs that must "
                         "hold little device memory")
    ap.add_argument("--autotune", type=int, default=0,
                    help="scan: run the scan autotuner (hprmat_b200_scan_autotune) on the scan's blocks before "
                         "the warm-up, outside the timed region")
    ap.add_argument("--ref-budget-s", type=float, default=150.0,
                    help="--impl reference and the cpu_baseline leg: wall-time budget of the timed N = 25600 CPU "
                         "solves; a solve starts only while the projected end stays inside it (at least one runs)")
    ap.add_argument("--tune-cache", default="",
                    help="scan with --autotune: JSON file of the tuned table; loaded when present, written "
                         "after tuning otherwise")
    return ap.parse_args()


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ CPU baseline
def cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def blas_warmup(times: int = 1):
    """The reference's warm-up of the BLAS thread pool before its timed solves: a 512 x 512
    zgetrf (examples/Ex0/benchmark_large.f90:84-98)."""
    from scipy.linalg import lapack
    ww = np.ones((512, 512), dtype=np.complex128, order="F")
    ww[np.arange(512), np.arange(512)] = 1024.0
    for _ in range(max(times, 1)):
        lapack.zgetrf(ww.copy(order="F"))


def cpu_type1_solves(nch: int, max_solves: int, budget_s: float):
    """Time whole Type 1 solves (the oracle's restatement of src/rmatrix_hp.F90:246-368 with
    LAPACK zgesv, the call of src/rmat_solvers.F90:127) of the production workload at `nch`
    channels, one after another, while the projected end of the next solve stays inside
    budget_s (at least one solve).  Returns (seconds of each solve, N, U of the last solve)."""
    from hprmat_b200 import workloads
    from oracle import rmatrix_oracle as orc
    w = workloads.production(nch=nch)
    mesh = orc.rmat_ini(w.nr, 1, w.rmax)
    ts, res = [], None
    t_begin = time.perf_counter()
    while len(ts) < max(max_solves, 1):
        if ts and (time.perf_counter() - t_begin) + max(ts) > budget_s:
            break
        t = time.perf_counter()
        res = orc.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, mesh, w.cpot)
        ts.append(time.perf_counter() - t)
    return ts, w.n, res.cu


def run_reference(args):
    rank, world, _ = dist_info()
    if rank != 0:
        return 0
    os.environ.setdefault("OPENBLAS_NUM_THREADS", str(cores()))
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    blas_warmup(args.warmup)
    ts, n, _ = cpu_type1_solves(args.nch, args.steps, args.ref_budget_s)
    t_mean = sum(ts) / len(ts)
    value = 1.0 / t_mean
    nthreads = int(os.environ["OPENBLAS_NUM_THREADS"])
    why = ("" if len(ts) == args.steps else
           f"; {len(ts)} of the {args.steps} requested steps timed: one solve takes {t_mean:.0f} s, and the "
           f"arm stops starting solves once the next would end after its {args.ref_budget_s:.0f} s budget")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": len(ts), "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": t_mean * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic (seeded production generator, hprmat_b200/workloads.py)",
        "config": {"workload": "production: 128 channels x 200 points, N=25600, nrhs=128, E=10 MeV",
                   "N": n, "nrhs": args.nch},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                         "sample": f"oracle Type 1 path (assembly, OpenBLAS zgesv on {nthreads} threads, R, U) on "
                                   f"the production workload itself (N={n}); warm-up: {args.warmup} x 512^2 "
                                   f"zgetrf as examples/Ex0/benchmark_large.f90:84-98; wall time per whole solve "
                                   f"{', '.join(f'{t:.1f}' for t in ts)} s" + why},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ batched energy scan
def run_scan(args):
    """One step = the whole scan: 12 J-pi blocks (nch ~ U{4..64}, 60 mesh points, N = 240..3840)
    x 256 energies = 3072 collision matrices, through hprmat_b200_rmatrix_scan.  With N ranks
    the blocks are sharded by cost (hprmat_b200.scan_shard.lpt_shards: greedy longest
    processing time on nenergies x N^3 over runs of 32 energies), independent units, no
    collective on the data path."""
    rank, world, local = dist_info()
    import torch
    import torch.distributed as dist
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    from hprmat_b200 import api, workloads
    from oracle import rmatrix_oracle as orc
    from hprmat_b200.scan_shard import shard_units
    blocks = workloads.scan_blocks()
    if args.scan_blocks > 0:
        blocks = blocks[:args.scan_blocks]
    if args.scan_energies > 0:
        blocks = [(w, np.asarray(e)[:args.scan_energies]) for w, e in blocks]
    all_inputs = []
    for w, energies in blocks:
        ks = [workloads.channel_kinematics(e, w.thresholds, w.hm, w.params.z1z2) for e in energies]
        all_inputs.append((w.lval, w.cpot, np.array([k[0] for k in ks]), np.array([k[1] for k in ks])))
    # this rank's runs of 32 energies (one run per block when alone), sharded by cost
    units, inputs = shard_units(all_inputs, 60, rank, world, chunk=None if world == 1 else 32,
                                method=args.scan_method)
    mine = [(blocks[b][0], np.asarray(blocks[b][1])[idx]) for b, idx in units]
    flops = sum(len(e) * 8.0 * float(w.n) ** 3 / 3.0 for w, e in mine)
    nunits = sum(len(e) for _, e in mine)
    if args.reuse < 0:
        args.reuse = 0
    ctx = api.Context(device=local, precision="mixed", max_refine=3, tol=1e-12, reuse_factors=bool(args.reuse))
    from hprmat_b200 import _native as nat
    lib = nat.load()
    tune = None
    if args.autotune:
        if args.tune_cache and os.path.exists(args.tune_cache):
            with open(args.tune_cache) as f:
                table = json.load(f)["table"]
            ctx.set_scan_tune_table(table)
            tune = {"source": args.tune_cache, "table": ctx.scan_tune_table()}
        else:
            table = ctx.scan_autotune(inputs, 20.0, 60, nworkers=args.workers)
            tune = {"source": "tuned", "seconds": ctx.last_autotune_seconds, "table": table}
            if args.tune_cache and rank == 0:
                import torch as _t
                with open(args.tune_cache, "w") as f:
                    json.dump({"device": _t.cuda.get_device_name(local), "workers": args.workers, "table": table}, f)
    # warm-up: the LU method's first block already runs on every worker; the shifted method
    # puts up to three blocks in flight, so its warm-up takes all of them (worker contexts and
    # their buffers are created outside the timed steps)
    for _ in range(args.warmup):
        ctx.rmatrix_scan(inputs if args.scan_method == "shifted" else inputs[:1], 20.0, 60, nworkers=args.workers,
                         allow_unconverged=True, raise_on_unit_error=False, method=args.scan_method)
    lib.hprmat_b200_dev_factorizations(ctx._h, 1)
    secs = []
    res = None
    for _ in range(args.steps):
        if world > 1:
            dist.barrier()
        res = ctx.rmatrix_scan(inputs, 20.0, 60, nworkers=args.workers, allow_unconverged=True,
                               raise_on_unit_error=False, method=args.scan_method)
        secs.append(ctx.last_scan_seconds)
    t = max(secs) / 1.0
    t_local = torch.tensor([sum(secs)], dtype=torch.float64, device=f"cuda:{local}")
    if world > 1:
        dist.all_reduce(t_local, op=dist.ReduceOp.MAX)
    tot_units = torch.tensor([float(nunits)], dtype=torch.float64, device=f"cuda:{local}")
    tot_flops = torch.tensor([flops], dtype=torch.float64, device=f"cuda:{local}")
    if world > 1:
        dist.all_reduce(tot_units)
        dist.all_reduce(tot_flops)
    wall = float(t_local.item())
    value = float(tot_units.item()) * args.steps / wall
    nfact = int(lib.hprmat_b200_dev_factorizations(ctx._h, 1)) / max(1, args.steps)
    # sampled accuracy: the largest and smallest block at their first and last energy, vs the oracle
    errs = []
    mesh = orc.rmat_ini(60, 1, 20.0)
    picks = sorted(range(len(mine)), key=lambda i: mine[i][0].nch)
    for i in ({picks[0], picks[-1]} if picks else set()):
        w, energies = mine[i]
        for e in (0, len(energies) - 1):
            lval, cpot, qk, eta = inputs[i]
            if res[i][2][e] != 0:
                continue
            ref = orc.rmatrix(w.nch, lval, qk[e], eta[e], 20.0, mesh, cpot)
            cu = res[i][0][e]
            no = ref.nopen
            errs.append(float(np.linalg.norm(cu[:no, :no] - ref.cu) / np.linalg.norm(ref.cu)))
    # CPU baseline: the oracle's Type 1 path (OpenBLAS zgesv, all host cores) on one energy of
    # each block, extrapolated to the scan by the blocks' energy counts
    cpu = None
    if rank == 0:
        t_cpu = 0.0
        for i, (w, energies) in enumerate(mine):
            lval, cpot, qk, eta = inputs[i]
            e = len(energies) // 2
            t1 = time.perf_counter()
            try:
                orc.rmatrix(w.nch, lval, qk[e], eta[e], 20.0, mesh, cpot)
            except Exception:
                pass
            t_cpu += (time.perf_counter() - t1) * len(energies)
        cpu = {"value": nunits / t_cpu, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
               "sample": "oracle Type 1 path at the middle energy of every block, scaled by the block's energy count"}
    bad = int(sum(int(((r[2] != 0) & (r[2] != 99)).sum()) for r in res))
    unconverged = int(sum(int((r[2] == 99).sum()) for r in res))
    if rank == 0:
        print(json.dumps({
            "metric": "scan solves/s", "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None,
            "dtype": ("c128 (Hessenberg reduction, shifted solves, FP64 refinement)" if args.scan_method == "shifted"
                      else "c64 via 3xTF32 tensor cores + c128 refinement"),
            "data": "synthetic (seeded scan generator, hprmat_b200/workloads.py)",
            "config": {"workload": "batched energy scan: 12 J-pi blocks, nch ~ U{4..64} x 60 points "
                                   "(N = 240..3840), 256 energies each, 3072 solves"
                                   + (f" (first {len(blocks)} block(s) only)" if len(blocks) < 12 else "")
                                   + (f" (first {args.scan_energies} energies of each)" if args.scan_energies > 0
                                      else ""),
                       "method": args.scan_method, "blocks": len(blocks),
                       "energies_per_block": args.scan_energies or None,
                       # the LU scan's worker streams; the shifted scan keeps the library's
                       # default of 3 blocks in flight
                       "workers": args.workers if args.scan_method == "lu" else 3,
                       "reuse_factors": bool(args.reuse),
                       "autotune": bool(args.autotune)},
            "autotune": tune,
            "lu_equivalent_complex_tflops": float(tot_flops.item()) * args.steps / wall / 1e12,
            "factorizations_per_step": nfact,
            "units_failed": bad, "units_failed_note": "COULFG ifail=-5 (high-l channels just above threshold); "
                                                      "the oracle fails on the same units",
            "units_not_converged": unconverged,
            "u_rel_err_sampled": max(errs) if errs else None, "cpu_baseline": cpu}))
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------ adjoint gradients
def run_adjoint(args):
    """One step = loss sum_E sum |U - U_target|^2 over 64 energies at N = 3200 (32 channels x
    100 points) and its gradient with respect to the 6 potential parameters and the potential
    at all mesh points (torch.autograd: forward solves keep X on the device, the backward forms
    the gradient from it, hprmat_b200_rmatrix_x / hprmat_b200_adjoint_from_x).  Checked once
    against central finite differences (step 1e-6) of the device forward and against the FP64
    oracle adjoint at two energies."""
    import torch
    from hprmat_b200 import api, workloads
    from hprmat_b200.autograd import collision_matrices, potential_matrix
    from oracle import rmatrix_oracle as orc
    w, energies = workloads.adjoint_case()
    r = torch.from_numpy(workloads.lagrange_radii(w.nr, w.rmax))
    coup = torch.from_numpy(w.coupling)
    p0 = torch.tensor(w.params.as_array(), dtype=torch.float64)
    ptarget = p0 * torch.tensor([1.02, 0.97, 1.01, 1.03, 0.95, 1.04], dtype=torch.float64)
    if args.reuse < 0:
        args.reuse = 0
    ctx = api.Context(precision="mixed", max_refine=8, tol=1e-12, reuse_factors=bool(args.reuse))
    from hprmat_b200 import _native as nat
    lib = nat.load()
    # energies where COULFG (the reference's algorithm) cannot evaluate an open channel just above
    # its threshold are dropped (the oracle fails on them too)
    from oracle import special_functions as sf

    def coulfg_ok(qk, eta):
        return all(sf.coulfg(qk[c] * w.rmax, eta[c], float(w.lval[c]))[4] == 0 for c in range(w.nch) if qk[c] > 0)

    kin_all = [workloads.channel_kinematics(e, w.thresholds, w.hm, w.params.z1z2) for e in energies]
    kin = [k for k in kin_all if coulfg_ok(*k)]
    tgt = np.asfortranarray(potential_matrix(r, coup, ptarget, w.hm, w.params.z1z2).numpy())
    targets = [ctx.rmatrix(w.nch, w.lval, qk, eta, w.rmax, w.nr, 1, tgt)[0] for qk, eta in kin]

    # the energies' solves run concurrently on a pool of contexts (one host thread and stream each)
    pool = [ctx] + [api.Context(precision="mixed", max_refine=8, tol=1e-12, reuse_factors=bool(args.reuse))
                    for _ in range(max(1, args.workers) - 1)]

    def loss(p):
        cp = potential_matrix(r, coup, p, w.hm, w.params.z1z2)
        us = collision_matrices(cp, pool, w.lval, kin, w.rmax, w.nr)
        tot = 0.0
        for u, ut in zip(us, targets):
            no = u.shape[0]
            tot = tot + torch.sum(torch.abs(u - torch.from_numpy(ut[:no, :no])) ** 2)
        return tot, cp

    for _ in range(args.warmup):
        p = p0.clone().requires_grad_(True)
        L, _ = loss(p)
        L.backward()
    times = []
    for c in pool:
        lib.hprmat_b200_dev_factorizations(c._h, 1)
    for _ in range(args.steps):
        t = time.perf_counter()
        p = p0.clone().requires_grad_(True)
        L, cp = loss(p)
        cp.retain_grad()
        L.backward()
        times.append(time.perf_counter() - t)
    nfact = sum(int(lib.hprmat_b200_dev_factorizations(c._h, 1)) for c in pool) / max(1, args.steps)
    g = p.grad.numpy().copy()
    # central finite differences of the device forward, step 1e-6 (relative to the parameter);
    # the forward solves of the differences run to tighter tolerances, so that the noise of U
    # (~1e-11 at the default surface tolerance) does not dominate the difference quotient
    for c in pool:
        c.set_precision("mixed", tol=1e-14, surface_tol=1e-13)
    fd_err = 0.0
    for k in range(6):
        e = torch.zeros(6, dtype=torch.float64)
        e[k] = 1e-6 * max(1.0, abs(float(p0[k])))
        with torch.no_grad():
            fd = (float(loss(p0 + e)[0]) - float(loss(p0 - e)[0])) / (2 * float(e[k]))
        fd_err = max(fd_err, abs(fd - g[k]) / max(abs(fd), 1e-300))
    # FP64 CPU reference gradient (oracle adjoint) at the first and last energy
    mesh = orc.rmat_ini(w.nr, 1, w.rmax)
    c_np = np.asfortranarray(potential_matrix(r, coup, p0, w.hm, w.params.z1z2).numpy())
    ref_err = 0.0
    for i in (0, len(kin) - 1):
        qk, eta = kin[i]
        u0 = orc.rmatrix(w.nch, w.lval, qk, eta, w.rmax, mesh, c_np).cu
        gu = 2 * (u0 - targets[i][:u0.shape[0], :u0.shape[0]])
        _, gref = orc.rmatrix_adjoint(w.nch, w.lval, qk, eta, w.rmax, mesh, c_np, gu)
        _, _, gdev = ctx.rmatrix_adjoint(w.nch, w.lval, qk, eta, w.rmax, w.nr, c_np, gu)
        ref_err = max(ref_err, float(np.linalg.norm(gdev - gref) / np.linalg.norm(gref)))
    sec = min(times)
    print(json.dumps({
        "metric": "adjoint gradient evaluations/s", "value": 1.0 / sec, "unit": "gradients/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec, "higher_is_better": True,
        "scaling": "none", "vs_baseline": None, "dtype": "c64 3xTF32 forward + c128 refinement; c128 adjoint",
        "data": "synthetic (seeded adjoint generator, hprmat_b200/workloads.py)",
        "config": {"workload": "adjoint: 32 channels x 100 points (N = 3200), 64 energies, loss sum |U - U_target|^2, "
                               "gradients w.r.t. 6 potential parameters and the potential at all mesh points",
                   "workers": len(pool)},
        "energies_used": len(kin), "energies_dropped_coulfg": len(kin_all) - len(kin),
        "solves_per_step": len(kin), "factorizations_per_step": nfact, "reuse_factors": bool(args.reuse),
        "backward": "symmetric potential: gradient from the forward solution kept on the device (no second solve)",
        "fd_rel_err_max": fd_err, "fd_step": 1e-6, "oracle_grad_rel_err_max": ref_err,
        "loss": float(L.detach())}))
    for c in pool:
        c.close()
    return 0


# ------------------------------------------------------------------ precision sweep
def run_sweep(args):
    """The precision sweep: the production generator with closed-channel thresholds at 40 MeV at
    nch = 20, 50, 80, 128, 256 (N = 4000 .. 51200).  Per size: the mixed solve (best of
    --steps after --warmup, CUDA-event time on the context's stream), its refinement record,
    and its U against the device FP64 LU's (an independent algorithm and precision; no CPU
    oracle finishes at the larger sizes)."""
    import ctypes
    import torch
    from hprmat_b200 import api, workloads
    rows = []
    for nch in workloads.SWEEP_NCH:
        w = workloads.sweep(nch)
        ctx = api.Context(precision="mixed")
        stream = torch.cuda.Stream()
        ctx.set_stream(stream.cuda_stream)
        for _ in range(args.warmup):
            ctx.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
        best = None
        for _ in range(max(1, args.steps)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            cu_m, nopen = ctx.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        st = ctx.last_stats
        # tensor-pipe use: one more mixed solve with the trailing updates bracketed by events
        lib = ctx._lib
        lib.hprmat_b200_dev_counters(ctx._h, None, None, None, None, 1)
        lib.hprmat_b200_dev_set_profile(ctx._h, 1)
        ctx.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
        lib.hprmat_b200_dev_set_profile(ctx._h, 0)
        tc_ms, tc_flops, tc_n = ctypes.c_double(0), ctypes.c_double(0), ctypes.c_int(0)
        lib.hprmat_b200_dev_counters(ctx._h, None, ctypes.byref(tc_ms), ctypes.byref(tc_flops), ctypes.byref(tc_n), 1)
        # the FP64 LU of the same C(E), with its 1-norm condition estimate (Hager-Higham on the
        # FP64 factors; reported separately from the timed mixed solves)
        ctx.set_precision("fp64")
        # a small FP64 solve first, so that the timed one does not include the FP64 path's first-use setup
        a_w = np.eye(300, dtype=np.complex128) * 4.0 + 0.01
        ctx.solve_linear(a_w, np.ones((300, 1), np.complex128))
        ctx.set_estimate_condition(True)
        cu_d, _ = ctx.rmatrix(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, w.cpot)
        fp64_ms = ctx.last_stats["ms_total"] - ctx.last_stats["ms_condest"]
        kappa1 = ctx.last_stats["cond_estimate"]
        condest_ms = ctx.last_stats["ms_condest"]
        diff = float(np.linalg.norm(cu_m[:nopen, :nopen] - cu_d[:nopen, :nopen]) / np.linalg.norm(cu_d[:nopen, :nopen]))
        # against the oracle's U (FP64 zgesv) where the committed fixture exists (N = 10000 .. 25600)
        fx = os.path.join(ROOT, "tests", "golden", f"sweep_u_nch{nch}.npz")
        err_fx = None
        if os.path.exists(fx):
            ref = np.load(fx)["u"]
            err_fx = float(np.linalg.norm(cu_m[:nopen, :nopen] - ref) / np.linalg.norm(ref))
        n = w.n
        rows.append({"N": n, "nch": nch, "nopen": nopen, "ms_per_solve": best, "solves_per_s": 1e3 / best,
                     "complex_tflops": 8.0 * n ** 3 / 3.0 / (best * 1e-3) / 1e12, "nb": st["nb"],
                     "refine_steps": st["refine_steps"], "inner_iterations": st["inner_iterations"],
                     "rel_residual": st["rel_residual"], "residual_floor": st["residual_floor"],
                     "pivot_growth": st["pivot_growth"], "fp64_fallback": st["fp64_fallback"],
                     "u_rel_diff_vs_device_fp64": diff, "u_rel_err_vs_oracle_fixture": err_fx,
                     "device_fp64_ms": fp64_ms,
                     "mixed_over_fp64": fp64_ms / best, "cond1_estimate": kappa1, "cond1_estimate_ms": condest_ms,
                     "tc_update_tflops": tc_flops.value / max(tc_ms.value, 1e-9) / 1e9,
                     "tc_update_share": tc_ms.value / best})
        ctx.close()
        del cu_m, cu_d
        torch.cuda.empty_cache()
    print(json.dumps({"metric": "precision sweep", "unit": "per size", "n_gpus": 1, "steps": args.steps,
                      "warmup": args.warmup, "higher_is_better": True, "dtype": "c64 via 3xTF32 + c128 refinement",
                      "data": "synthetic (seeded sweep generator, hprmat_b200/workloads.py)",
                      "config": {"workload": "precision sweep: production generator, closed channels at 40 MeV, "
                                             "nch = 20, 50, 80, 128, 256 x 200 points"},
                      "sizes": rows}))
    return 0


# ------------------------------------------------------------------ our arm
def main():
    args = parse()
    if args.precision != "mixed" and (not args.solves_only or args.workload != "production"):
        print("bench: --precision fp64 is for --solves-only runs of the production workload (the headline is the "
              "mixed path)", file=sys.stderr)
        return 2
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "scan":
        return run_scan(args)
    if args.workload == "adjoint":
        return run_adjoint(args)
    if args.workload == "sweep":
        return run_sweep(args)
    rank, world, local = dist_info()
    import torch
    import torch.distributed as dist
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    import ctypes
    from hprmat_b200 import _native as nat
    from hprmat_b200 import api, workloads

    w = workloads.production(nch=args.nch)
    n_full = w.n
    ctx = api.Context(device=local, precision=args.precision, max_refine=3, tol=1e-12)
    stream = torch.cuda.Stream(device=dev)
    ctx.set_stream(stream.cuda_stream)
    ctx.rmat_ini(w.nr, 1, w.rmax)
    ncp1, ndim = w.cpot.shape[0], w.nch
    d_cpot = torch.from_numpy(np.asfortranarray(w.cpot).ravel(order="F").view(np.float64)).to(dev)
    d_cu = torch.zeros(ndim * ndim * 2, dtype=torch.float64, device=dev)
    lib = nat.load()

    def step_device():
        # a step that stops at max_refine above its tolerance is recorded (status 99), not hidden:
        # the timed loop keeps every step's status and the run exits nonzero if one did not converge
        return ctx.rmatrix_device(w.nch, w.lval, w.qk, w.eta, w.rmax, w.nr, 1, d_cpot.data_ptr(), ncp1, ndim,
                                  d_cu.data_ptr(), allow_unconverged=True)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(args.warmup):
        step_device()
    st_warm = dict(ctx.last_stats or {})
    # ---- timed region (device-resident inputs)
    lib.hprmat_b200_dev_counters(ctx._h, None, None, None, None, 1)
    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    stats = []
    for _ in range(args.steps):
        step_device()
        stats.append(dict(ctx.last_stats))
    e1.record(stream)
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    launches = ctypes.c_ulonglong(0)
    lib.hprmat_b200_dev_counters(ctx._h, ctypes.byref(launches), None, None, None, 1)
    t_local = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t_local, op=dist.ReduceOp.MAX)
    ms_max = float(t_local.item())
    ms_per_step = ms_max / args.steps
    value = world * args.steps / (ms_max / 1e3)

    # ---- U accuracy against the committed FP64 oracle fixture
    cu = d_cu.cpu().numpy().view(np.complex128).reshape(ndim, ndim, order="F")
    nopen = int((w.qk > 0).sum())
    u_err = None
    fx = os.path.join(ROOT, "tests", "golden", f"production_u_nch{args.nch}.npz")
    if os.path.exists(fx):
        ref = np.load(fx)["u"]
        u_err = float(np.linalg.norm(cu[:nopen, :nopen] - ref) / np.linalg.norm(ref))

    if args.solves_only:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                              "warmup": args.warmup, "ms_per_step": ms_per_step, "N": n_full, "u_rel_err": u_err,
                              "precision": args.precision,
                              "gpu_launches": int(launches.value), "clocks": clk}))
        ctx.close()
        if world > 1:
            dist.destroy_process_group()
        return 0

    # ---- end to end through the host C ABI: pinned host cpot in, U out, every step
    h_cpot = torch.from_numpy(np.asfortranarray(w.cpot).ravel(order="F").view(np.float64)).pin_memory()
    h_cu = torch.zeros(ndim * ndim * 2, dtype=torch.float64).pin_memory()
    P = ctypes.POINTER(ctypes.c_double)
    lval = np.ascontiguousarray(w.lval, dtype=np.int32)
    qk = np.ascontiguousarray(w.qk)
    eta = np.ascontiguousarray(w.eta)
    nop = ctypes.c_int(0)
    sst = nat.Stats()

    def step_host():
        s = lib.hprmat_b200_rmatrix(ctx._h, w.nch, lval.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                    qk.ctypes.data_as(P), eta.ctypes.data_as(P), w.rmax, w.nr, 1,
                                    ctypes.cast(h_cpot.data_ptr(), P), ncp1, ndim, ctypes.cast(h_cu.data_ptr(), P),
                                    ctypes.byref(nop), ctypes.byref(sst))
        nat.check(s, (nat.OK, nat.NOT_CONVERGED))

    step_host()
    barrier()
    e0.record(stream)
    for _ in range(args.steps):
        step_host()
    e1.record(stream)
    barrier()
    t_e2e = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t_e2e, op=dist.ReduceOp.MAX)
    e2e_value = world * args.steps / (float(t_e2e.item()) / 1e3)

    # ---- roofline of the dominant kernel (tensor-core trailing update), one profiled solve
    lib.hprmat_b200_dev_set_profile(ctx._h, 1)
    step_device()
    lib.hprmat_b200_dev_set_profile(ctx._h, 0)
    tc_ms, tc_flops, tc_n = ctypes.c_double(0), ctypes.c_double(0), ctypes.c_int(0)
    lib.hprmat_b200_dev_counters(ctx._h, None, ctypes.byref(tc_ms), ctypes.byref(tc_flops), ctypes.byref(tc_n), 1)
    peaks = {}
    pk_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk_path):
        peaks = json.load(open(pk_path))
    # TF32 dense peak = half the measured bf16 rate (sustained: the kernel runs inside a long step)
    bf16 = peaks.get("bf16_tflops_sustained") or 1400.0
    tf32_peak = bf16 / 2.0
    achieved = (tc_flops.value / max(tc_n.value, 1)) / ((tc_ms.value / max(tc_n.value, 1)) / 1e3) / 1e12
    # DRAM traffic per launch: ncu measured 1.05x the algorithmic bytes (C read + write and the
    # operand planes) for the trailing update at N = 12800; scaled here to the mean algorithmic
    # bytes of this solve's trailing updates
    nb_ = 128
    ms_ = [n_full - (s + 1) * nb_ for s in range((n_full + nb_ - 1) // nb_ - 1)]
    alg_bytes = float(np.mean([16.0 * m * m + 2.0 * m * nb_ * 16.0 for m in ms_])) if ms_ else 0.0
    roofline = {"bound": "tensor", "achieved": achieved, "peak": tf32_peak, "unit": "TFLOP/s",
                "frac": achieved / tf32_peak, "traffic": 1.05 * alg_bytes,
                "traffic_note": "bytes per launch: 1.05 x the mean algorithmic bytes, ratio from one ncu capture "
                                "at N = 12800 (dram__bytes_read.sum + dram__bytes_write.sum)",
                "kernel": "tc_update_kernel (3xTF32 complex trailing update)",
                "launches": tc_n.value, "ms_total": tc_ms.value,
                "peak_source": "MEASURED_PEAKS.json bf16_tflops_sustained / 2 (dense TF32 = half of BF16)"
                if peaks else "fallback 1400/2",
                "note": "achieved counts algorithmic complex-LU flops (8 M^2 nb per update); the tensor cores "
                        "execute 3x that (4 real products x 3 TF32 terms / 4 = 3)"}

    # ---- FP64 device comparators (outside the headline's timed region): each the median of
    # n_cmp runs timed with CUDA events on the stream the work is ordered on, after a warm-up
    comparators = {}
    if not args.no_comparators:
        n_cmp = 3

        def event_ms(fn, s):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize(dev)
            a.record(s)
            fn()
            b.record(s)
            torch.cuda.synchronize(dev)
            return a.elapsed_time(b)

        ctx.set_precision("fp64")
        step_device()  # warm-up: FP64 buffers, as the mixed steps had theirs
        ts64, tf64 = [], []
        for _ in range(n_cmp):
            ts64.append(event_ms(step_device, stream))
            tf64.append(float(ctx.last_stats["ms_factor"]))
        comparators["own_fp64_lu_solves_per_s"] = 1e3 / statistics.median(ts64)
        comparators["own_fp64_lu_ms"] = ts64
        # the factorisation alone (host clock around the FP64 LU, which ends synchronised), the
        # like-for-like figure for the library getrf below
        comparators["own_fp64_factor_ms"] = tf64
        cu64 = d_cu.cpu().numpy().view(np.complex128).reshape(ndim, ndim, order="F")
        if u_err is not None:
            comparators["own_fp64_lu_u_rel_err"] = float(np.linalg.norm(cu64[:nopen, :nopen] - ref) /
                                                          np.linalg.norm(ref))
        ctx.set_precision("mixed", max_refine=3, tol=1e-12)
        try:
            A = torch.randn(N_FULL, N_FULL, dtype=torch.complex128, device=dev)
            A.diagonal().add_(2.0 * N_FULL)
            cur = torch.cuda.current_stream(dev)
            torch.linalg.lu_factor(A[:512, :512])
            tsl = []
            for _ in range(n_cmp):
                tsl.append(event_ms(lambda: torch.linalg.lu_factor(A), cur))
            comparators["library_zgetrf_solves_per_s"] = 1e3 / statistics.median(tsl)
            comparators["library_zgetrf_ms"] = tsl
            comparators["own_fp64_factor_over_library_zgetrf"] = statistics.median(tf64) / statistics.median(tsl)
            comparators["library_zgetrf"] = ("torch.linalg.lu_factor(complex128) (cuSOLVER getrf), factorisation "
                                             "only, of a diagonally dominant random matrix of the same order")
            del A
        except Exception as e:  # noqa: BLE001
            comparators["library_zgetrf_error"] = str(e)[:200]
        best = max(v for k, v in comparators.items() if k.endswith("solves_per_s"))
        comparators["mixed_over_best_fp64"] = value / world / best
        comparators["timing"] = f"median of {n_cmp} CUDA-event-timed runs after one warm-up"

    # ---- CPU baseline (rank 0, N = 1 only): one whole Type 1 solve of this same workload
    cpu = None
    if rank == 0 and world == 1:
        os.environ.setdefault("OPENBLAS_NUM_THREADS", str(cores()))
        os.environ.setdefault("OMP_NUM_THREADS", "1")
        blas_warmup()
        ts_cpu, n_s, cu_cpu = cpu_type1_solves(args.nch, 1, args.ref_budget_s)
        cpu = {"value": 1.0 / ts_cpu[0], "unit": UNIT, "cores": int(os.environ["OPENBLAS_NUM_THREADS"]),
               "kind": "port",
               "sample": f"one whole oracle Type 1 solve (assembly, OpenBLAS zgesv, R, U) of this workload "
                         f"(N={n_s}) after a 512^2 zgetrf warm-up: {ts_cpu[0]:.1f} s",
               "u_rel_err_vs_gpu": float(np.linalg.norm(cu_cpu - cu[:nopen, :nopen]) / np.linalg.norm(cu_cpu))}

    last = stats[-1] if stats else st_warm
    step_status = [int(s_.get("status", -1)) for s_ in stats]
    not_converged = sum(1 for v in step_status if v == nat.NOT_CONVERGED)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64 via 3xTF32 tensor cores + c128 refinement",
        "data": "synthetic (seeded production generator, hprmat_b200/workloads.py)",
        "config": {"workload": "production: 128 channels x 200 points, N=25600, nrhs=128, E=10 MeV",
                   "N": N_FULL, "nrhs": 128, "nb": last.get("nb"),
                   "l2": "inputs larger than L2 (5.2 GB complex64 working matrix per solve)"},
        "complex_tflops": value * FLOPS_PER_SOLVE / 1e12,
        "u_rel_err": u_err,
        "step_status": {"ok": sum(1 for v in step_status if v == nat.OK), "not_converged": not_converged,
                        "refine_steps": [int(s_.get("refine_steps", -1)) for s_ in stats],
                        "surface_change_max": max((float(s_.get("surface_change", -1)) for s_ in stats),
                                                  default=None)},
        "refine": {"steps": last.get("refine_steps"), "rel_residual": last.get("rel_residual"),
                   "history": last.get("residual_history"), "ms_factor": last.get("ms_factor"),
                   "ms_refine": last.get("ms_refine"), "pivot_growth": last.get("pivot_growth"),
                   "fp64_fallback": last.get("fp64_fallback")},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h_cpot.numel() * 8),
                "d2h_bytes_per_step": int(h_cu.numel() * 8)},
        "gpu_launches": int(launches.value),
        "roofline": roofline,
        "clocks": clk,
        "comparators": comparators,
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(line))
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if not_converged:
        print(f"bench: {not_converged} timed step(s) ended with HPRMAT_B200_NOT_CONVERGED", file=sys.stderr)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
