"""Benchmark: RVE homogenization solves per second on B200.

Workload (one "step"): 4096 independent micro-RVEs, structured hex8 meshes
with n drawn uniformly from {8, 12, 16, 20} elements per edge, a centred
z-aligned fiber of radius U(0.1, 0.35), matrix E = 1e9 Pa, fiber/matrix
stiffness ratio log-uniform in [2, 100], Poisson ratios U(0.2, 0.35); each RVE
is solved for its 6 unit-strain load cases to a 1e-8 relative FP64 residual
and volume-averaged (the 6x6 homogenized tangent).  One persistent launch per
step: FP32 Jacobi-PCG on the matrix-free element-type stencil (or, with
--op ell, on assembled FP32 ELL values) with FP64 residual refinement.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank solves its own 4096 RVEs (seeded by rank, no
collective on the data path) and rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RVE solves/sec + p50/p99 latency @1e-8 rel residual, batched-mixed vs plain GPU"
UNIT = "RVE solves/s"
SIZES = (8, 12, 16, 20)
E_MATRIX = 1e9


def workload_params(nrve: int, seed: int, sizes=SIZES):
    rng = np.random.default_rng(seed)
    n = rng.choice(sizes, size=nrve)
    radius = rng.uniform(0.1, 0.35, size=nrve)
    ratio = np.exp(rng.uniform(np.log(2.0), np.log(100.0), size=nrve))
    nu_m = rng.uniform(0.2, 0.35, size=nrve)
    nu_f = rng.uniform(0.2, 0.35, size=nrve)
    return n, radius, ratio, nu_m, nu_f


def workload_descs(mb, nrve: int, seed: int, sizes=SIZES):
    n, radius, ratio, nu_m, nu_f = workload_params(nrve, seed, sizes)
    return [mb.rve_desc(int(n[i]), float(radius[i]), (E_MATRIX, E_MATRIX * float(ratio[i])),
                        (float(nu_m[i]), float(nu_f[i]))) for i in range(nrve)]


def nnz_true(n: int) -> int:
    """Structural nonzeros of the 3D hex8 ELL matrix: 9 (3N-2)^3, N = n+1."""
    return 9 * (3 * (n + 1) - 2) ** 3


def algorithmic_bytes(sizes, inner_its, outer_its, k=6, stencil=True):
    """Bytes the batched solve must move per launch.  Per CG iteration: the
    SpMM input and output vectors, plus, for the assembled operator, the
    FP32 matrix values (4 B per structural nonzero) and one int32 column node
    per 3x3 block (the node-sliced ELL stores one per block), or, for the
    stencil operator, one material byte per element; and 8 FP32 vector
    passes.  Per refinement step 3 FP64 vector passes, plus one for the
    residual of the boundary values alone (the right-hand side the stopping
    rule is relative to; the solve starts from the affine field).  Once per
    RVE the node-sliced values written (assembled operator) or the stencil's
    Jacobi diagonal."""
    total = 0.0
    for n, it, ot in zip(sizes, inner_its, outer_its):
        n, it, ot = int(n), float(it), float(ot)
        ndof = 3 * (n + 1) ** 3
        nelm = n ** 3
        if stencil:
            spmm = nelm + 2 * k * ndof * 4
            setup = ndof * 4
        else:
            spmm = nnz_true(n) * 4 + nnz_true(n) // 9 * 4 + 2 * k * ndof * 4
            setup = ((n + 1) ** 3 + 31) // 32 * 32 * 243 * 4  # node-sliced values written
        vec = 8 * k * ndof * 4
        refine = 3 * k * ndof * 8
        total += it * (spmm + vec) + (ot + 2) * refine + setup
    return total


def l2_note(args, sizes, batch):
    if args.op == "ell":
        return ("inputs larger than L2 (FP32 ELL values alone are "
                f"{sum(3 * (n + 1) ** 3 * 84 * 4 for n in sizes) / 1e9:.1f} GB)")
    return ("inputs larger than L2: the stencil keeps no matrix; the batch's device buffers "
            f"(CG work spaces of the RVEs in flight, plans, materials) are "
            f"{batch.device_bytes() / 1e9:.2f} GB")


def argv_tail(args):
    """The workload-defining flags of this run, in a fixed order, to match a
    profile's command line."""
    return [f"--nrve {args.nrve}", "--sizes " + " ".join(str(x) for x in args.sizes),
            f"--op {args.op}", f"--threads {args.threads}", f"--ctas {args.ctas}",
            f"--inner-rtol {args.inner_rtol:g}"]


# DRAM traffic per launch (dram__bytes_read.sum + dram__bytes_write.sum) from
# one ncu capture of exactly these workloads; the command of each capture is
# in the summary under profiles/ named for its kernel and workload.  The
# bench cannot count DRAM bytes itself, so a run whose workload differs
# reports null.
PROFILED_TRAFFIC = {
    # k_batch, stencil operator, autotuned shape: ncu --metrics dram__bytes_read.sum,
    # dram__bytes_write.sum,gpu__time_duration.sum --clock-control none
    # -k regex:k_batch -s 13 -c 1 python bench.py --steps 1 --warmup 3 ...
    "k_batch --nrve 4096 --sizes 8 12 16 20 --op stencil --threads 0 --ctas 0 "
    "--inner-rtol 0.003": 663920980224,
    # k_spmv_rve, the n = 40 structured matrix, cold L2
    "k_spmv_rve structured ELL n=40": 214213376,
}


def profiled_traffic(kernel: str, workload: str):
    """(bytes per launch, source) of the ncu capture of this workload, or
    (None, reason) when none was taken of it."""
    tb = PROFILED_TRAFFIC.get(f"{kernel} {workload}")
    if tb is None:
        return None, "no ncu capture of this workload"
    return tb, "ncu capture of this workload (dram__bytes_read.sum + dram__bytes_write.sum)"


def structured_ell(n: int, seed: int = 5):
    """84-slot ELL with the sparsity of the hex8 RVE stiffness on an n^3 mesh:
    row 3a + d holds the 3 dofs of every node within one grid step of node a
    (stored slots first, -1 after), random values."""
    N = n + 1
    nn = N ** 3
    a = np.arange(nn, dtype=np.int64)
    i, j, k = a % N, (a // N) % N, a // (N * N)
    nbs = []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                ok = ((i + dx >= 0) & (i + dx < N) & (j + dy >= 0) & (j + dy < N) &
                      (k + dz >= 0) & (k + dz < N))
                nbs.append(np.where(ok, a + dx + dy * N + dz * N * N, -1))
    nb = np.stack(nbs, 1)
    cols = np.where(nb[:, :, None] >= 0, 3 * nb[:, :, None] + np.arange(3), -1).reshape(nn, 81)
    cols = np.take_along_axis(cols, np.argsort(cols < 0, axis=1, kind="stable"), 1)
    full = np.full((3 * nn, 84), -1, np.int32)
    full[:, :81] = np.repeat(cols, 3, axis=0)
    vals = np.where(full >= 0, np.random.default_rng(seed).uniform(-1.0, 1.0, full.shape), 0.0)
    return full, vals


def measure_spmv(mb, stream, sptr, n=40, reps=20):
    """The resident FP64 ELL SpMV (sp_ell_dev_mvp) on one matrix larger than
    L2, at the lanes-per-row width the library's upload-time autotuner chose
    (no override), L2 flushed before every timed launch; achieved =
    algorithmic bytes (stored slots x 12 + x read + y write) / CUDA-event
    time per launch."""
    import torch
    cols, vals = structured_ell(n)
    m = mb.ell_matrix()
    m.nrow = m.ncol = cols.shape[0]
    m.nnz = cols.shape[1]
    m.cols = cols.ctypes.data_as(C.POINTER(C.c_int))
    m.vals = vals.ctypes.data_as(C.POINTER(C.c_double))
    h = mb._vp()
    mb.check(mb.lib().sp_ell_upload(C.byref(m), C.byref(h)), "sp_ell_upload")
    try:
        nrow, wp, nnz = C.c_int(), C.c_int(), C.c_longlong()
        mb.check(mb.lib().sp_ell_dev_info(h, C.byref(nrow), C.byref(wp), C.byref(nnz)), "info")
        lanes, cached = C.c_int(), C.c_int()
        trial = (C.c_float * 4)()
        mb.check(mb.lib().sp_ell_dev_lanes(h, C.byref(lanes), trial, C.byref(cached)), "lanes")
        x_h = np.random.default_rng(6).standard_normal(nrow.value)
        x = torch.from_numpy(x_h).cuda()
        y = torch.empty_like(x)
        xp, yp = C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr())
        # spot check of 2000 rows against numpy
        mb.check(mb.lib().sp_ell_dev_mvp(h, xp, yp, sptr), "mvp")
        torch.cuda.synchronize()
        rows = np.arange(0, nrow.value, max(1, nrow.value // 2000))
        cr = cols[rows]
        ref = (vals[rows] * np.where(cr >= 0, x_h[np.maximum(cr, 0)], 0.0)).sum(1)
        err = float(np.abs(y.cpu().numpy()[rows] - ref).max() / np.abs(ref).max())
        # every timed launch starts from a cold L2: a 256 MB buffer (> 126 MB
        # L2) is read before it, outside the events (a read leaves clean
        # lines, so no write-back of the flush lands inside the timing)
        flush = torch.ones(64 << 20, dtype=torch.float32, device="cuda")
        sink = torch.empty(1, dtype=torch.float32, device="cuda")
        for _ in range(3):
            mb.lib().sp_ell_dev_mvp(h, xp, yp, sptr)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(reps)]
        torch.cuda.synchronize()
        for e0, e1 in evs:
            torch.sum(flush, dim=0, out=sink[0])
            e0.record(stream)
            mb.lib().sp_ell_dev_mvp(h, xp, yp, sptr)
            e1.record(stream)
        torch.cuda.synchronize()
        ms = sum(e0.elapsed_time(e1) for e0, e1 in evs) / reps
        del flush, sink
        abytes = nnz.value * 12 + 2 * nrow.value * 8
        peak, peak_kind = measured_peak()
        ach = abytes / (ms / 1e3) / 1e9
        return {"kernel": "k_spmv_rve (sp_ell_dev_mvp, FP64 ELL, hoisted loads)",
                "matrix": f"hex8 RVE sparsity n={n}: {nrow.value} rows x 84 slots, "
                          f"{nnz.value} stored, {(vals.nbytes + cols.nbytes) / 1e6:.0f} MB > L2",
                "l2": "flushed before every timed launch (a 256 MB read)",
                "lanes_per_row": lanes.value,
                "lanes_source": "the library's upload-time autotuner" +
                                (" (cached choice)" if cached.value else ""),
                "autotuner_trial_us": {str(w): round(float(t), 2)
                                       for w, t in zip((4, 8, 16, 32), trial)},
                "ms": ms, "algorithmic_bytes": abytes,
                "traffic": profiled_traffic("k_spmv_rve", f"structured ELL n={n}")[0],
                "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": ach / peak, "peak_kind": peak_kind, "max_rel_err_vs_numpy": err}
    finally:
        mb.lib().sp_ell_dev_free(h)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------- CPU legs ---

def _oracle_rve(args):
    n, radius, ratio, nu_m, nu_f = args
    from oracle import oracle as O
    m = O.cube_mesh(int(n))
    et = O.fiber_types(m, [1.0, 1.0], float(radius))
    t = time.perf_counter()
    O.unit_tangent(m, et, (E_MATRIX, E_MATRIX * float(ratio)), (float(nu_m), float(nu_f)),
                   rtol=1e-8, lin_rtol=5e-9)
    return int(n), time.perf_counter() - t


def cpu_sample(work, procs: int):
    """Time the oracle (FP64 Jacobi-PCG from the reference's zero start, 6
    load cases) on RVEs of the workload, given as (n, radius, ratio, nu_m,
    nu_f) tuples; returns seconds per RVE for each mesh size, the wall time
    and the per-RVE results."""
    work = sorted(work, key=lambda w: -w[0])  # largest first keeps the pool busy to the end
    if procs > 1:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(procs) as pool:
            pool.map(_oracle_rve, [(8, 0.2, 2.0, 0.3, 0.3)] * procs)  # start-up outside timing
            t0 = time.perf_counter()
            res = list(pool.imap_unordered(_oracle_rve, work, chunksize=1))
            wall = time.perf_counter() - t0
    else:
        t0 = time.perf_counter()
        res = [_oracle_rve(w) for w in work]
        wall = time.perf_counter() - t0
    per = {s: [t for (nn, t) in res if nn == s] for s in SIZES}
    return per, wall, res


def workload_items(nrve: int, seed: int, sizes=SIZES):
    """The workload's RVEs as (n, radius, ratio, nu_m, nu_f) tuples, in the
    order the GPU arm builds them."""
    n, radius, ratio, nu_m, nu_f = workload_params(nrve, seed, sizes)
    return [(int(n[i]), float(radius[i]), float(ratio[i]), float(nu_m[i]), float(nu_f[i]))
            for i in range(nrve)]


def per_size_sample(items, per_size: int):
    """The first `per_size` RVEs of every mesh size."""
    out = []
    for s_ in sorted(set(w[0] for w in items)):
        out += [w for w in items if w[0] == s_][:per_size]
    return out


def mix_rate(per_size_times):
    """RVE/s for the uniform mix of sizes given seconds per RVE per size."""
    mean_t = np.mean([np.mean(v) for v in per_size_times.values() if v])
    return 1.0 / mean_t


def rank_seed(rank: int) -> int:
    """Seed of a rank's workload: every rank solves its own RVEs (weak scaling,
    no data exchange)."""
    return 1234 + rank


def max_over_ranks(dist, value: float, device) -> float:
    """The largest per-rank value (device time of the same steps); every rank
    takes part, in the same order, in warm-up, timing and error paths alike."""
    import torch
    if dist is None:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, nrve: int, steps: int, total_ms: float) -> float:
    """RVE solves per second of the whole job: every rank's RVEs over the
    slowest rank's time."""
    return world * nrve * steps / (total_ms / 1000.0)


def workload_config(args, sizes):
    return {"workload": f"batched tangent: {args.nrve} RVEs per GPU, n uniform in "
                        f"{set(args.sizes)}, 6 unit-strain load cases, rtol 1e-8",
            "nrve_per_gpu": args.nrve, "load_cases": 6, "rtol": 1e-8}


def oracle_check(descs, stress, per_size: int, seed: int = 31):
    """Per-RVE error of the timed batch's stresses against the FP64 oracle
    (relative residual 1e-12) on a seeded sample of the mix, `per_size` RVEs
    of every mesh size: |sigma - sigma_oracle|max / |sigma_oracle|max over the
    6 unit-strain load cases of each RVE."""
    from oracle import pool as OP
    rng = np.random.default_rng(seed)
    picked = []
    for s_ in sorted(set(int(d.n[0]) for d in descs)):
        idx = [i for i, d in enumerate(descs) if d.n[0] == s_]
        picked += sorted(rng.choice(idx, size=min(per_size, len(idx)), replace=False).tolist())
    items = [(int(descs[i].n[0]), descs[i].radius, (descs[i].E[0], descs[i].E[1]),
              (descs[i].nu[0], descs[i].nu[1]), np.eye(6)) for i in picked]
    t0 = time.perf_counter()
    want = OP.run(OP.homogenize, items)
    errs = [float(np.abs(stress[i] - w).max() / np.abs(w).max()) for i, w in zip(picked, want)]
    return {"rves": len(picked), "per_size": per_size, "max": max(errs),
            "p99": float(np.percentile(errs, 99)), "median": float(np.median(errs)),
            "per_rve": [{"rve": int(i), "n": int(descs[i].n[0]), "err": e}
                        for i, e in zip(picked, errs)],
            "oracle": "FP64 Jacobi-PCG restatement, relative residual 1e-12",
            "oracle_s": time.perf_counter() - t0}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    O.lib()
    cores = os.cpu_count() or 1
    per_step = 4 * cores  # RVEs per step: four per core, so the pool stays busy
    # the GPU arm's own RVEs (rank 0's seed), a bounded slice per step
    items = workload_items(args.nrve, rank_seed(0), tuple(args.sizes))
    for _ in range(args.warmup):
        cpu_sample(items[:min(cores, 4)], min(cores, 4))
    rates = []
    t_all = 0.0
    for k in range(args.steps):
        sl = [items[(k * per_step + j) % len(items)] for j in range(per_step)]
        per, wall, res = cpu_sample(sl, cores)
        rates.append(len(res) / wall)
        t_all += wall
    value = float(np.mean(rates))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * t_all / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "impl": "reference",
        "config": {**workload_config(args, args.sizes),
                   "sample_rves_per_step": per_step, "solver": "FP64 Jacobi-PCG (oracle port)",
                   "parallelism": f"rank 0 of {args.gpus}: all host cores"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{per_step} consecutive RVEs of the GPU arm's own "
                                   f"{args.nrve}-RVE workload per step (step k takes RVEs "
                                   f"k*{per_step} on), spawned process pool, one process per core"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------- GPU legs ---

def run_ours(args):
    import torch
    import madmax_b200 as mb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    mb.check(mb.lib().sp_init(local), "sp_init")
    # a real stream: events and the library's launches must share it (the
    # legacy default stream's handle is 0, which the library reads as "its
    # own stream")
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sptr = C.c_void_p(stream.cuda_stream)
    assert sptr.value, "expected a non-default stream"

    descs = workload_descs(mb, args.nrve, rank_seed(rank), tuple(args.sizes))
    sizes = [d.n[0] for d in descs]
    t0 = time.time()
    batch = mb.Batch(descs, nrhs=6, threads=args.threads, ctas_per_sm=args.ctas,
                     cluster=args.cluster, inner_rtol=args.inner_rtol,
                     op=mb.SP_OP_STENCIL if args.op == "stencil" else mb.SP_OP_ELL)
    setup_s = time.time() - t0
    shape = batch.shape()
    tuned = batch.tune_report()

    for _ in range(args.warmup):
        batch.launch(sptr)
    torch.cuda.synchronize()

    # ---- device-resident timing (value) ----
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    evs[0].record(stream)
    for k in range(args.steps):
        batch.launch(sptr)
        evs[k + 1].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    per_launch_ms = [evs[k].elapsed_time(evs[k + 1]) for k in range(args.steps)]
    total_ms = max_over_ranks(dist, sum(per_launch_ms), "cuda")
    value = whole_job_rate(world, args.nrve, args.steps, total_ms)

    stress = np.zeros((args.nrve, 6, 6))
    info = (mb.sp_solve_info * args.nrve)()
    batch.download(stress, None, info, sptr)
    torch.cuda.synchronize()
    inf = mb.info_array(info)
    converged = bool((inf["status"] == 0).all())

    # ---- end to end through the C ABI with host buffers ----
    pin = lambda shape: torch.zeros(shape, dtype=torch.float64, pin_memory=True).numpy()
    h_strain = pin((args.nrve, 6, 6))
    for i in range(args.nrve):
        h_strain[i] = np.eye(6)
    h_mats = pin((args.nrve, 4))
    for i, d in enumerate(descs):
        h_mats[i] = (d.E[0], d.nu[0], d.E[1], d.nu[1])
    h_stress = pin((args.nrve, 6, 6))
    h_info = (mb.sp_solve_info * args.nrve)()
    ee = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.e2e_steps)]
    torch.cuda.synchronize()
    for k in range(args.e2e_steps):
        ee[2 * k].record(stream)
        batch.upload(h_strain, h_mats, sptr)
        batch.launch(sptr)
        batch.download(h_stress, None, h_info, sptr)
        ee[2 * k + 1].record(stream)
        stream.synchronize()
    e2e_ms = max_over_ranks(dist, sum(ee[2 * k].elapsed_time(ee[2 * k + 1])
                                       for k in range(args.e2e_steps)), "cuda")
    e2e_value = whole_job_rate(world, args.nrve, args.e2e_steps, e2e_ms)
    h2d = h_strain.nbytes + h_mats.nbytes
    d2h = h_stress.nbytes + C.sizeof(h_info)

    line = None
    if rank == 0:
        abytes = algorithmic_bytes(sizes, inf["inner"], inf["outer"], stencil=args.op == "stencil")
        traffic, traffic_src = profiled_traffic("k_batch", " ".join(argv_tail(args)))
        avg_ms = total_ms / args.steps
        achieved = abytes / (avg_ms / 1000.0) / 1e9
        peak, peak_kind = measured_peak()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": avg_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 CG + f64 refinement", "data": "synthetic",
            "config": {**workload_config(args, sizes),
                       "precision": "mixed", "cta_threads": shape[0], "ctas_per_sm": shape[1],
                       "persistent_grid": shape[2],
                       "cluster": args.cluster, "inner_rtol": args.inner_rtol,
                       "shape_source": "autotuner" if tuned else "given",
                       "operator": args.op,
                       "l2": l2_note(args, sizes, batch),
                       "parallelism": f"replicas x{world} (independent RVEs per rank)"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": traffic, "traffic_source": traffic_src,
                         "algorithmic_bytes": abytes,
                         "peak_kind": peak_kind, "kernel": "k_batch (persistent)"},
            "clocks": clocks,
            "converged": converged, "max_relres": float(inf["relres"].max()),
            "autotuner": tuned,
            "solve": {"converged": converged, "max_relres": float(inf["relres"].max()),
                      "mean_inner_its": float(inf["inner"].mean()),
                      "mean_outer_its": float(inf["outer"].mean()),
                      "rhs_solves_per_s": 6 * value, "setup_s": setup_s},
        }
        if world == 1 and args.oracle_sample > 0:
            oc = oracle_check(descs, stress, args.oracle_sample)
            line["oracle_err"] = oc
            line["oracle_err_max"] = oc["max"]
            line["oracle_err_p99"] = oc["p99"]
        if world == 1 and not args.no_spmv:
            line["spmv"] = measure_spmv(mb, stream, sptr)
        if world == 1 and not args.no_plain:
            line["plain_gpu"] = plain_gpu(mb, descs, args)
            line["plain_gpu"]["batched_speedup"] = value / line["plain_gpu"]["value"]
            line["batched_speedup"] = line["plain_gpu"]["batched_speedup"]
        if world == 1 and not args.no_ell:
            line["ell_batch"] = ell_batch(mb, descs, args, stream, sptr)
            if "plain_gpu" in line:
                line["ell_batch"]["batched_speedup"] = (line["ell_batch"]["value"] /
                                                        line["plain_gpu"]["value"])
        if world == 1 and not args.no_serve:
            sv = serving(mb, args)
            line["serving"] = sv
            # the metric's latency half at the top level: the lowest arrival
            # rate's p50/p99 in both warm-start modes and for the plain path
            low = str(args.serve_rates[0])
            line["serve_p50_ms"] = sv["warm_last"]["rates"][low]["p50_ms"]
            line["serve_p99_ms"] = sv["warm_last"]["rates"][low]["p99_ms"]
            line["serve_predict_p50_ms"] = sv["predict"]["rates"][low]["p50_ms"]
            line["serve_predict_p99_ms"] = sv["predict"]["rates"][low]["p99_ms"]
            line["plain_serve_p50_ms"] = sv["plain"]["p50_ms"]
            line["plain_serve_p99_ms"] = sv["plain"]["p99_ms"]
            line["serve_speedup_vs_plain"] = sv["speedup_vs_plain"]["warm_last"]
        if world == 1 and not args.no_fe2:
            line["fe2"] = fe2_step(mb, args)
        if world == 1 and not args.no_cpu:
            items = workload_items(args.nrve, rank_seed(rank), tuple(args.sizes))
            per, wall, res = cpu_sample(per_size_sample(items, args.cpu_sample), 1)
            line["cpu_baseline"] = {
                "value": mix_rate(per), "unit": UNIT, "cores": 1, "kind": "port",
                "sample": f"{len(res)} RVEs of the timed workload ({args.cpu_sample} of each size), "
                          f"FP64 Jacobi-PCG oracle from the reference's zero start on 1 core "
                          f"({wall:.1f} s), rate = 1 / mean over sizes of s per RVE"}
    batch.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if line:
        print(json.dumps(line), flush=True)


def serve_geometries(mb, ngeom: int, seed: int):
    """256 resident geometries, n uniform in 8..32, fibers and materials as
    in the batched workload."""
    rng = np.random.default_rng(seed)
    n = rng.integers(8, 33, size=ngeom)
    radius = rng.uniform(0.1, 0.35, size=ngeom)
    ratio = np.exp(rng.uniform(np.log(2.0), np.log(100.0), size=ngeom))
    nu_m = rng.uniform(0.2, 0.35, size=ngeom)
    nu_f = rng.uniform(0.2, 0.35, size=ngeom)
    return [mb.rve_desc(int(n[i]), float(radius[i]), (E_MATRIX, E_MATRIX * float(ratio[i])),
                        (float(nu_m[i]), float(nu_f[i]))) for i in range(ngeom)]


def fe2_step(mb, args):
    """A full FE2 step: 40x10x10 hex8 cantilever (14,883 dof, 32,000 Gauss
    points), tip traction 1e6 Pa, every Gauss point bound to one of 64
    seeded RVEs (n = 16, fibre radius U(0.15, 0.3), matrix E 1e9 nu 0.3,
    fibre E 1e10 nu 0.2), FP64 macro solve; micro answers from the serving
    loop.  Three runs: the linear micro mode (one FD tangent per RVE, the
    reference micro's own behaviour for linear materials) with the
    reference's 1e-6 strain clip, the same without the clip, and one serving
    request per Gauss point per Newton iteration (32,000 per iteration)."""
    rng = np.random.default_rng(5150)
    rves = [mb.rve_desc(16, float(rng.uniform(0.15, 0.3)), (1e9, 1e10), (0.3, 0.2))
            for _ in range(64)]

    def one(label, its, **kw):
        t0 = time.perf_counter()
        f = mb.Fe2(rves, newton_its=its, **kw)
        setup = time.perf_counter() - t0
        t0 = time.perf_counter()
        info = f.run()
        step = time.perf_counter() - t0
        f.close()
        bn = [info.bnorm[i] for i in range(info.newton_its)]
        r = {"mode": label, "newton_its": info.newton_its, "setup_s": setup, "step_s": step,
             "bnorm": bn, "final_rel_residual": bn[-1] / bn[0],
             "pcg_its": [info.pcg_its[i] for i in range(info.newton_its)],
             "tip_displacement": list(info.tip), "micro_requests": info.micro_requests,
             "device_ms": {"residual": info.residual_ms, "assemble": info.assemble_ms,
                           "solve": info.solve_ms}}
        if info.micro_s > 0:
            r["micro_s"] = info.micro_s
            r["micro_requests_per_s"] = info.micro_requests / info.micro_s
        return r

    # without the clip the loop converges; it stops once ||b|| <= 1e-6 N (1e-11
    # of the first residual), since a right-hand side at the round-off level
    # of the internal forces cannot be reduced by the macro PCG's relative
    # tolerance
    tol = 1e-6
    out = {"macro": "40x10x10 hex8 cantilever, 14883 dof, 32000 Gauss points, traction 1e6 Pa",
           "rves": "64 x n=16 (seeded)",
           "linear_clip": one("linear micro, strain clip 1e-6 (macro/src/assembly.c:319)", 5),
           "linear_noclip": one("linear micro, no strain clip", 5, strain_clip=0.0,
                                newton_tol=tol)}
    if not args.no_fe2_per_gp:
        out["per_gauss_point"] = one("one serving request per Gauss point per iteration, "
                                     "no strain clip", 5, micro=mb.SP_FE2_PER_GP,
                                     strain_clip=0.0, newton_tol=tol)
    return out


def serve_traces(args, ngeom: int, seed: int = 99):
    """Poisson traces, one per arrival rate: (rate, arrival times, geometry
    ids, strains N(0, 1e-3))."""
    rng = np.random.default_rng(seed)
    out = []
    for lam in args.serve_rates:
        nreq = int(min(args.serve_max_req, max(200, lam * args.serve_seconds)))
        t_arr = np.cumsum(rng.exponential(1.0 / lam, size=nreq))
        out.append((lam, t_arr, rng.integers(0, ngeom, size=nreq),
                    rng.normal(0, 1e-3, size=(nreq, 6))))
    return out


def serve_mode(mb, geoms, traces, warm_start):
    """One server over the resident geometries: a cold first request on every
    geometry, then every trace replayed open-loop (arrivals on the host clock,
    completion times from the done flags)."""
    t0 = time.time()
    srv = mb.Server(geoms, hbm_budget=150 * 10 ** 9, warm_start=warm_start)
    setup = time.time() - t0
    srv.start()
    rng = np.random.default_rng(7)
    g0 = np.arange(len(geoms))
    td0, _, _, info0 = srv.replay(g0, rng.normal(0, 1e-3, (len(geoms), 6)), np.zeros(len(geoms)),
                                  timeout=600)
    out = {"setup_s": setup,
           "cold_first_pass": {"requests": len(geoms), "seconds": float(td0.max()),
                               "solves_per_s": len(geoms) / float(td0.max()),
                               "mean_inner_its": float(np.mean([i.inner_its for i in info0]))},
           "rates": {}}
    for lam, t_arr, geo, eps in traces:
        td, st, tg, info = srv.replay(geo, eps, t_arr, timeout=900)
        lat = (td - t_arr) * 1000.0
        span = td.max() - t_arr.min()
        out["rates"][str(lam)] = {
            "requests": len(t_arr), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "solves_per_s": len(t_arr) / span,
            "all_converged": all(i.status == 0 for i in info),
            "solved_fraction": float(np.mean([i.outer_its > 0 for i in info])),
            "mean_inner_its": float(np.mean([i.inner_its for i in info])),
            "max_relres": float(max(i.relres for i in info))}
    srv.stop()
    srv.close()
    return out


def plain_replay(mb, geoms, trace, nreq: int):
    """The plain comparator, run for real: the first `nreq` requests of a
    trace served one at a time in arrival order by the plain FP64 path
    (sp_rve_homogenize on the geometry's resident ELL matrix, the request's 7
    load cases eps and eps + 0.005 e_i, cold start).  Every geometry the
    sample uses is created and solved once before the replay (resident and
    warm, like the server's); each request starts at max(arrival, previous
    completion) on the host clock."""
    import torch
    lam, t_arr, geo, eps = trace
    t_arr, geo, eps = t_arr[:nreq], geo[:nreq], eps[:nreq]
    rves = {}
    e7 = lambda e: np.vstack([e] + [e + 0.005 * np.eye(6)[i] for i in range(6)])
    for g in sorted(set(int(x) for x in geo)):
        rves[g] = mb.Rve(geoms[g])
        rves[g].homogenize(e7(np.zeros(6)))
    torch.cuda.synchronize()
    done = np.zeros(len(t_arr))
    ok = True
    t0 = time.perf_counter()
    for i in range(len(t_arr)):
        wait = t0 + t_arr[i] - t_arr[0] - time.perf_counter()
        if wait > 0:
            time.sleep(wait)
        _, _, _, info = rves[int(geo[i])].homogenize(e7(eps[i]))
        ok = ok and info.status == 0
        done[i] = time.perf_counter() - t0
    for r in rves.values():
        r.close()
    lat = (done - (t_arr - t_arr[0])) * 1000.0
    return {"rate": lam, "requests": len(t_arr), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "solves_per_s": len(t_arr) / done.max(),
            "all_converged": ok,
            "path": "sp_rve_homogenize, FP64 ELL + FP64 Jacobi-PCG, one request at a time, "
                    "7 load cases, cold start"}


def serving(mb, args):
    """Open-loop Poisson load on the device-resident server over 256 resident
    geometries, in both warm-start modes, and the plain comparator replayed
    on the first requests of the lowest-rate trace."""
    geoms = serve_geometries(mb, args.serve_geoms, 4321)
    traces = serve_traces(args, len(geoms))
    out = {"geometries": len(geoms), "n_range": [8, 32], "budget_bytes": 150 * 10 ** 9}
    out["warm_last"] = serve_mode(mb, geoms, traces, mb.SP_WARM_LAST)
    out["warm_last"]["warm_start"] = ("each load case starts from the geometry's last solution "
                                      "of it; every request is solved by CG to 1e-8")
    out["predict"] = serve_mode(mb, geoms, traces, mb.SP_WARM_PREDICT)
    out["predict"]["warm_start"] = ("first-order prediction from the geometry's last solved "
                                    "request, verified by the FP64 residual; requests that miss "
                                    "1e-8 are solved")
    plain = plain_replay(mb, geoms, traces[0], args.plain_replay)
    out["plain"] = plain
    # capacity against the plain path: the saturated batched rate (highest
    # arrival rate) over the plain path's rate under its own overload
    top = str(traces[-1][0])
    out["speedup_vs_plain"] = {
        "warm_last": out["warm_last"]["rates"][top]["solves_per_s"] / plain["solves_per_s"],
        "predict": out["predict"]["rates"][top]["solves_per_s"] / plain["solves_per_s"],
        "at_rate": traces[-1][0]}
    return out


def ell_batch(mb, descs, args, stream, sptr, steps: int = 2):
    """The same mix on the assembled operator (SP_OP_ELL): every launch
    assembles each RVE's FP32 ELL values (8-colour scatter, node-sliced
    copy) and runs the FP32 CG on them, FP64 refinement as in the headline.
    One warm-up launch, then `steps` launches timed with CUDA events."""
    import torch
    t0 = time.time()
    b = mb.Batch(descs, nrhs=6, inner_rtol=args.inner_rtol, op=mb.SP_OP_ELL)
    setup = time.time() - t0
    try:
        b.launch(sptr)
        torch.cuda.synchronize()
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        evs[0].record(stream)
        for k in range(steps):
            b.launch(sptr)
            evs[k + 1].record(stream)
        torch.cuda.synchronize()
        ms = sum(evs[k].elapsed_time(evs[k + 1]) for k in range(steps)) / steps
        info = (mb.sp_solve_info * len(descs))()
        b.download(None, None, info, sptr)
        torch.cuda.synchronize()
        inf = mb.info_array(info)
        shape = b.shape()
        return {"value": len(descs) / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms,
                "steps": steps, "operator": "assembled FP32 ELL (node-sliced), assembly in the launch",
                "cta_threads": shape[0], "ctas_per_sm": shape[1],
                "converged": bool((inf["status"] == 0).all()),
                "max_relres": float(inf["relres"].max()),
                "mean_inner_its": float(inf["inner"].mean()),
                "device_bytes": b.device_bytes(), "setup_s": setup}
    finally:
        b.close()


def plain_gpu(mb, descs, args):
    """The plain path: one RVE at a time, FP64 ELL + FP64 Jacobi-PCG, every
    step a grid-wide kernel (sp_rve_tangent), on a sample of the workload."""
    import torch
    per = {s: [] for s in SIZES}
    picked = []
    for s in SIZES:
        picked += [d for d in descs if d.n[0] == s][:args.plain_per_size]
    for d in picked:
        r = mb.Rve(d)
        r.tangent()  # warm (graph build)
        torch.cuda.synchronize()
        t = time.perf_counter()
        r.tangent()
        per[d.n[0]].append(time.perf_counter() - t)
        r.close()
    return {"value": mix_rate(per), "unit": UNIT,
            "sample": f"{len(picked)} RVEs ({args.plain_per_size} per size), FP64, one RVE "
                      "per solve, 6 load cases per solve, host wall time per tangent",
            "s_per_rve": {str(k): float(np.mean(v)) for k, v in per.items() if v}}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nrve", type=int, default=4096)
    ap.add_argument("--threads", type=int, default=0, help="threads per CTA (0: the library's choice)")
    ap.add_argument("--ctas", type=int, default=0, help="CTAs per SM (0: the library's choice)")
    ap.add_argument("--cluster", type=int, default=1)
    ap.add_argument("--inner-rtol", type=float, default=3e-3,
                    help="CG residual reduction per refinement step (the library's mixed-precision default)")
    ap.add_argument("--op", default="stencil", choices=["stencil", "ell"],
                    help="inner CG operator: element-type stencil or assembled ELL values")
    ap.add_argument("--sizes", type=int, nargs="+", default=list(SIZES),
                    help="mesh sizes to draw from (the headline workload uses 8 12 16 20)")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--plain-per-size", type=int, default=16)
    ap.add_argument("--oracle-sample", type=int, default=8,
                    help="RVEs per mesh size checked against the oracle after timing")
    ap.add_argument("--no-ell", action="store_true",
                    help="skip the assembled-ELL batched rate on the same mix")
    ap.add_argument("--cpu-sample", type=int, default=2,
                    help="RVEs of each mesh size timed on the CPU oracle (1 core)")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-spmv", action="store_true")
    ap.add_argument("--no-fe2", action="store_true")
    ap.add_argument("--no-fe2-per-gp", action="store_true",
                    help="skip the FE2 run with a serving request per Gauss point")
    ap.add_argument("--serve-geoms", type=int, default=256)
    ap.add_argument("--serve-rates", type=float, nargs="+", default=[1e3, 1e4, 1e5])
    ap.add_argument("--serve-seconds", type=float, default=2.0)
    ap.add_argument("--serve-max-req", type=int, default=4000)
    ap.add_argument("--plain-replay", type=int, default=200,
                    help="requests of the lowest-rate trace served by the plain path")
    args = ap.parse_args(argv)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
