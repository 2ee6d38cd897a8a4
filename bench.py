"""Benchmark of the per-timestep GRMHD update: zone-updates/s on the 3-D magnetised torus.

A "step" is one full RK2 timestep (two advance() substeps with bounds and fixups) of the
Fishbone-Moncrief torus on one grid.  Default workload: 384 x 192 x 128 zones (r, theta,
phi), WENO5, HLL, Toth flux-CT, mixed precision (FP32 reconstruction/HLL/CT, FP64 update and
inversion) with the learned starting point of the inversion, initial state built on the
host (synthetic, seeded).  Before the timed region the plain method runs a few steps and
dumps its (U, P) pairs, and the network is trained on them on the GPU.  The plain FP64
device path and the mixed path with the plain guess are timed on the same grid beside it.

Multi-GPU: the torus update does not shard in this build (one GPU per grid), so
`--gpus N` runs N independent replicas, one per rank, and reports their aggregate.

`--impl reference` times the reference HARM code itself (built from its sources into
oracle/_ref/, OpenMP on all host cores, FP64) on a bounded sample of the same workload: the
192 x 96 x 64 torus with the same reconstruction, flux formula and flux-CT.  At 384 x 192 x 128
the reference's static arrays need 117 GB of host memory and its initialisation (metric and
connection per cell) takes some twenty minutes, so its rate per zone-update is measured on
the grid an eighth that size.  Where that binary is absent or does not fit the host's
memory, the CPU restatement of the algorithm (oracle/, OpenMP) is timed on a slab instead.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

CONFIGS = {
    # name: (n1, n2, n3, lim) -- the reconstruction of each torus configuration: WENO5 in 3-D,
    # MC for the 2-D CPU-runnable case
    "torus3d_384x192x128": (384, 192, 128, 2),
    "torus3d_256x128x64": (256, 128, 64, 2),
    "torus3d_192x96x64": (192, 96, 64, 2),
    "torus2d_128x128": (128, 128, 1, 0),
}
LIMNAME = {0: "mc", 1: "ppm", 2: "weno5", 3: "paraline"}
LIMS = {"mc": 0, "ppm": 1, "weno5": 2, "paraline": 3}
FLUXES = {"hll": 0, "laxf": 1}
METRIC = "zone-updates/s on 3D torus: learned+mixed vs plain FP64 GPU at L1 err≤1e-6"


def bytes_per_zone_update(n3: int) -> float:
    """Algorithmic HBM bytes of one zone-update of the full RK2 step: FP64 state traffic
    322 B (substep 0: read P^n, write P^(n+1/2); substep 1: read P^n, P^(n+1/2), write
    P^(n+1); two flag writes) plus the per-(i,j) metric tables (~1400 B per substep, reused
    along phi) divided by n3."""
    return 322.0 + 2800.0 / n3


def update_kernel_bytes_per_cell(n3: int, precision: int) -> float:
    """Algorithmic bytes of the update+inversion kernel per active cell: p_i, p_b (64 B
    each), the five non-field fluxes of three directions and three EMFs (FP64: 8 B, mixed:
    4 B each), p_f (64 B), the flag (1 B) and the CENT metric, connection and floors
    (94 doubles per (i,j), reused along phi)."""
    w = 8 if precision == 0 else 4
    return 64 + 64 + 15 * w + 3 * w + 64 + 1 + 94 * 8 / n3


def flux_bytes_per_cell(n3: int, precision: int, lim: str = "weno5") -> float:
    """Algorithmic bytes of the flux stage per active cell: each direction reads the 8 FP64
    primitives once (64 B) and writes 8 fluxes (FP32 in the mixed path: 32 B, FP64: 64 B),
    plus the face metric record (28 values per (i,j), reused along phi).  WENO5 adds the cell
    pass: it reads the primitives once (64 B) and writes the 9 dP line quantities, of which
    each direction reads back its 3."""
    w = 4 if precision == 1 else 8
    b = 3 * (64 + 8 * w + 28 * w / n3)
    if lim == "weno5":
        b += 64 + 9 * w + 3 * 3 * w
    return b


# DRAM traffic of the flux stage (k_cellprep and three k_fluxt launches; ncu dram__bytes_read.sum +
# dram__bytes_write.sum) per active cell, measured on the 192x96x64 torus and scaled to a
# workload by its cell count
FLUX_TRAFFIC_PER_CELL = {("weno5", "mixed"): 449.0}


def clock_sampler(stop: threading.Event, out: list, dev: int):
    cmd = ["nvidia-smi", "-i", str(dev), "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
           "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
           "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
           "--format=csv,noheader,nounits", "-lms", "200"]
    try:
        p = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    except OSError:
        return
    try:
        while not stop.is_set():
            line = p.stdout.readline()
            if not line:
                break
            out.append(line.strip())
    finally:
        p.terminate()
        try:
            p.wait(timeout=2)
        except Exception:
            p.kill()


def summarize_clocks(lines: list) -> dict:
    sm, mx, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for ln in lines:
        f = [x.strip() for x in ln.split(",")]
        if len(f) < 7:
            continue
        try:
            sm.append(float(f[0]))
            mx.append(float(f[1]))
        except ValueError:
            continue
        for nm, v in zip(names, f[3:7]):
            if v.lower().startswith("active"):
                reasons.add(nm)
    return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
            "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "src": "measured"}
    return {"hbm_gbs": 6650.0, "src": "fallback"}


def dist_init(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# the reference binary the CPU legs time: the 192x96x64 torus built with MAXBND 6 (the ghost
# width WENO5BND needs; MC, PPM and PARALINE run on it unchanged)
REF_SAMPLE = (192, 96, 64, 6)
REF_STATIC_BYTES = 17.5e9   # its static arrays (bss), which the host must hold


def reference_binary_time(args, lim, nsteps) -> dict | None:
    """Rate of the reference HARM code itself on the host cores (oracle/_ref/): `nsteps` full
    RK2 steps of the REF_SAMPLE torus after its initialisation and one untimed step.  None
    where the binary is absent or the host's memory is too small for it."""
    from oracle import ref as R
    n1, n2, n3, ng = REF_SAMPLE
    if not R.available(n1, n2, n3, ng):
        return None
    try:
        mem = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES")
    except (ValueError, OSError):
        mem = 0
    if mem < 1.25 * REF_STATIC_BYTES:
        return None
    cores = os.cpu_count() or 1
    r = R.time_steps(n1, n2, n3, ng, lim, FLUXES[args.flux], nsteps, cores, timeout=1800)
    return {"value": r["zone_cycles_per_s"], "unit": "zone-updates/s", "cores": cores, "kind": "reference",
            "sample": f"the reference HARM code (its own sources, OpenMP, FP64) on the {n1}x{n2}x{n3} torus, "
                      f"{LIMNAME[lim]} + {args.flux} + flux-CT, {r['steps']} full RK2 steps after its init and "
                      f"one untimed step ({r['seconds']:.1f} s)"}


def run_reference(args, ws, rank):
    """CPU baseline arm (rank 0 only): the reference HARM code on all host cores (a bounded
    number of steps of the REF_SAMPLE torus), else the oracle restatement on a slab."""
    if rank != 0:
        return
    n1, n2, n3, lim = CONFIGS[args.config]
    lim = LIMS.get(args.lim, lim)
    ksteps = max(1, min(args.steps, args.ref_max_steps))
    ref = reference_binary_time(args, lim, ksteps)
    if ref is not None:
        line = {
            "impl": "reference", "metric": METRIC, "value": ref["value"], "unit": "zone-updates/s", "n_gpus": ws,
            "steps": ksteps, "warmup": 1, "ms_per_step": 1e3 * REF_SAMPLE[0] * REF_SAMPLE[1] * REF_SAMPLE[2]
            / ref["value"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (the reference's own seeded Fishbone-Moncrief torus)",
            "config": {"workload": args.config + f"_{LIMNAME[lim]}_{args.flux}_fluxct",
                       "sample_grid": list(REF_SAMPLE[:3])},
            "cpu_baseline": ref,
            "e2e": {"value": ref["value"], "unit": "zone-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return
    from harm_harm_b200 import Grid
    from oracle import oracle as O
    sn3 = min(n3, args.cpu_sample_n3)
    g = Grid.torus(n1, n2, sn3, lim=lim, fluxmethod=FLUXES[args.flux])
    geom, conn, aux = g.geometry()
    P = g.torus_init(geom, aux, seed=args.seed)
    cores = os.cpu_count() or 1
    orc = O.Oracle(g, geom, conn, aux, nthreads=cores)
    orc.bound_prim(P)
    F = [np.zeros_like(P) for _ in range(3)]
    ndt = orc.fluxcalc(P, *F)
    dt = 1.0 / sum(1.0 / x for x in ndt if x < 1e99)
    for _ in range(args.warmup):
        dt, _ = orc.step_ch(P, dt)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        dt, _ = orc.step_ch(P, dt)
    el = time.perf_counter() - t0
    zones = n1 * n2 * sn3
    value = zones * args.steps / el
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "zone-updates/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Fishbone-Moncrief torus, host-built)",
        "config": {"workload": args.config + f"_{LIMNAME[lim]}_{args.flux}_fluxct", "sample_n3": sn3},
        "cpu_baseline": {"value": value, "unit": "zone-updates/s", "cores": cores, "kind": "port",
                         "sample": f"{n1}x{n2}x{sn3} zones of the same torus, full RK2 steps, FP64"},
        "e2e": {"value": value, "unit": "zone-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline_sample(args, lim) -> dict:
    """Bounded timing on the host cores for our own line: the reference HARM code on the
    REF_SAMPLE torus (a few steps), else the CPU port on a slab of the workload."""
    if args.cpu_baseline == "reference":
        ref = reference_binary_time(args, lim, args.cpu_ref_steps)
        if ref is not None:
            return ref
    from harm_harm_b200 import Grid
    from oracle import oracle as O
    n1, n2, n3, _ = CONFIGS[args.config]
    sn3 = min(n3, args.cpu_sample_n3)
    g = Grid.torus(n1, n2, sn3, lim=lim, fluxmethod=FLUXES[args.flux])
    geom, conn, aux = g.geometry()
    P = g.torus_init(geom, aux, seed=args.seed)
    cores = os.cpu_count() or 1
    orc = O.Oracle(g, geom, conn, aux, nthreads=cores)
    orc.bound_prim(P)
    F = [np.zeros_like(P) for _ in range(3)]
    ndt = orc.fluxcalc(P, *F)
    dt = 1.0 / sum(1.0 / x for x in ndt if x < 1e99)
    dt, _ = orc.step_ch(P, dt)
    nst, t0 = 0, time.perf_counter()
    while True:
        dt, _ = orc.step_ch(P, dt)
        nst += 1
        el = time.perf_counter() - t0
        if el > args.cpu_seconds or nst >= 50:
            break
    return {"value": n1 * n2 * sn3 * nst / el, "unit": "zone-updates/s", "cores": cores, "kind": "port",
            "sample": f"{nst} RK2 steps of a {n1}x{n2}x{sn3} slab of the torus, FP64, OpenMP ({el:.1f} s)"}


def train_guess(dev, Pd, dt0, prec, args):
    """The plain method runs `train_steps` steps from the initial state; after each, its
    (U, P) pairs are dumped (every `stride`-th cell); `synth_pairs` synthetic states on the
    grid's metric are added (harm_b200_mlp_synth: rho, u/rho, sigma log-uniform, Lorentz factor
    uniform to 50, isotropic directions); the network is trained on both."""
    import torch
    from harm_harm_b200 import HARM_GUESS_PREV
    g = dev.grid.g
    ncell = g.n1 * g.n2 * g.n3
    stride = max(1, (ncell * args.train_steps) // args.train_pairs)
    cap = ncell // stride + 1
    nsyn = max(0, args.synth_pairs)
    feat = torch.zeros((cap * args.train_steps + nsyn, 10), device="cuda", dtype=torch.float32)
    targ = torch.zeros((cap * args.train_steps + nsyn, 2), device="cuda", dtype=torch.float32)
    P = Pd.clone()
    dt, n = dt0, 0
    t0 = time.perf_counter()
    for s in range(args.train_steps):
        dt, _ = dev.step_ch(P, dt, precision=prec, guess=HARM_GUESS_PREV, stats=False)
        n += dev.mlp_dump(P, feat[n:n + cap], targ[n:n + cap], stride=stride, phase=s % stride)
    del P
    ndump = n
    if nsyn:
        dev.mlp_synth(feat[n:n + nsyn], targ[n:n + nsyn], seed=args.seed)
        n += nsyn
    feat, targ = feat[:n].contiguous(), targ[:n].contiguous()
    norm = torch.zeros(24, device="cuda", dtype=torch.float32)
    params = torch.zeros(9154, device="cuda", dtype=torch.float32)
    dev.mlp_norm(feat, targ, norm)
    dev.mlp_init(params, seed=args.seed)
    t1 = time.perf_counter()
    hist = dev.mlp_train(feat, targ, norm, params, steps=args.train_iters, batch=8192, lr=3e-3, seed=args.seed)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    dev.mlp_set(params, norm, args.start_bias)
    return {"pairs": n, "dumped_pairs": ndump, "synthetic_pairs": nsyn, "dump_steps": args.train_steps, "dump_stride": stride, "adam_steps": args.train_iters,
            "batch": 8192, "dump_s": round(t1 - t0, 3), "train_s": round(t2 - t1, 3),
            "loss_first": float(hist[0]), "loss_last100": float(hist[-100:].mean()), "start_bias": args.start_bias}


def divb_max(g, geom_cent_gdet, P):
    """max of Toth's corner divergence of sqrt(-g) B (the quantity flux-CT keeps at round-off)
    over the corners whose cells are all active in x1 and x2 (x3 is periodic), absolute and
    relative to max |sqrt(-g) B| / min(dx); P on the device"""
    import torch
    gg = g.g
    U = P[5:8] * geom_cent_gdet[None, None]
    ng, ng3, n1, n2, n3 = gg.ng, gg.ng3, gg.n1, gg.n2, gg.n3
    dx = gg.dx

    def sl(a, dk, dj, di):
        return a[ng3 + dk:ng3 + dk + n3 + 1, ng + 1 + dj:ng + dj + n2, ng + 1 + di:ng + di + n1]

    if n3 == 1:
        u1, u2 = U[0, 0], U[1, 0]
        s2 = (lambda a, dj, di: a[ng + 1 + dj:ng + dj + n2, ng + 1 + di:ng + di + n1])
        div = (0.5 * (s2(u1, 0, 0) + s2(u1, -1, 0) - s2(u1, 0, -1) - s2(u1, -1, -1)) / dx[1]
               + 0.5 * (s2(u2, 0, 0) + s2(u2, 0, -1) - s2(u2, -1, 0) - s2(u2, -1, -1)) / dx[2])
        scale = float(U[:2].abs().max()) / min(dx[1], dx[2])
    else:
        u1, u2, u3 = U[0], U[1], U[2]
        div = (0.25 * (sl(u1, 0, 0, 0) + sl(u1, 0, -1, 0) + sl(u1, -1, 0, 0) + sl(u1, -1, -1, 0)
                       - sl(u1, 0, 0, -1) - sl(u1, 0, -1, -1) - sl(u1, -1, 0, -1) - sl(u1, -1, -1, -1)) / dx[1]
               + 0.25 * (sl(u2, 0, 0, 0) + sl(u2, 0, 0, -1) + sl(u2, -1, 0, 0) + sl(u2, -1, 0, -1)
                         - sl(u2, 0, -1, 0) - sl(u2, 0, -1, -1) - sl(u2, -1, -1, 0) - sl(u2, -1, -1, -1)) / dx[2]
               + 0.25 * (sl(u3, 0, 0, 0) + sl(u3, 0, 0, -1) + sl(u3, 0, -1, 0) + sl(u3, 0, -1, -1)
                         - sl(u3, -1, 0, 0) - sl(u3, -1, 0, -1) - sl(u3, -1, -1, 0) - sl(u3, -1, -1, -1)) / dx[3])
        scale = float(U.abs().max()) / min(dx[1], dx[2], dx[3])
    m = float(torch.abs(div).max())
    return m, m / max(scale, 1e-300)


def vector_errors(gc, a, b):
    """L1 and Linf of the difference of two spatial vector fields relative to the first, each
    measured by its metric length sqrt(g_ij x^i x^j); gc: CENT metric records [28][1][n2][n1],
    a, b: [3][n3][n2][n1]"""
    g11, g12, g13, g22, g23, g33 = gc[4], gc[5], gc[6], gc[7], gc[8], gc[9]

    def length(x):
        q = (g11 * x[0] * x[0] + g22 * x[1] * x[1] + g33 * x[2] * x[2]
             + 2.0 * (g12 * x[0] * x[1] + g13 * x[0] * x[2] + g23 * x[1] * x[2]))
        return np.sqrt(np.maximum(q, 0.0))

    la, ld = length(a), length(a - b)
    return float(ld.mean() / max(la.mean(), 1e-300)), float(ld.max() / max(la.max(), 1e-300))


def run_ours(args, ws, rank, local):
    import torch
    from harm_harm_b200 import (HARM_GUESS_MLP, HARM_GUESS_PREV, HARM_PREC_FP64, HARM_PREC_FP64_FMA, HARM_PREC_MIXED,
                                Grid, Harm)
    torch.cuda.set_device(local)
    n1, n2, n3, lim = CONFIGS[args.config]
    lim = LIMS.get(args.lim, lim)
    g = Grid.torus(n1, n2, n3, lim=lim, fluxmethod=FLUXES[args.flux])
    geom, conn, aux = g.geometry()
    P0 = g.torus_init(geom, aux, seed=args.seed + rank)
    dev = Harm(g, geom, conn, aux, device=local)
    prec = HARM_PREC_MIXED if args.precision == "mixed" else HARM_PREC_FP64
    guess = HARM_GUESS_MLP if args.guess == "mlp" else HARM_GUESS_PREV
    Pd = torch.from_numpy(P0).cuda()
    dev.bound_prim(Pd)
    torch.cuda.synchronize()
    # initial dt from the fluxes of the initial state
    F = [torch.empty_like(Pd) for _ in range(3)]
    ndt = dev.fluxcalc(Pd, *F)
    del F
    dt0 = 1.0 / sum(1.0 / x for x in ndt if x < 1e99)
    stream = torch.cuda.ExternalStream(dev.stream_ptr)
    zones = n1 * n2 * n3
    mlp_info = train_guess(dev, Pd, dt0, prec, args) if guess == HARM_GUESS_MLP else None

    def timed(precision, gs, P, K, W):
        dt = dt0
        dt, _ = dev.step_ch(P, dt, precision=precision, guess=gs, nsteps=W, stats=False)
        barrier(ws)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = dev.launches
        e0.record(stream)
        dt, st = dev.step_ch(P, dt, precision=precision, guess=gs, nsteps=K, stats=True)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(ws)
        ms = e0.elapsed_time(e1)
        return ms, st, dev.launches - l0

    # plain FP64 path on the same grid: the FP64 build at its best speed (FMA contraction,
    # shared reciprocals in the inversion) is the denominator of the speed-up; the
    # IEEE-ordered FP64 build (the one the parity tests pin) is timed beside it
    Pf = Pd.clone()
    k64 = max(1, args.steps // 2)
    ms64, st64, _ = timed(HARM_PREC_FP64_FMA, HARM_GUESS_PREV, Pf, k64, args.warmup)
    Pf.copy_(Pd)
    k64i = max(1, args.steps // 8)
    ms64i, _, _ = timed(HARM_PREC_FP64, HARM_GUESS_PREV, Pf, k64i, args.warmup)
    del Pf
    # the headline precision with the plain guess
    if guess == HARM_GUESS_MLP:
        Pp = Pd.clone()
        msp, stp, _ = timed(prec, HARM_GUESS_PREV, Pp, args.steps, args.warmup)
        del Pp
    # headline path, with clocks sampled during the timed region
    stop, clines = threading.Event(), []
    th = threading.Thread(target=clock_sampler, args=(stop, clines, local), daemon=True)
    th.start()
    Pm = Pd.clone()
    ms, st, launches = timed(prec, guess, Pm, args.steps, args.warmup)
    stop.set()
    th.join(timeout=5)
    ms = max_over_ranks(ms, ws)
    ms64 = max_over_ranks(ms64, ws)
    ms64i = max_over_ranks(ms64i, ws)
    value = ws * zones * args.steps / (ms * 1e-3)
    value64 = ws * zones * k64 / (ms64 * 1e-3)
    value64i = ws * zones * k64i / (ms64i * 1e-3)
    if guess == HARM_GUESS_MLP:
        msp = max_over_ranks(msp, ws)
        value_prev = ws * zones * args.steps / (msp * 1e-3)
    # div B of the headline path's state after its warm-up and timed steps
    divb_abs, divb_rel = divb_max(g, torch.from_numpy(np.ascontiguousarray(geom[0, 26])).to(Pm.device), Pm)
    # accuracy of the headline path against the FP64 path after the same number of steps, each
    # path with its own CFL dt (their states then also differ by the offset of their simulation
    # times), and with the FP64 path's dt sequence for both (the error of the arithmetic alone)
    def steps_of(P, precision, g_, dts=None):
        dt, used = dt0, []
        for s in range(args.err_steps):
            dt_in = dts[s] if dts is not None else dt
            dt, _ = dev.step_ch(P, dt_in, precision=precision, guess=g_, nsteps=1, stats=False)
            used.append(dt_in)
        return used

    Pa, Pb = Pd.clone(), Pd.clone()
    dts64 = steps_of(Pa, HARM_PREC_FP64, HARM_GUESS_PREV)
    dtsm = steps_of(Pb, prec, guess)
    act = (slice(None),) + g.active
    a, b = Pa.cpu().numpy()[act], Pb.cpu().numpy()[act]
    fields = (("rho", 0), ("u", 1), ("U1", 2), ("U2", 3), ("U3", 4), ("B1", 5), ("B2", 6), ("B3", 7))
    # the velocity and field vectors measured by their length in the metric (|x|^2 = g_ij x^i x^j
    # at the cell centre): a component that is small where the vector is not (u~^2, B^3 of a
    # poloidal loop) is judged against the vector it belongs to
    gc = geom[0][:, g.active[1], g.active[2]][:, None]

    def field_errors(x, y):
        e1 = {nm: float(np.abs(x[pl] - y[pl]).mean() / max(np.abs(x[pl]).mean(), 1e-300)) for nm, pl in fields}
        ei = {nm: float(np.abs(x[pl] - y[pl]).max() / max(np.abs(x[pl]).max(), 1e-300)) for nm, pl in fields}
        for nm, p0 in (("U_vec", 2), ("B_vec", 5)):
            e1[nm], ei[nm] = vector_errors(gc, x[p0:p0 + 3], y[p0:p0 + 3])
        return e1, ei

    l1, linf = field_errors(a, b)
    t_offset = (sum(dtsm) - sum(dts64)) / sum(dts64)
    Pb.copy_(Pd)
    steps_of(Pb, prec, guess, dts64)
    l1_same, linf_same = field_errors(a, Pb.cpu().numpy()[act])
    # the round-off floor of the same evolution: the FP64 build with FMA contraction against
    # the IEEE-ordered one
    Pb.copy_(Pd)
    dev.step_ch(Pb, dt0, precision=HARM_PREC_FP64_FMA, nsteps=args.err_steps, stats=False)
    c = Pb.cpu().numpy()[act]
    l1_fma = {nm: float(np.abs(a[pl] - c[pl]).mean() / max(np.abs(a[pl]).mean(), 1e-300)) for nm, pl in fields[:2]}
    del Pa, Pb
    # stage times and roofline of the dominant kernels
    stages = dev.time_stages(Pm, dt0, precision=prec, guess=guess, reps=3)
    peaks = measured_peaks()
    flux_bytes = flux_bytes_per_cell(n3, prec, LIMNAME[lim]) * zones
    ach_flux = flux_bytes / (stages["flux"] * 1e-3) / 1e9
    upd_bytes = update_kernel_bytes_per_cell(n3, prec) * zones
    ach = upd_bytes / (stages["update_invert"] * 1e-3) / 1e9
    # end to end through the host-buffer entry point: H2D of P, step, D2H of P every step (the
    # copies of consecutive steps overlapped by harm_b200_step_host_n)
    Ph = torch.from_numpy(P0.copy()).pin_memory()
    dev.step_ch_host_n(Ph.numpy(), dt0, precision=prec, guess=guess, nsteps=2)
    torch.cuda.synchronize()
    ke = max(2, args.steps // 4)
    t0 = time.perf_counter()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    dte, _ = dev.step_ch_host_n(Ph.numpy(), dt0, precision=prec, guess=guess, nsteps=ke)
    e1.record(stream)
    torch.cuda.synchronize()
    wall_e2e = time.perf_counter() - t0
    ms_e2e = max(e0.elapsed_time(e1), 1e3 * wall_e2e)
    ms_e2e = max_over_ranks(ms_e2e, ws)
    e2e_value = ws * zones * ke / (ms_e2e * 1e-3)
    # the same with one step per call (harm_b200_step_host: no overlap between the steps' copies)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for _ in range(ke):
        dte, _ = dev.step_ch_host(Ph.numpy(), dte, precision=prec, guess=guess)
    ms_e2e1 = max_over_ranks(1e3 * (time.perf_counter() - t1), ws)
    e2e_one_per_call = ws * zones * ke / (ms_e2e1 * 1e-3)
    pbytes = 8 * g.cells * 8
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(args, lim)
    if rank == 0:
        ninv = max(st["cells_inverted"], 1.0)
        line = {
            "metric": METRIC, "value": value, "unit": "zone-updates/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 flux / f64 update+inversion" if prec == HARM_PREC_MIXED else "f64",
            "data": "synthetic (seeded Fishbone-Moncrief torus, host-built)",
            "config": {"workload": f"{args.config}_{LIMNAME[lim]}_{args.flux}_fluxct_{args.precision}_{args.guess}",
                       "grid": [n1, n2, n3], "reconstruction": LIMNAME[lim], "riemann": args.flux, "ct": "toth",
                       "precision": args.precision, "guess": args.guess,
                       "l2": "inputs larger than L2 (P is %.0f MB)" % (pbytes / 1e6),
                       "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU"},
            "fp64_value": value64, "speedup_vs_fp64": value / value64,
            "fp64_of": "FP64 everywhere, FMA contraction and shared reciprocals (HARM_PREC_FP64_FMA)",
            "fp64_ieee_value": value64i, "speedup_vs_fp64_ieee": value / value64i,
            "plain_guess_value": value_prev if guess == HARM_GUESS_MLP else value,
            "l1_rel_err_vs_fp64": l1, "linf_rel_err_vs_fp64": linf, "err_steps": args.err_steps,
            "sim_time_offset_vs_fp64": t_offset,
            "l1_rel_err_vs_fp64_same_dt": l1_same, "linf_rel_err_vs_fp64_same_dt": linf_same,
            "l1_rel_err_fp64_fma_vs_fp64": l1_fma,
            "divb_max": {"abs": divb_abs, "rel": divb_rel,
                         "of": "Toth corner divergence of sqrt(-g) B after the timed steps, rel to max|sqrt(-g) B|/min dx"},
            "newton_iters_per_cell": st["newton_iters"] / ninv,
            "newton_iters_per_cell_plain_guess": (stp if guess == HARM_GUESS_MLP else st)["newton_iters"]
            / max((stp if guess == HARM_GUESS_MLP else st)["cells_inverted"], 1.0),
            "newton_iters_per_cell_fp64": st64["newton_iters"] / max(st64["cells_inverted"], 1.0),
            "mlp_fallback_rate": st["mlp_fallbacks"] / ninv, "inversion_failures": st["inversion_failures"],
            "mlp_start_rate": st["mlp_cells"] / ninv,
            "mlp_engine": os.environ.get("HARM_B200_MLP_ENGINE", "gated"),
            "mlp_gate": float(os.environ.get("HARM_B200_MLP_GATE", "0.02")),
            "learned_guess": mlp_info,
            "stage_ms": stages,
            "roofline": {"bound": "hbm", "kernel": "k_fluxt (WENO5/PPM/MC reconstruction + HLL, 3 directions)",
                         "achieved": ach_flux, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": ach_flux / peaks["hbm_gbs"], "peak_src": peaks["src"],
                         "traffic": (FLUX_TRAFFIC_PER_CELL[(LIMNAME[lim], args.precision)] * zones
                                     if (LIMNAME[lim], args.precision) in FLUX_TRAFFIC_PER_CELL else None),
                         "unit_of_launch": "one flux stage (the WENO5 cell pass k_cellprep and three k_fluxt "
                                           "launches, all directions)",
                         "algorithmic_bytes_per_cell": flux_bytes_per_cell(n3, prec, LIMNAME[lim]),
                         "limiter": "instruction issue, not HBM: 75 % of issue slots, ALU 56 %, FMA 52 %, "
                                    "DRAM 6 % (ncu, WENO5 FP32 tile kernel, 192x96x64)"},
            "roofline_update_invert": {"bound": "hbm",
                                       "kernel": "conserved update + learned start + k_invert + k_invert_rare",
                                       "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                                       "frac": ach / peaks["hbm_gbs"],
                                       "algorithmic_bytes_per_cell": update_kernel_bytes_per_cell(n3, prec),
                                       "limiter": "FP64 pipe (55 %) and the dependent divisions of the Newton "
                                                  "chain in k_invert; load latency in the conserved passes (ncu)"},
            "step_roofline": {"bytes_per_zone_update": bytes_per_zone_update(n3),
                              "achieved_gbs": value / ws * bytes_per_zone_update(n3) / 1e9,
                              "frac": value / ws * bytes_per_zone_update(n3) / 1e9 / peaks["hbm_gbs"]},
            "e2e": {"value": e2e_value, "unit": "zone-updates/s", "h2d_bytes_per_step": pbytes,
                    "d2h_bytes_per_step": pbytes, "entry_point": "harm_b200_step_host_n",
                    "one_step_per_call_value": e2e_one_per_call},
            "gpu_launches": launches,
            "clocks": summarize_clocks(clines),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    dev.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="torus3d_384x192x128", choices=list(CONFIGS))
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--lim", default="config", choices=["config", "mc", "ppm", "weno5", "paraline"])
    ap.add_argument("--flux", default="hll", choices=list(FLUXES), help="face flux formula (fluxmethod)")
    ap.add_argument("--guess", default="mlp", choices=["prev", "mlp"])
    ap.add_argument("--train-steps", type=int, default=4, help="plain steps whose (U,P) pairs train the guess")
    ap.add_argument("--train-pairs", type=int, default=2000000, help="pairs dumped over those steps")
    ap.add_argument("--train-iters", type=int, default=15000, help="Adam steps of the training")
    ap.add_argument("--synth-pairs", type=int, default=2000000, help="synthetic (U,P) pairs added to the training set")
    ap.add_argument("--start-bias", type=float, default=0.0, help="added to the predicted log(W'/D)")
    ap.add_argument("--seed", type=int, default=12345)
    ap.add_argument("--err-steps", type=int, default=100, help="steps of the mixed-vs-FP64 error measurement")
    ap.add_argument("--cpu-baseline", default="reference", choices=["reference", "port"],
                    help="what our line's cpu_baseline times: the reference binary, or the CPU port")
    ap.add_argument("--cpu-ref-steps", type=int, default=3, help="reference steps timed for cpu_baseline")
    ap.add_argument("--ref-max-steps", type=int, default=10, help="at most this many reference steps per run")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--cpu-sample-n3", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    ws, rank, local = dist_init(args)
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        else:
            run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
