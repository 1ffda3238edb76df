"""Benchmark of the k-space first-order time loop on B200.

Workload (the configuration the headline metric is quoted on): 3-D
heterogeneous absorbing nonlinear kspaceFirstOrder3D at 256^3, dx = 0.2 mm,
blob sound speed (1500 m/s + 8 Gaussian blobs), density 1000 + 0.6 (c - 1500),
alpha_coeff 0.75 dB/(MHz^y cm), alpha_power 1.5, BonA 6, a 64 x 64 plane
pressure source (additive) driven by a 1 MHz 3-cycle Hann-windowed tone burst
at 1 MPa, PML 10, CFL 0.3, Nt = 1000, sensor = the central xy-plane plus a
256-point line along z, recording p and p_max.  Inputs are seeded synthetic
data.

One bench step is one complete simulation (Nt time steps).  ``value`` is the
whole-job throughput in Gcell-steps/s with every input resident on the device
(CUDA events on the library's stream); ``e2e`` is the same metric through the
public kspaceFirstOrder3D call with host arrays (setup, host->device upload,
loop and device->host outputs inside the timed region).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

With --gpus N > 1 (launched by torch.distributed.run) each rank runs an
independent replica on its own GPU: the loop has no exchange between
simulations, so the job is replicas only (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "k-wave-ii_b200"))

METRIC = "Gcell-steps/s (256³ FP32); served p50/p99 vs plain GPU path at ≤1e-4 rel-L2"
UNIT = "Gcell-steps/s"
BYTES_PER_CELL_STEP = 144.0      # 4 B x (6 state reads + 7 state writes + 7 medium + 2 x 8 spectral ops)
BYTES_PER_CELL_SRC_STEP = 8.0    # one more spectral application on source-active steps
HBM_FALLBACK_GBS = 6650.0


def blob_speed(shape, rng, n_blobs=8, pml=10):
    c = np.full(shape, 1500.0)
    axes = [np.arange(s, dtype=np.float64) for s in shape]
    for _ in range(n_blobs):
        ctr = [rng.uniform(pml, s - pml) for s in shape]
        sig = rng.uniform(5.0, 20.0)
        amp = rng.uniform(-100.0, 200.0)
        g = [np.exp(-(a - c0) ** 2 / (2 * sig * sig)) for a, c0 in zip(axes, ctr)]
        c += amp * g[0][:, None, None] * g[1][None, :, None] * g[2][None, None, :]
    return c


def hann_burst(dt, f0=1e6, cycles=3, amp=1e6):
    n = int(math.floor(cycles / f0 / dt + 1e-9)) + 1
    t = np.arange(n) * dt
    w = 0.5 - 0.5 * np.cos(2 * np.pi * np.arange(n) / (n - 1))
    return amp * np.sin(2 * np.pi * f0 * t) * w


def workload(seed=0, N=256, Nt=1000, dx=0.2e-3, pml=10):
    rng = np.random.default_rng(seed)
    shape = (N, N, N)
    c = blob_speed(shape, rng, pml=pml)
    rho = 1000.0 + 0.6 * (c - 1500.0)
    medium = {"sound_speed": c, "density": rho, "alpha_coeff": 0.75, "alpha_power": 1.5, "BonA": 6.0}
    dt = 0.3 * dx / c.max()
    p_mask = np.zeros(shape)
    h = N // 2
    p_mask[pml, h - 32:h + 32, h - 32:h + 32] = 1
    sig = hann_burst(dt)
    source = {"p_mask": p_mask, "p": sig[None, :]}
    sensor_mask = np.zeros(shape)
    sensor_mask[:, :, h] = 1                   # central xy-plane
    sensor_mask[3 * N // 4, h, :] = 1          # 256-point line along z
    sensor = {"mask": sensor_mask, "record": ["p", "p_max"]}
    return dict(shape=shape, dx=dx, Nt=Nt, dt=dt, medium=medium, source=source, sensor=sensor,
                options={"PMLSize": pml}, src_len=len(sig))


def workload2d(seed=0, N=256, Nt=500, dx=0.1e-3, pml=10, absorbing=True):
    """2-D heterogeneous run: blob sound speed, disc p0, one sensor line."""
    rng = np.random.default_rng(seed)
    c = np.full((N, N), 1500.0)
    ax = np.arange(N, dtype=np.float64)
    for _ in range(6):
        cx, cy = rng.uniform(pml, N - pml, 2)
        sg = rng.uniform(4.0, 16.0)
        c += rng.uniform(-100.0, 200.0) * np.exp(-((ax[:, None] - cx) ** 2 + (ax[None, :] - cy) ** 2) / (2 * sg * sg))
    medium = {"sound_speed": c, "density": 1000.0 + 0.6 * (c - 1500.0)}
    if absorbing:
        medium.update(alpha_coeff=0.75, alpha_power=1.5)
    yy, xx = np.meshgrid(ax, ax)
    p0 = ((xx - N / 2) ** 2 + (yy - N / 2) ** 2 <= (N / 16) ** 2).astype(np.float64)
    sensor_mask = np.zeros((N, N))
    sensor_mask[pml + 2, :] = 1
    return dict(shape=(N, N), dx=dx, Nt=Nt, dt=0.3 * dx / c.max(), medium=medium, source={"p0": p0},
                sensor={"mask": sensor_mask, "record": ["p", "p_max"]}, options={"PMLSize": pml}, src_len=0)


# Layered medium of the large 512^3 simulation: sound speed per layer (the
# recipe's 1480 / 1560 / 2800 / 1560 m/s), density tied to speed as in the
# blob medium, alpha_power 1.1.  The recipe gives no absorption coefficient;
# these per-layer values (dB/(MHz^y cm)) are this benchmark's choice.
LAYER_C = (1480.0, 1560.0, 2800.0, 1560.0)
LAYER_ALPHA = (0.5, 1.0, 4.0, 1.0)


def rough_surface(n0, n1, rng, rms=3.0, corr=8.0):
    """Random interface height (cells) over an n0 x n1 plane: white noise
    low-passed by a Gaussian of `corr` cells, scaled to `rms` cells RMS."""
    k0 = np.fft.fftfreq(n0)[:, None]
    k1 = np.fft.fftfreq(n1)[None, :]
    filt = np.exp(-2.0 * (np.pi * corr) ** 2 * (k0 ** 2 + k1 ** 2))
    h = np.real(np.fft.ifft2(np.fft.fft2(rng.standard_normal((n0, n1))) * filt))
    return h * (rms / h.std())


def focused_burst(t, delay, f0, cycles, amp):
    """amp sin(2 pi f0 tau) times a Hann window over `cycles` periods,
    tau = t - delay, zero outside the window (one row per delay)."""
    T = cycles / f0
    tau = t[None, :] - delay[:, None]
    inside = (tau >= 0) & (tau <= T)
    return np.where(inside, amp * np.sin(2 * np.pi * f0 * tau) * (0.5 - 0.5 * np.cos(2 * np.pi * tau / T)), 0.0)


def layered_workload(seed=0, N=512, Nt=2000, dx=0.1e-3, pml=20, f0=500e3, cycles=5, focus=300, src=128,
                     amp=1e6):
    """Large single 3-D simulation: four layers along x with rough interfaces
    (3-cell RMS), alpha_power 1.1, B/A drawn from 5..9 per layer, a src x src
    phased plane pressure source at x = pml (0-based) focused `focus` cells
    deep by per-element delays, a Hann-windowed `cycles`-cycle burst at f0,
    and full-volume p_max / p_rms (the mask is every cell)."""
    rng = np.random.default_rng(seed)
    shape = (N, N, N)
    x = np.arange(N, dtype=np.float64)[:, None, None]
    layer = np.zeros(shape, dtype=np.int8)
    for k in (1, 2, 3):
        depth = pml + (N - 2 * pml) * k / 4.0
        layer += (x >= (depth + rough_surface(N, N, rng))[None, :, :]).astype(np.int8)
    c = np.asarray(LAYER_C)[layer]
    bona = rng.integers(5, 10, size=4).astype(np.float64)
    medium = {"sound_speed": c, "density": 1000.0 + 0.6 * (c - 1500.0),
              "alpha_coeff": np.asarray(LAYER_ALPHA)[layer], "alpha_power": 1.1, "BonA": bona[layer]}
    del layer
    dt = 0.3 * dx / c.max()
    h = N // 2
    lo, hi = h - src // 2, h - src // 2 + src
    p_mask = np.zeros(shape, dtype=bool)
    p_mask[pml, lo:hi, lo:hi] = True
    # source points in find(p_mask) order (column-major: y fastest, then z)
    zz, yy = np.meshgrid(np.arange(lo, hi), np.arange(lo, hi), indexing="ij")
    dist = dx * np.sqrt(focus ** 2 + (yy.ravel() - h) ** 2 + (zz.ravel() - h) ** 2)
    delay = (dist.max() - dist) / LAYER_C[0]
    # the signal ends with the last element's burst (the source is active
    # only while it has samples)
    src_len = int(min(Nt, math.ceil((delay.max() + cycles / f0) / dt) + 1))
    sig = focused_burst(np.arange(src_len) * dt, delay, f0, cycles, amp)
    sensor = {"mask": np.ones(shape, dtype=bool), "record": ["p_max", "p_rms"]}
    return dict(shape=shape, dx=dx, Nt=Nt, dt=dt, medium=medium, source={"p_mask": p_mask, "p": sig},
                sensor=sensor, options={"PMLSize": pml}, src_len=src_len)


def make_grid(kw, w):
    if len(w["shape"]) == 2:
        g = kw.kWaveGrid(w["shape"][0], w["dx"], w["shape"][1], w["dx"])
        g.setTime(w["Nt"], w["dt"])
        return g
    g = kw.kWaveGrid(w["shape"][0], w["dx"], w["shape"][1], w["dx"], w["shape"][2], w["dx"])
    g.setTime(w["Nt"], w["dt"])
    return g


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons while running."""

    def __init__(self, device, path):
        self.path = path
        self.proc = None
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(device), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() in ("active", "1"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(w, steps, single=False):
    """The oracle (NumPy/SciPy, all host cores) on a bounded sample of the
    same workload: the first ``steps`` time steps, in FP64 (the reference's
    default) or FP32 (its DataCast 'single')."""
    sys.path.insert(0, ROOT)
    from oracle import kspace as oracle
    g = oracle.KWaveGrid(w["shape"][0], w["dx"], w["shape"][1], w["dx"], w["shape"][2], w["dx"])
    g.setTime(steps, w["dt"])
    oracle.kspace_first_order(g, w["medium"], w["source"], w["sensor"], Single=single, **w["options"])
    secs = oracle.LAST_LOOP_SECONDS
    cells = float(np.prod(w["shape"]))
    return {"value": cells * steps / secs / 1e9, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": "first %d of %d time steps of the %s workload, %s NumPy/SciPy oracle "
                      "(scipy.fft workers=%d); loop time only"
                      % (steps, w["Nt"], "x".join(str(n) for n in w["shape"]), "FP32" if single else "FP64",
                         os.cpu_count()),
            "seconds": secs}


def cfg1_workload(N=128, dx=0.1e-3, c=1500.0, pml=20):
    """The 2-D homogeneous lossless case: 128^2, dx 0.1 mm, disc p0 of radius
    5 at the centre (smoothed), PML 20 / alpha 2, CFL 0.3, t_end = 1.2 x the
    grid diagonal / c (Nt = 725), 64 points on a circle of radius 40 cells
    mapped to the grid by nearest neighbour, recording p."""
    import kwave_b200 as kw
    t_end = 1.2 * math.sqrt(2) * N * dx / c
    g = kw.kWaveGrid(N, dx, N, dx)
    g.makeTime(c, 0.3, t_end)
    return dict(shape=(N, N), dx=dx, Nt=g.Nt, dt=g.dt, t_end=t_end, medium={"sound_speed": c, "density": 1000.0},
                source={"p0": kw.makeDisc(N, N, N // 2 + 1, N // 2 + 1, 5)},
                sensor={"mask": kw.makeCartCircle(40 * dx, 64)},
                options={"PMLSize": pml, "PMLAlpha": 2.0, "CartInterp": "nearest"})


def cfg1_section(kw, device, runs=20, cpu=True):
    """The 2-D case as specified, device-resident on the GPU (runs complete
    simulations timed with CUDA events) and the FP64 oracle at its full Nt on
    the host cores; rel-L2 of the GPU p against the oracle's."""
    w = cfg1_workload()
    cells = float(np.prod(w["shape"]))
    g = kw.kWaveGrid(w["shape"][0], w["dx"], w["shape"][1], w["dx"])
    g.setTime(w["Nt"], w["dt"])
    with kw.Simulation(2, g, w["medium"], w["source"], w["sensor"], **dict(w["options"], DeviceNum=device)) as sim:
        p = sim.run()
        sim.run_timed(2)
        ms = sim.run_timed(runs)
    out = {"workload": "kspaceFirstOrder2D 128^2 homogeneous lossless, disc p0 r=5, PML 20, Nt=%d, "
                       "64-point circle r=40 (nearest), record p" % w["Nt"],
           "gpu": {"value": cells * w["Nt"] * runs / (ms / 1e3) / 1e9, "unit": UNIT,
                   "ms_per_simulation": ms / runs, "note": "launch-bound: 16 384 cells per step"}}
    if cpu:
        sys.path.insert(0, ROOT)
        from oracle import kspace as oracle
        og = oracle.KWaveGrid(w["shape"][0], w["dx"], w["shape"][1], w["dx"])
        og.setTime(w["Nt"], w["dt"])
        ref = oracle.kspace_first_order(og, w["medium"], w["source"], w["sensor"], **w["options"])
        secs = oracle.LAST_LOOP_SECONDS
        out["cpu_fp64"] = {"value": cells * w["Nt"] / secs / 1e9, "unit": UNIT, "cores": os.cpu_count(),
                           "kind": "port", "sample": "the full run (Nt=%d), loop time only" % w["Nt"]}
        out["rel_l2_gpu_vs_oracle"] = _rel_l2(p, ref)
    return out


def dist_setup(backend=None):
    """One process per GPU (torch.distributed.run sets RANK / WORLD_SIZE);
    NCCL on GPUs, gloo when no GPU is visible.  The process group only
    carries the barrier and the max-over-ranks timing: the replicas never
    exchange simulation data."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def dist_max(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(ws, cells, Nt, steps, ms_local):
    """Whole-job Gcell-steps/s of ws replicas that each ran ``steps``
    simulations of ``cells`` x ``Nt``: total work over the slowest rank's
    device time."""
    ms_max = dist_max(ms_local, ws)
    return ws * cells * Nt * steps / (ms_max / 1e3) / 1e9, ms_max


def dist_barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def run_reference(args, ws, rank):
    """The reference arm: the reference's CPU implementation of the loop.  MATLAB
    is not installed, so the FP64 restatement of the reference solver runs on
    the host cores (kind 'port'); each step is a bounded sample of the
    workload (its first --cpu-steps time steps)."""
    if rank != 0:
        return
    w = workload(seed=0)
    sys.path.insert(0, ROOT)
    for _ in range(args.warmup):
        cpu_baseline(w, 1)
    secs = 0.0
    for _ in range(args.steps):
        r = cpu_baseline(w, args.cpu_steps)
        secs += r["seconds"]
    cells = float(np.prod(w["shape"]))
    value = cells * args.cpu_steps * args.steps / secs / 1e9
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": {"workload": "kspaceFirstOrder3D 256^3 absorbing BonA plane source",
                                                      "step": "first %d time steps" % args.cpu_steps},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                             "sample": r["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _latency_stats(lat_ms):
    v = np.sort(np.asarray(lat_ms, dtype=np.float64))
    return {"p50_ms": float(np.percentile(v, 50)), "p99_ms": float(np.percentile(v, 99)), "mean_ms": float(v.mean())}


def _rel_l2(a, b):
    if isinstance(b, dict):
        return max(_rel_l2(a[k], b[k]) for k in b)
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (d if d > 0 else 1.0))


SERVE_EDGES = (64, 96, 128, 160, 192, 256, 320, 384)


def served_request(rng, dx=0.2e-3, nt_scale=1.0, pml=10):
    """One request of the served stream: a 3-D simulation whose edge along
    each axis is drawn log-uniformly from SERVE_EDGES (so grids are
    anisotropic), a blob medium as in the headline workload (absorbing,
    BonA 6), a point pressure source at a random interior position driven by
    a Hann-windowed 3-cycle tone burst of 0.5-2 MHz at 1 MPa, Nt uniform in
    500-2000 (times nt_scale), FP32; p recorded at 32 random points and p_max
    on the central xy-plane."""
    logs = np.log(SERVE_EDGES)
    shape = tuple(int(SERVE_EDGES[int(np.argmin(np.abs(logs - rng.uniform(logs[0], logs[-1]))))]) for _ in range(3))
    Nt = max(1, int(round(rng.integers(500, 2001) * nt_scale)))
    c = blob_speed(shape, rng, pml=pml)
    medium = {"sound_speed": c, "density": 1000.0 + 0.6 * (c - 1500.0), "alpha_coeff": 0.75, "alpha_power": 1.5,
              "BonA": 6.0}
    dt = 0.3 * dx / c.max()
    pm = np.zeros(shape, dtype=bool)
    pm[tuple(int(rng.integers(pml + 2, n - pml - 2)) for n in shape)] = True
    f0 = rng.uniform(0.5e6, 2e6)
    sig = hann_burst(dt, f0=f0, cycles=3, amp=1e6)
    sm = np.zeros(shape, dtype=bool)
    sm[:, :, shape[2] // 2] = True
    pts = np.zeros(shape, dtype=bool)
    for _ in range(32):
        pts[tuple(int(rng.integers(pml, n - pml)) for n in shape)] = True
    return dict(shape=shape, dx=dx, Nt=Nt, dt=dt, medium=medium, source={"p_mask": pm, "p": sig[None, :]},
                sensor={"mask": sm | pts, "record": ["p", "p_max"]}, options={"PMLSize": pml},
                src_len=len(sig), f0=f0)


def served_section(kw, device, n_req=40, seed=7, load=0.8, nt_scale=0.2):
    """Continuous batching against the plain path on the same request stream.

    The stream is the served-stream recipe (3-D requests, per-axis edges
    log-uniform over 64..384, blob media, point sources of 0.5-2 MHz,
    Nt uniform in 500-2000) as a time-scaled subset: n_req requests with Nt
    scaled by nt_scale.  Two passes per path over the same requests:
    'saturated' submits everything at t = 0 (aggregate Gcell-steps/s =
    cell-steps / makespan); 'poisson' submits at Poisson arrival times whose
    rate is `load` x the plain path's capacity (p50 / p99 of submit->result
    latency).  The plain path runs the requests one after another through
    the drop-in call on a prepared problem (plan, loop, outputs to host);
    the served path hands them to kwave_b200.Server.  Host setup (input
    checking) is done beforehand for both.  Every served result is compared
    with the plain result of the same request.
    """
    rng = np.random.default_rng(seed)
    preps, cells, reqs = {}, {}, []
    for i in range(n_req):
        w = served_request(rng, nt_scale=nt_scale)
        preps[i] = kw.Server.prepare(3, make_grid(kw, w), w["medium"], w["source"], w["sensor"],
                                     **dict(w["options"], DeviceNum=device))
        cells[i] = float(np.prod(w["shape"])) * w["Nt"]
        reqs.append((w["shape"], w["Nt"]))
    picks = np.arange(n_req)
    work = float(sum(cells[k] for k in picks))

    def plain(arrivals):
        lat, outs = [], []
        t0 = time.perf_counter()
        for k, a in zip(picks, arrivals):
            now = time.perf_counter() - t0
            if a > now:
                time.sleep(a - now)
            with kw.Simulation.from_prepared(preps[k]) as sim:
                outs.append(sim.run())
            lat.append((time.perf_counter() - t0 - a) * 1e3)
        return time.perf_counter() - t0, lat, outs

    def served(arrivals):
        with kw.Server(device=device) as srv:
            t0 = time.perf_counter()
            tickets = []
            for k, a in zip(picks, arrivals):
                now = time.perf_counter() - t0
                if a > now:
                    time.sleep(a - now)
                tickets.append(srv.submit_prepared(preps[k]))
            res = [srv.result(t, with_latency=True) for t in tickets]
            span = time.perf_counter() - t0
            st = srv.stats()
        worker = {k: st[k] for k in ("setup_seconds", "issue_seconds", "retire_seconds", "wait_seconds")}
        return span, [r[1] for r in res], [r[0] for r in res], worker

    # warm both paths (module load, first plans, graph capture paths)
    for k in preps:
        with kw.Simulation.from_prepared(preps[k]) as sim:
            sim.run()
    zeros = np.zeros(n_req)
    p_span, _, p_outs = plain(zeros)
    s_span, _, s_outs, s_worker = served(zeros)
    err = max(_rel_l2(a, b) for a, b in zip(s_outs, p_outs))
    rate = load * n_req / p_span
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n_req))
    arrivals -= arrivals[0]
    pp_span, pp_lat, _ = plain(arrivals)
    sp_span, sp_lat, sp_outs, _ = served(arrivals)
    err = max(err, max(_rel_l2(a, b) for a, b in zip(sp_outs, p_outs)))
    edges = [s for shp, _ in reqs for s in shp]
    mix = {"requests": n_req, "nt_scale": nt_scale, "Nt_range": [min(n for _, n in reqs), max(n for _, n in reqs)],
           "cells_range": [min(int(np.prod(s)) for s, _ in reqs), max(int(np.prod(s)) for s, _ in reqs)],
           "edge_counts": {str(e): edges.count(e) for e in SERVE_EDGES},
           "anisotropic": sum(len(set(s)) > 1 for s, _ in reqs)}
    return {
        "stream": "3-D requests, per-axis edges log-uniform over %s, blob media, point source 0.5-2 MHz, "
                  "Nt uniform 500-2000 x %g (time-scaled subset of the 2000-request stream)"
                  % (list(SERVE_EDGES), nt_scale),
        "requests": n_req, "mix": mix, "cell_steps": work,
        "saturated": {"served_gcell_steps_per_s": work / s_span / 1e9, "plain_gcell_steps_per_s": work / p_span / 1e9,
                      "served_makespan_s": s_span, "plain_makespan_s": p_span, "served_worker_seconds": s_worker},
        "poisson": {"rate_per_s": rate, "load_vs_plain_capacity": load,
                    "served": _latency_stats(sp_lat), "plain": _latency_stats(pp_lat),
                    "served_gcell_steps_per_s": work / sp_span / 1e9, "plain_gcell_steps_per_s": work / pp_span / 1e9},
        "max_rel_l2_served_vs_plain": err, "tolerance": 1e-4,
        "latency": "submit -> outputs on the host, wall clock",
    }


def ricker(dt, Nt, f0=1e6):
    """Ricker wavelet (1 - 2 (pi f0 tau)^2) exp(-(pi f0 tau)^2), tau = t - 1.5 / f0."""
    tau = np.arange(Nt) * dt - 1.5 / f0
    a = (np.pi * f0 * tau) ** 2
    return (1.0 - 2.0 * a) * np.exp(-a)


def adjoint_workload(N=512, Nt=3000, n_elem=256, radius=230, n_shots=16, dx=0.1e-3, seed=4, c_ref=1800.0):
    """Sound-speed inversion set-up: a ring array of n_elem elements (radius in
    cells) around a blob medium; n_shots elements fire in turn a 1 MHz Ricker
    wavelet (additive point source) and every element records p."""
    rng = np.random.default_rng(seed)
    ax = np.arange(N, dtype=np.float64) - N / 2
    c_true = np.full((N, N), 1500.0)
    for _ in range(6):
        r0 = rng.uniform(0, 0.6 * radius)
        ang = rng.uniform(0, 2 * np.pi)
        cx, cy = r0 * np.cos(ang), r0 * np.sin(ang)
        sg = rng.uniform(10.0, 30.0)
        c_true += rng.uniform(-80.0, 150.0) * np.exp(-((ax[:, None] - cx) ** 2 + (ax[None, :] - cy) ** 2) / (2 * sg * sg))
    dt = 0.3 * dx / c_ref
    return dict(N=N, Nt=Nt, dx=dx, dt=dt, c_true=c_true, c_start=np.full((N, N), 1500.0), rho=np.full((N, N), 1000.0),
                n_elem=n_elem, radius=radius, n_shots=n_shots, c_ref=c_ref, src=1e5 * ricker(dt, Nt))


def _adjoint_problem(kw, w, c, shot, mask_cells):
    g = kw.kWaveGrid(w["N"], w["dx"], w["N"], w["dx"])
    g.setTime(w["Nt"], w["dt"])
    shape = (w["N"], w["N"])
    pm = np.zeros(shape)
    pm[np.unravel_index(mask_cells[shot * (len(mask_cells) // w["n_shots"])], shape, order="F")] = 1
    ring = np.zeros(shape)
    ring[np.unravel_index(mask_cells, shape, order="F")] = 1
    med = {"sound_speed": c, "density": w["rho"], "sound_speed_ref": w["c_ref"]}
    return kw.Server.prepare(2, g, med, {"p_mask": pm, "p": w["src"][None, :]}, {"mask": ring}, PMLSize=20, Smooth=False)


def tr_gradient_cosine(kw, c0, rho, kgrid_args, Nt, dt, pm, sig, ring, c_ref, pml, residual, g_adj, inside):
    """Cosine similarity, over `inside`, between an adjoint sound-speed
    gradient and the time-reversal image: the residual re-injected at the
    sensors by the time-reversal mode (sensor.time_reversal_boundary_data,
    kspaceFirstOrder3D.m:715-788) gives a back-propagated field q; the image
    is sum_t (2 / c0) dp/dt q at each cell, with p the forward field."""
    def grid():
        g = kw.kWaveGrid(*kgrid_args)
        g.setTime(Nt, dt)
        return g
    med = {"sound_speed": c0, "density": rho, "sound_speed_ref": c_ref}
    hist = None
    with kw.Simulation(2, grid(), med, {"p_mask": pm, "p": sig[None, :]}, {"mask": ring, "record": ["p_final"]},
                       PMLSize=pml, Smooth=False) as sim:
        for t in range(Nt):
            sim.step(1)
            f = sim.copy_outputs()["p_final"]
            if hist is None:
                hist = np.zeros((Nt,) + f.shape, dtype=np.float32)
            hist[t] = f
    img = np.zeros(hist.shape[1:])
    with kw.Simulation(2, grid(), med, {}, {"mask": ring, "time_reversal_boundary_data": residual},
                       PMLSize=pml, Smooth=False) as sim:
        for s in range(1, Nt):
            sim.step(1)
            t = Nt - s - 1                 # time-reversal step s is physical time Nt - s (0-based t)
            if 1 <= t <= Nt - 2:
                pt = (hist[t + 1].astype(np.float64) - hist[t - 1]) / (2 * dt)
                img += pt * sim.copy_outputs()
    img *= 2.0 / c0
    a, b = img[inside], g_adj[inside]
    return float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))


def tr_check(kw, N=256, n_elem=128, radius=110, Nt=1500, dx=0.1e-3, seed=5):
    """The time-reversal comparison on a reduced ring case (shot 0): cosine
    between the adjoint sound-speed gradient and the time-reversal image."""
    w = adjoint_workload(N=N, Nt=Nt, n_elem=n_elem, radius=radius, n_shots=1, dx=dx, seed=seed)
    g = kw.kWaveGrid(N, dx, N, dx)
    ring_mask, _, _ = kw.cart2grid(g, kw.makeCartCircle(radius * dx, n_elem))
    cells = np.flatnonzero(ring_mask.ravel(order="F"))
    with kw.Simulation.from_prepared(_adjoint_problem(kw, w, w["c_true"], 0, cells)) as sim:
        d = sim.run().astype(np.float64)
    with kw.Simulation.from_prepared(_adjoint_problem(kw, w, w["c_start"], 0, cells)) as sim:
        r = sim.run().astype(np.float64) - d
        g_adj, _ = sim.adjoint_gradient(r, density=False)
    shape = (N, N)
    pm = np.zeros(shape)
    pm[np.unravel_index(cells[0], shape, order="F")] = 1
    ring = np.zeros(shape)
    ring[np.unravel_index(cells, shape, order="F")] = 1
    ax = np.arange(N) - N / 2
    inside = (ax[:, None] ** 2 + ax[None, :] ** 2) < (0.8 * radius) ** 2
    return tr_gradient_cosine(kw, w["c_start"], w["rho"], (N, dx, N, dx), Nt, w["dt"], pm, w["src"], ring, w["c_ref"], 20,
                              r, g_adj, inside)


LARGE_BYTES_PER_CELL_STEP = 164.0   # 4 B x (6 + 7 state + 8 medium + 2 x 8 spectral + 4 full-volume accumulators)


def large_section(kw, device, N=512, Nt=2000, seed=11):
    """The large layered simulation (512^3, full-volume p_max / p_rms) at its
    full Nt with every input resident.  Warm-up: the first source_steps + 8
    steps (every step structure is captured); then one whole simulation,
    stepped as its source-active part and its quiet part (each call returns
    when its steps are done), so the two kinds of step are timed apart;
    per-class device times from the first 200 steps of a further run."""
    t0 = time.perf_counter()
    w = layered_workload(seed=seed, N=N, Nt=Nt)
    cells = float(np.prod(w["shape"]))
    src_steps = min(w["src_len"], Nt)
    with kw.Simulation(3, make_grid(kw, w), w["medium"], w["source"], w["sensor"], **dict(w["options"], DeviceNum=device)) as sim:
        setup_s = time.perf_counter() - t0
        dev_gb = sim.device_bytes() / 1e9
        sim.step(min(Nt, src_steps + 8))
        sim.reset()
        ta = time.perf_counter()
        sim.step(src_steps)
        tb = time.perf_counter()
        if Nt > src_steps:
            sim.step(Nt - src_steps)
        tc = time.perf_counter()
        ms = (tc - ta) * 1e3
        classes = {}
        n_cls = min(Nt, 200)
        sim.reset()
        sim.set_timing(["zstage_u", "zstage_r", "zstage_p", "ypass", "xpass", "sensor", "source"])
        sim.step(n_cls)
        for c in ("zstage_u", "zstage_r", "zstage_p", "ypass", "xpass", "sensor", "source"):
            classes[c] = round(sim.timing(c)[0] / n_cls * 1e3, 1)
        sim.set_timing([])
    peak, peak_kind = measured_peak()
    alg = cells * (LARGE_BYTES_PER_CELL_STEP * Nt + BYTES_PER_CELL_SRC_STEP * src_steps)
    achieved = alg / (ms / 1e3) / 1e9
    phases = {"source_active": {"steps": src_steps, "ms_per_step": (tb - ta) * 1e3 / src_steps,
                                "gcell_steps_per_s": cells * src_steps / (tb - ta) / 1e9}}
    if Nt > src_steps:
        phases["quiet"] = {"steps": Nt - src_steps, "ms_per_step": (tc - tb) * 1e3 / (Nt - src_steps),
                           "gcell_steps_per_s": cells * (Nt - src_steps) / (tc - tb) / 1e9}
    return {"workload": "kspaceFirstOrder3D %d^3 layered 1480/1560/2800/1560 m/s (rough interfaces, 3-cell RMS), "
                        "alpha_power 1.1, per-layer alpha_coeff %s dB/(MHz^y cm) and BonA 5..9, 128x128 phased plane "
                        "p source focused 300 cells deep, 500 kHz 5-cycle burst, PML 20, full-volume p_max + p_rms"
                        % (N, "/".join("%g" % a for a in LAYER_ALPHA)),
            "Nt": Nt, "source_steps": src_steps, "value": cells * Nt / (ms / 1e3) / 1e9, "unit": UNIT,
            "ms_per_time_step": ms / Nt, "device_gb": round(dev_gb, 2), "host_setup_s": round(setup_s, 1),
            "phases": phases, "timing": "wall clock around synchronous step calls (graph-replayed steps)",
            "class_us_per_step_over": "first %d steps" % min(Nt, 200),
            "roofline": {"achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind, "alg_bytes_per_cell_step": LARGE_BYTES_PER_CELL_STEP},
            "us_per_time_step": classes}


def adjoint_section(kw, device, Nt=3000, n_shots=16, fd_cells=32, seed=4, tr=True, workers=8):
    """Gradient of J = 1/2 sum over shots of |p(ring) - d|^2 at the homogeneous
    starting model (16 shots, Nt steps, sqrt(Nt) checkpointing), timed per
    shot, and central finite differences of J for shot 0 at fd_cells random
    cells inside the ring (FP32 forward runs, h = 1 % of c)."""
    w = adjoint_workload(Nt=Nt, n_shots=n_shots, seed=seed)
    g = kw.kWaveGrid(w["N"], w["dx"], w["N"], w["dx"])
    ring_mask, _, _ = kw.cart2grid(g, kw.makeCartCircle(w["radius"] * w["dx"], w["n_elem"]))
    cells = np.flatnonzero(ring_mask.ravel(order="F"))
    data = []
    for s in range(n_shots):
        with kw.Simulation.from_prepared(_adjoint_problem(kw, w, w["c_true"], s, cells)) as sim:
            data.append(sim.run())
    def one_shot(s):
        with kw.Simulation.from_prepared(_adjoint_problem(kw, w, w["c_start"], s, cells)) as sim:
            sim.keep_checkpoints()   # the misfit's forward run is the gradient's checkpointing run
            y = sim.run()
            r = y.astype(np.float64) - data[s]
            gc, _ = sim.adjoint_gradient(r)
        return gc, 0.5 * float(np.sum(r * r))

    grad = np.zeros((w["N"], w["N"]))
    J = 0.0
    shot_s = []
    per_shot = []
    for s in range(n_shots):
        t0 = time.perf_counter()
        gc, js = one_shot(s)
        shot_s.append(time.perf_counter() - t0)
        per_shot.append(gc)
        grad += gc
        J += js
    g0 = per_shot[0]
    # the shots are independent: the same 16 gradients with several shots in
    # flight at once (one plan and stream per host thread), summed in shot order
    from concurrent.futures import ThreadPoolExecutor
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=workers) as ex:
        conc = list(ex.map(one_shot, range(n_shots)))
    conc_s = time.perf_counter() - t0
    grad_c = np.zeros_like(grad)
    for gc, _ in conc:
        grad_c += gc
    conc_diff = float(np.max(np.abs(grad_c - grad)) / max(np.max(np.abs(grad)), 1e-300))
    # finite differences for shot 0
    rng = np.random.default_rng(seed + 1)
    fd, ad = [], []
    h = 15.0
    inside = np.argwhere((np.arange(w["N"])[:, None] - w["N"] / 2) ** 2 + (np.arange(w["N"])[None, :] - w["N"] / 2) ** 2
                         < (0.8 * w["radius"]) ** 2)
    for k in rng.choice(len(inside), size=fd_cells, replace=False):
        x, yy = inside[k]
        vals = []
        for sgn in (1, -1):
            c = w["c_start"].copy()
            c[x, yy] += sgn * h
            with kw.Simulation.from_prepared(_adjoint_problem(kw, w, c, 0, cells)) as sim:
                rr = sim.run().astype(np.float64) - data[0]
            vals.append(0.5 * float(np.sum(rr * rr)))
        fd.append((vals[0] - vals[1]) / (2 * h))
        ad.append(float(g0[x, yy]))
    fd, ad = np.array(fd), np.array(ad)
    big = np.abs(fd) > 0.05 * np.abs(fd).max()
    tr_cos = None
    if tr:
        # the inversion case's own ring (512^2, 256 elements, radius 230,
        # Nt 3000) and, for contrast, a dense and a sparse ring on 256^2
        tr_cos = [{"grid": 512, "elements": 256, "radius": 230, "Nt": Nt,
                   "cosine_with_adjoint_gradient": tr_check(kw, N=512, n_elem=256, radius=230, Nt=Nt, seed=seed)}]
        tr_cos += [{"grid": 256, "elements": ne, "radius": 110, "Nt": 1500,
                    "cosine_with_adjoint_gradient": tr_check(kw, n_elem=ne)} for ne in (512, 128)]
    return {
        "workload": "2D %dx%d ring array of %d elements (radius %d cells), %d shots, 1 MHz Ricker, Nt=%d, "
                    "homogeneous 1500 m/s start, blob true medium" % (w["N"], w["N"], w["n_elem"], w["radius"],
                                                                       n_shots, Nt),
        "checkpoint_interval": int(round(np.sqrt(Nt))), "misfit": J,
        "seconds_per_shot": float(np.median(shot_s)), "seconds_all_shots": float(np.sum(shot_s)),
        "seconds_per_shot_note": "forward run + gradient (forward with checkpoints, per-segment re-run, adjoint)",
        "concurrent": {"workers": workers, "seconds_all_shots": conc_s, "seconds_per_shot": conc_s / n_shots,
                       "max_rel_diff_vs_one_at_a_time": conc_diff},
        "fd_check": {"cells": fd_cells, "h_m_per_s": h,
                     "cosine": float(np.dot(fd, ad) / (np.linalg.norm(fd) * np.linalg.norm(ad))),
                     "max_rel_err_where_fd_above_5pct": float(np.max(np.abs(ad[big] - fd[big]) / np.abs(fd[big]))),
                     "median_rel_err_where_fd_above_5pct": float(np.median(np.abs(ad[big] - fd[big]) / np.abs(fd[big])))},
        "time_reversal_check": None if tr_cos is None else {
            "rings": tr_cos,
            "case": "shot 0 of each ring: image sum_t (2/c) dp/dt q of the forward field p and the field q of the "
                    "time-reversal run fed the residual, inside 0.8 x radius; the time-reversal mode pins p at the "
                    "sensor cells, so sparse rings scatter and the image departs from the exact gradient"},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=5)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--Nt", type=int, default=1000)
    ap.add_argument("--N", type=int, default=256)
    ap.add_argument("--serve-requests", type=int, default=40, help="0 skips the served-stream section")
    ap.add_argument("--serve-nt-scale", type=float, default=0.2, help="Nt scale of the served-stream subset")
    ap.add_argument("--cfg1-runs", type=int, default=20, help="0 skips the 2-D 128^2 section")
    ap.add_argument("--adjoint-shots", type=int, default=16, help="0 skips the adjoint section")
    ap.add_argument("--adjoint-fd", type=int, default=32, help="finite-difference cells of the adjoint check")
    ap.add_argument("--adjoint-workers", type=int, default=8, help="adjoint shots in flight at once")
    ap.add_argument("--large-Nt", type=int, default=2000, help="time steps of the 512^3 layered run (0 skips it)")
    args = ap.parse_args()
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, ws, rank)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import kwave_b200 as kw
    w = workload(seed=rank, N=args.N, Nt=args.Nt)
    opts = dict(w["options"], DeviceNum=local)
    sim = kw.Simulation(3, make_grid(kw, w), w["medium"], w["source"], w["sensor"], **opts)
    cells = float(np.prod(w["shape"]))
    Nt = w["Nt"]
    dev_gb = sim.device_bytes() / 1e9

    # warm-up (full simulations)
    sim.run_timed(max(args.warmup, 0)) if args.warmup > 0 else None

    # timed region: K complete simulations, device events on the library stream
    # raw clock samples go to KW_CLOCKS_DIR (default: the system temp dir);
    # the bench line carries their summary
    clk_dir = os.environ.get("KW_CLOCKS_DIR") or tempfile.gettempdir()
    os.makedirs(clk_dir, exist_ok=True)
    clk = Clocks(local, os.path.join(clk_dir, "clocks_rank%d.csv" % rank))
    l0 = sim.launch_count()
    dist_barrier(ws)
    ms = sim.run_timed(args.steps)
    dist_barrier(ws)
    launches = sim.launch_count() - l0
    clocks = clk.stop()
    value, ms_max = job_throughput(ws, cells, Nt, args.steps, ms)

    # kernel classes (separate run with per-launch events; not part of the timed region)
    sim.set_timing(["zstage_u", "zstage_r", "zstage_p", "ypass", "xpass", "sensor", "source"])
    sim.run_device()
    classes = {}
    tot = 0.0
    for c in ("zstage_u", "zstage_r", "zstage_p", "ypass", "xpass", "sensor", "source"):
        t, n = sim.timing(c)
        classes[c] = {"ms_per_sim": t, "launches_per_sim": n}
        tot += t
    for c in classes:
        classes[c]["share"] = classes[c]["ms_per_sim"] / tot if tot else 0.0
    sim.set_timing([])

    # roofline for the time step (the unit the bytes-per-cell-step model describes)
    peak, peak_kind = measured_peak()
    src_steps = min(w["src_len"], Nt)
    alg_bytes_per_sim = cells * (BYTES_PER_CELL_STEP * Nt + BYTES_PER_CELL_SRC_STEP * src_steps)
    achieved = alg_bytes_per_sim / (ms / args.steps / 1e3) / 1e9
    # DRAM bytes of one time step, per-kernel ncu captures of the 256^3
    # workload (profiles/traffic_256cube_per_kernel.md); ncu runs each launch
    # with cold caches (the file also gives the figure without the flush)
    traffic, traffic_src = None, None
    tf = os.path.join(ROOT, "profiles", "step_traffic_256.json")
    if os.path.exists(tf) and args.N == 256:
        try:
            tj = json.load(open(tf))
            traffic = tj.get("dram_bytes_per_step")
            traffic_src = {"file": "profiles/step_traffic_256.json", "measured_at_commit": tj.get("measured_at_commit"),
                           "method": tj.get("method"), "caveat": tj.get("caveat")}
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "traffic_source": traffic_src, "peak_source": peak_kind,
                "kernel": "one time step of the loop (all its launches)",
                "alg_bytes_per_cell_step": BYTES_PER_CELL_STEP}
    sim.close()

    # end to end through the public API with host arrays
    e2e = None
    if args.e2e_steps > 0:
        h2d = d2h = 0
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            with kw.Simulation(3, make_grid(kw, w), w["medium"], w["source"], w["sensor"], **opts) as s2:
                out = s2.run()
                h2d = s2.h2d_bytes
                d2h = int(sum(v.nbytes for v in out.values()))
        secs = time.perf_counter() - t0
        secs = dist_max(secs, ws)
        e2e = {"value": ws * cells * Nt * args.e2e_steps / secs / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": args.e2e_steps,
               "call": "kwave_b200.Simulation(...).run() == kspaceFirstOrder3D(kgrid, medium, source, sensor)"}

    served = None
    if args.serve_requests > 0:
        served = served_section(kw, local, n_req=args.serve_requests, seed=7 + rank, nt_scale=args.serve_nt_scale)

    cfg1 = None
    if args.cfg1_runs > 0:
        cfg1 = cfg1_section(kw, local, runs=args.cfg1_runs, cpu=(rank == 0 and not args.no_cpu))

    adjoint = None
    if args.adjoint_shots > 0:
        adjoint = adjoint_section(kw, local, n_shots=args.adjoint_shots, fd_cells=args.adjoint_fd, seed=4 + rank,
                                  workers=args.adjoint_workers)

    large = None
    if args.large_Nt > 0:
        large = large_section(kw, local, Nt=args.large_Nt, seed=11 + rank)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        try:
            cpu = cpu_baseline(w, args.cpu_steps)
            cpu.pop("seconds", None)
            c32 = cpu_baseline(w, args.cpu_steps, single=True)
            c32.pop("seconds", None)
            cpu["fp32"] = c32
        except Exception as e:  # the baseline is reported, not required
            cpu = {"error": str(e)}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded blob medium; no dataset)",
                "config": {"workload": "kspaceFirstOrder3D %d^3 heterogeneous absorbing (y=1.5) BonA=6, "
                                       "64x64 additive plane p source, 1 MHz 3-cycle burst, PML 10, Nt=%d"
                                       % (args.N, Nt),
                           "grid": list(w["shape"]), "Nt": Nt, "step": "one complete simulation (Nt time steps)",
                           "l2": "no flush: inputs larger than L2 (device working set %.2f GB vs 126 MB L2)" % dev_gb,
                           "parallelism": "replicas x%d" % ws},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
                "clocks": clocks, "kernel_classes": classes, "served": served, "adjoint": adjoint,
                "large_512": large, "cfg1_2d": cfg1}
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
