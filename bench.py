"""Benchmark of the multislice hot path: probe.slice steps/s on the STEM HAADF+BF scan workload.

Workload (the headline STEM configuration): cubic SrTiO3 (a = 3.905 A; Sr at 0, Ti at the body centre, O at the face
centres) tiled 8 x 8 x 20 (31.24 x 31.24 x 78.1 A, 6,400 atoms), 512 x 512 grid, 20 slices of 3.905 A, Lobato
infinite-projection potential, 200 keV probe of 20 mrad semiangle with C10 = C30 = 0, a 64 x 64 GridScan over one
central unit cell (start (4a, 4a), end (5a, 5a), endpoint false), annular detectors BF 0-20 mrad and HAADF 50-200 mrad.
One bench step = the whole scan: 4,096 positions x 20 slices = 81,920 probe.slice steps. Synthetic structure, no dataset.

Timed region (`value`): `simk_scan_device` with the potential's transmissions already on the device, positions and
detector outputs on the device; K scans between CUDA events on the library's stream (torch's current stream),
synchronised and barriered on both sides, max over ranks. The waves of a batch (up to 1 GiB) exceed L2 (126 MB), so
no flush is needed between steps. `e2e`: the public `STEM.scan` call from host arrays (structure -> potential built on
the device -> scan -> detector images back to the host), wall-clocked per call, the median of --e2e-steps calls (5)
after one warm-up call.

`forms`: after the headline, one timed scan of each form (plain float32, fused float32, bf16x3 split-BF16 tensor-core
stages) on the same stream, and, with the CPU leg, each form's relative L2 error per detector image against the float64
oracle at the CPU leg's sample positions (the bound for every form is 1e-4).

`--impl reference` and the `cpu_baseline` leg: the reference's CPU path restated in C++17 float64
(oracle/cpu/simk_cpu.cpp: its mixed-radix / Bluestein FFT2D, runCPU, Probe.build and the annular detectors, checked
against the float64 NumPy oracle; the Swift original cannot build on Linux), timed on min(8, cores) host threads over
positions on a bounded sample of positions of the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

A0 = 3.905
NX = NY = 512
SLICE = 3.905
ENERGY = 200e3
SEMIANGLE = 20.0
SCAN_N = 64
DETECTORS = [("BF", 0.0, 20.0), ("HAADF", 50.0, 200.0)]
WORKLOAD = "STEM HAADF+BF scan, SrTiO3 8x8x20 (6400 atoms, 78.1 A), 512x512, 20 slices of 3.905 A, 200 keV, " \
           "20 mrad, 64x64 scan over one unit cell"


def srtio3(nx, ny, nz):
    frac = np.array([(0, 0, 0), (0.5, 0.5, 0.5), (0.5, 0.5, 0), (0.5, 0, 0.5), (0, 0.5, 0.5)], dtype=np.float64)
    nums = np.array([38, 22, 8, 8, 8])
    shifts = np.array([(i, j, k) for i in range(nx) for j in range(ny) for k in range(nz)], dtype=np.float64)
    pos = ((shifts[:, None, :] + frac[None, :, :]) * A0).reshape(-1, 3)
    return (nx * A0, ny * A0, nz * A0), np.tile(nums, len(shifts)), pos


def silicon(nx, ny, nz, a0=5.431):
    """Diamond-cubic Si: the 8 atoms of the conventional cell, x outermost (AtomicStructure.repeated's order)."""
    frac = np.array([(0, 0, 0), (0, 0.5, 0.5), (0.5, 0, 0.5), (0.5, 0.5, 0), (0.25, 0.25, 0.25), (0.25, 0.75, 0.75),
                     (0.75, 0.25, 0.75), (0.75, 0.75, 0.25)], dtype=np.float64)
    shifts = np.array([(i, j, k) for i in range(nx) for j in range(ny) for k in range(nz)], dtype=np.float64)
    pos = ((shifts[:, None, :] + frac[None, :, :]) * a0).reshape(-1, 3)
    return (nx * a0, ny * a0, nz * a0), np.full(len(pos), 14), pos


def amorphous(box, n_atoms, dmin, species, seed):
    """Random positions in `box` with a minimum separation `dmin` (periodic in x and y), by sequential addition on a
    cell grid of side >= dmin; Z drawn from `species` {Z: probability}. Deterministic for a seed."""
    rng = np.random.default_rng(seed)
    box = np.asarray(box, dtype=np.float64)
    nc = np.maximum(1, np.floor(box / dmin).astype(int))
    side = box / nc
    cells = -np.ones(tuple(nc) + (8,), dtype=np.int64)
    fill = np.zeros(tuple(nc), dtype=np.int64)
    pos = np.empty((n_atoms, 3))
    n = 0
    d2 = dmin * dmin
    while n < n_atoms:
        cand = rng.uniform(0, 1, (4096, 3)) * box
        for p in cand:
            c = np.minimum((p / side).astype(int), nc - 1)
            ok = True
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        cz = c[2] + dz
                        if cz < 0 or cz >= nc[2]:
                            continue
                        cx, cy = (c[0] + dx) % nc[0], (c[1] + dy) % nc[1]
                        for k in range(fill[cx, cy, cz]):
                            q = pos[cells[cx, cy, cz, k]]
                            d = p - q
                            d[:2] -= np.round(d[:2] / box[:2]) * box[:2]
                            if d @ d < d2:
                                ok = False
                                break
                        if not ok:
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok and fill[c[0], c[1], c[2]] < 8:
                pos[n] = p
                cells[c[0], c[1], c[2], fill[c[0], c[1], c[2]]] = n
                fill[c[0], c[1], c[2]] += 1
                n += 1
                if n == n_atoms:
                    break
    zs = np.array(sorted(species))
    nums = rng.choice(zs, n_atoms, p=[species[z] for z in zs])
    return tuple(box), nums, pos


def scan_positions():
    xs = np.arange(SCAN_N) * (A0 / SCAN_N) + 4 * A0
    return np.stack(np.meshgrid(xs, xs, indexing="ij"), axis=-1).reshape(-1, 2)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def traffic_from_profiles(kernel: str):
    """(dram bytes per launch, where they come from) of `kernel` on this workload from the committed ncu capture, or
    (None, None). The figure is not measured in this run: it is the one-pass ncu capture named in the file, and it
    goes stale when the kernel changes after that capture."""
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(p):
        d = json.load(open(p))
        v = d.get(kernel)
        if isinstance(v, dict):
            return v.get("dram_bytes_per_launch"), f"profiles/roofline_traffic.json ({d.get('_captured', 'undated')}, " \
                                                   f"{v.get('kernel')}), not measured in this run"
    return None, None


# ---------------------------------------------------------------------------------------------------------------------
# CPU: the reference's path restated (oracle), on host threads over positions
# ---------------------------------------------------------------------------------------------------------------------

def slowest_rank(value: float, dist=None, device: str = "cpu") -> float:
    """The largest of every rank's `value` (a time): the whole job's time when each rank runs the same work. Every rank
    calls it at the same point; without a process group it returns `value`."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, world: int, slowest_seconds: float) -> float:
    """Units all ranks processed per second of the slowest rank (replicas: every rank does the same work)."""
    return world * units_per_rank / slowest_seconds


def sample_indices(n_positions: int):
    """The positions of the scan the CPU legs run: every (4096 / n)-th position."""
    return np.arange(SCAN_N * SCAN_N)[:: max(1, (SCAN_N * SCAN_N) // n_positions)][:n_positions]


class CpuReference:
    """The C++ float64 restatement of STEM.cpuScan (oracle/cpu/simk_cpu.cpp: FFT2D's mixed-radix / Bluestein
    transforms, runCPU, Probe.build, the annular detectors) on a sample of the workload's positions, `threads` workers
    over positions as runCPUParallel. The potential, transmissions, propagators, probe spectrum and masks are built
    once, by the same C++ restatement, when the object is made, as runBatch shares them."""

    def __init__(self, n_positions: int, threads: int):
        from oracle import simk_cpu as K
        from oracle import simk_oracle as O
        box, nums, pos = srtio3(8, 8, 20)
        s = O.Structure(box, nums, pos)
        self.n_slices = len(O.slice_thicknesses(box[2], SLICE))
        self.inputs = K.ScanInputs.from_structure(O.ProbeSpec(ENERGY, SEMIANGLE), s, NX, NY,
                                                  O.slice_thicknesses(box[2], SLICE),
                                                  [(a, b) for _, a, b in DETECTORS])
        self.positions = scan_positions()[sample_indices(n_positions)]
        self.threads = threads

    def warm_up(self):
        """One scan of `threads` positions (each worker's FFT plans and buffers)."""
        self.inputs.scan(self.positions[:self.threads], threads=self.threads)

    def step(self):
        """One timed scan of the sample: (steps/s, seconds, positions, values [position][detector])."""
        t0 = time.perf_counter()
        vals = self.inputs.scan(self.positions, threads=self.threads)
        dt = time.perf_counter() - t0
        return len(self.positions) * self.n_slices / dt, dt, len(self.positions), vals


def cpu_reference(n_positions: int, threads: int, want_values: bool = False):
    """One warm-up and one timed scan of the C++ float64 restatement on `n_positions` positions of the workload.
    Returns (steps/s, seconds, positions) and, with want_values, the detector values at those positions
    ([detector][position])."""
    ref = CpuReference(n_positions, threads)
    ref.warm_up()
    v, dt, n, vals = ref.step()
    out = (v, dt, n)
    if want_values:
        return out + ([vals[:, d].copy() for d in range(len(DETECTORS))],)
    return out


CPU_SAMPLE = ("{n} of 4096 positions x 20 slices per step, C++17 float64 restatement of STEM.cpuScan "
              "(oracle/cpu/simk_cpu.cpp), {threads} threads over positions")


def host_threads() -> int:
    """Every host thread this process may run on."""
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except AttributeError:
        return max(1, os.cpu_count() or 1)


def cpu_sample_size(requested: int, threads: int) -> int:
    """Positions of the CPU sample: the requested count, at least two per thread so that every thread has work."""
    return min(4096, max(requested, 2 * threads))


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = host_threads()  # all the host threads it can use
    ref = CpuReference(cpu_sample_size(args.cpu_positions, threads), threads)
    for _ in range(args.warmup):
        ref.warm_up()
    vals = []
    for _ in range(args.steps):
        v, dt, n, _ = ref.step()
        vals.append(v)
    value = statistics.median(vals)
    line = {"metric": "probe.slice steps/s", "value": value, "unit": "probe.slice steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * n * 20 / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "config": {"workload": WORKLOAD, "form": "cpu float64"},
            "cpu_baseline": {"value": value, "unit": "probe.slice steps/s", "cores": threads, "kind": "port",
                             "sample": CPU_SAMPLE.format(n=n, threads=threads)},
            "e2e": {"value": value, "unit": "probe.slice steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------------------------------
# Further workloads (--workload 4dstem | surrogate): the same measurement on the other scan configurations
# ---------------------------------------------------------------------------------------------------------------------

def _device_scan(sk, L, engine, probe, pots, positions, dets, torch):
    """A callable running simk_scan_device over `positions` (device-resident) for `pots`, and its output buffers."""
    import ctypes as C
    handles = [p.handle(engine) for p in pots]
    n_pos = len(positions)
    pos_dev = torch.tensor(positions, dtype=torch.float64, device="cuda")
    counts = [int(np.prod(sk.detector_shape(d, probe.grid, probe.beam.energy) or [1])) for d in dets]
    outs = [torch.zeros(n_pos * c, dtype=torch.float64, device="cuda") for c in counts]
    harr = (C.c_void_p * len(handles))(*[h.handle for h in handles])
    darr = (L.Detector_t * len(dets))(*[d.c() for d in dets])
    oarr = (C.c_void_p * len(outs))(*[o.data_ptr() for o in outs])
    pc = probe.c()

    def run():
        L.check(engine.lib.simk_scan_device(engine.handle, C.byref(pc), len(handles), harr, n_pos,
                                            C.c_void_p(pos_dev.data_ptr()), len(dets), darr, oarr))
    return run, outs


def _time_scans(engine, run, steps, warmup, stream, torch, local,
                names=("fused_rows", "fused_cols", "line_fft", "pointwise", "detect")):
    for _ in range(warmup):
        run()
    torch.cuda.synchronize()
    engine.launch_count(reset=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            run()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = engine.launch_count()
    # per-kernel durations from a second, event-instrumented pass
    engine.set_timing(True)
    engine.kernel_time("fused_cols", reset=True)
    run()
    torch.cuda.synchronize()
    kt = {n: engine.kernel_time(n) for n in names}
    engine.set_timing(False)
    return ms, launches, clocks.summary(), kt


def _roofline(kt, n, step_rule=None):
    dom = max(kt, key=lambda k: kt[k][0])
    dms, dn, dbytes = kt[dom]
    peak, kind = measured_peaks()
    achieved = (dbytes / dn) / (dms / dn / 1e3) / 1e9 if dn else None
    total = sum(v[0] for v in kt.values())
    return {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak if achieved else None,
            "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if kind == "measured" else "fallback 6.65 TB/s",
            "traffic": None, "algorithmic_bytes_per_launch": dbytes / dn if dn else None,
            "avg_launch_ms": dms / dn if dn else None,
            "kernel_share": {k: round(v[0] / total, 4) for k, v in kt.items() if v[1]},
            "step_bytes_rule": step_rule or f"32*N bytes per probe.slice step, N = {n}x{n}"}


def run_4dstem(args, sk, L, engine, stream, torch, local):
    """4D-STEM with frozen phonons: Si 6x6x20, 768^2, 80 slices, 16 configurations, 48x48 scan, binned 128x128 up to
    60 mrad + COM (mrad)."""
    a = 5.431
    box, nums, pos = silicon(6, 6, 20)
    st = sk.AtomicStructure(box, nums, pos)
    fp = sk.FrozenPhonons(st, sigmas={14: 0.075}, configurations=args.configs, seed=1)
    pots = [sk.Potential(fp.configuration(c), 768, 768, slice_thickness=1.35775) for c in range(fp.count)]
    assert pots[0].slice_count == 80
    probe = sk.Probe(sk.ElectronBeam(300e3), pots[0].grid, sk.Aperture(25.0), sk.Aberrations(C10=-50.0))
    scan = sk.GridScan((3 * a, 3 * a), (4 * a, 4 * a), args.scan, args.scan)
    dets = [sk.BinnedPixelatedDetector(60.0, (128, 128)), sk.CenterOfMassDetector("valid", "mrad")]
    positions = np.asarray(scan.positions)
    run, outs = _device_scan(sk, L, engine, probe, pots, positions, dets, torch)
    ms, launches, clocks, kt = _time_scans(engine, run, args.steps, args.warmup, stream, torch, local)
    steps = len(positions) * 80 * len(pots)
    value = steps * args.steps / (ms / 1e3)
    cpu, errs = None, None
    if not args.no_cpu:
        # the oracle on config 0 at 2 positions (bounded sample), and the device's single-configuration values there
        from oracle import simk_oracle as O
        idx = [0, len(positions) // 2 + 24]
        x = fp.configuration(0)
        op = O.Potential.from_structure(O.Structure(x.box, x.numbers, x.positions), 768, 768, slice_thickness=1.35775)
        t0 = time.perf_counter()
        ref = O.stem_scan(O.ProbeSpec(300e3, 25.0, {"C10": -50.0}), [(op.grid, op.build(), op.thicknesses)],
                          positions[idx], [O.DetectorSpec("binned", {"nbx": 128, "nby": 128, "outer": 60.0}),
                                           O.DetectorSpec("com", {"mode": "valid", "units": "mrad"})])
        dt = time.perf_counter() - t0
        cpu = {"value": len(idx) * 80 / dt, "unit": "probe.slice steps/s", "cores": 1, "kind": "port",
               "sample": f"{len(idx)} positions x 80 slices of configuration 0 ({dt:.1f} s incl. its potential), "
                         "float64 NumPy restatement"}
        one, o1 = _device_scan(sk, L, engine, probe, pots[:1], positions[idx], dets, torch)
        one()
        torch.cuda.synchronize()
        errs = {"binned": float(np.linalg.norm(o1[0].cpu().numpy() - ref[0].ravel()) / np.linalg.norm(ref[0])),
                "com": float(np.linalg.norm(o1[1].cpu().numpy() - ref[1].ravel()) / np.linalg.norm(ref[1]))}
    return {"metric": "probe.slice steps/s", "value": value, "ms_per_step": ms / args.steps,
            "config": {"workload": f"4D-STEM with frozen phonons, Si 6x6x20 (5760 atoms, 108.6 A), 768x768, 80 "
                                   f"slices of 1.35775 A, {args.configs} configurations (sigma 0.075 A, seed 1), "
                                   f"300 keV, 25 mrad, C10 = -50 A, {args.scan}x{args.scan} scan over one unit cell, "
                                   "binned 128x128 up to 60 mrad + COM",
                       "form": args.form, "steps_per_scan": steps},
            "roofline": _roofline(kt, 768), "cpu_baseline": cpu, "rel_l2_vs_fp64": errs, "clocks": clocks,
            "gpu_launches": launches}


def run_surrogate(args, sk, L, engine, stream, torch, local):
    """The learned potential surrogate feeding a HAADF scan: amorphous 50x50x100 A (25,000 atoms, min separation
    1.4 A, Z from {6: 0.7, 8: 0.2, 14: 0.08, 79: 0.02}), finite projection on 1024^2 with 100 slices of 1 A, built by
    the quadrature and by the surrogate (trained on the device on quadrature-labelled samples); then a 32x32 HAADF
    scan (200 keV, 20 mrad, 50-200 mrad) through the surrogate's potential."""
    box, nums, pos = amorphous((50.0, 50.0, 100.0), 25000, 1.4, {6: 0.7, 8: 0.2, 14: 0.08, 79: 0.02}, seed=1)
    st = sk.AtomicStructure(box, nums, pos)

    def build(**kw):
        p = sk.Potential(st, 1024, 1024, slice_thickness=1.0, projection="finite", **kw)
        torch.cuda.synchronize()
        engine.set_timing(True)
        engine.kernel_time("finite_quadrature", reset=True)
        t0 = time.perf_counter()
        p.handle(engine)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        kq, ks = engine.kernel_time("finite_quadrature"), engine.kernel_time("surrogate_infer")
        engine.set_timing(False)
        return p, wall, kq[0], ks[0]

    pq, wall_q, tq, _ = build()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sur = sk.Surrogate([6, 8, 14, 79], n_samples=args.sg_samples, steps=args.sg_steps, batch=4096, seed=1,
                       engine=engine)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    ps, wall_s, tq_s, ts = build(surrogate=sur, error_bound=0.05)
    vq = pq.build(engine).values
    vs = ps.build(engine).values
    pot_err = {"max_abs_over_max": float(np.max(np.abs(vs - vq)) / np.max(np.abs(vq))),
               "rel_l2": float(np.linalg.norm(vs - vq) / np.linalg.norm(vq))}
    del vq, vs
    probe = sk.Probe(sk.ElectronBeam(200e3), pq.grid, sk.Aperture(20.0))
    scan = sk.GridScan((20.0, 20.0), (30.0, 30.0), 32, 32)
    positions = np.asarray(scan.positions)
    dets = [sk.AnnularDetector(50.0, 200.0)]
    run_s, out_s = _device_scan(sk, L, engine, probe, [ps], positions, dets, torch)
    ms, launches, clocks, kt = _time_scans(engine, run_s, args.steps, args.warmup, stream, torch, local)
    run_q, out_q = _device_scan(sk, L, engine, probe, [pq], positions, dets, torch)
    run_q()
    torch.cuda.synchronize()
    haadf_err = float(torch.linalg.norm(out_s[0] - out_q[0]) / torch.linalg.norm(out_q[0]))
    steps = len(positions) * 100
    value = steps * args.steps / (ms / 1e3)
    info = sur.info
    return {"metric": "probe.slice steps/s", "value": value, "ms_per_step": ms / args.steps,
            "config": {"workload": "amorphous 50x50x100 A (25,000 atoms, min separation 1.4 A, C/O/Si/Au "
                                   "70/20/8/2 %), finite projection 1024x1024, 100 slices of 1 A, learned surrogate, "
                                   "32x32 HAADF scan (50-200 mrad) at 200 keV, 20 mrad", "form": args.form,
                       "steps_per_scan": steps},
            "surrogate": {"train_s": train_s, "samples": args.sg_samples, "steps": args.sg_steps,
                          "val_rms_dF": info.get("val_rms_rel"), "val_max_dF": info.get("val_max_rel"),
                          "used": ps.used_surrogate, "judged_max_dP_over_Pinf": ps.judged_max_rel,
                          "profile_tables_ms": {"quadrature": tq, "surrogate": ts},
                          "potential_build_wall_s": {"quadrature": wall_q, "surrogate": wall_s},
                          "potential_error_vs_quadrature": pot_err,
                          "haadf_rel_l2_vs_quadrature_potential": haadf_err},
            "roofline": _roofline(kt, 1024), "cpu_baseline": None, "clocks": clocks, "gpu_launches": launches}


def hard_core_positions(box, density, dmin, rng):
    """Uniform random positions in `box` (periodic in x and y) at `density` [A^-3] with no two closer than `dmin`: a
    Matern type II hard-core process. Candidates are uniform at the intensity l0 for which the thinning keeps
    `density`, (1 - exp(-l0 v)) / v = density with v the exclusion volume 4/3 pi dmin^3; each gets a random priority,
    and a candidate with a closer one of lower priority is removed."""
    from scipy.spatial import cKDTree
    v = 4.0 / 3.0 * np.pi * dmin ** 3
    l0 = -np.log(1.0 - density * v) / v
    vol = box[0] * box[1] * box[2]
    n0 = int(rng.poisson(l0 * vol))
    pos = rng.uniform(0.0, 1.0, (n0, 3)) * np.asarray(box)
    prio = rng.permutation(n0)
    tree = cKDTree(pos, boxsize=(box[0], box[1], 4.0 * box[2]))  # z not periodic: a box far taller than the cell
    pairs = tree.query_pairs(dmin, output_type="ndarray")
    drop = np.zeros(n0, dtype=bool)
    if len(pairs):
        a, b = pairs[:, 0], pairs[:, 1]
        drop[np.where(prio[a] > prio[b], a, b)] = True
    return pos[~drop]


def random_jobs(n_jobs, seed):
    """The uneven batch: per job a grid from {256, 384, 500, 640}^2, 10-200 slices of U(1, 2) A, an orthogonal cell
    U(20, 40) A wide in x and y, U(80, 300) keV, a plane wave or a 20 mrad probe at the cell centre. Atoms at uniform
    random positions at 0.08 A^-3 with a minimum separation of 1.2 A (hard_core_positions), each atom's Z uniform in
    1-80."""
    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(n_jobs):
        n = int(rng.choice([256, 384, 500, 640]))
        slices = int(rng.integers(10, 201))
        dz = float(rng.uniform(1.0, 2.0))
        lx, ly = rng.uniform(20.0, 40.0, 2)
        box = (float(lx), float(ly), slices * dz)
        pos = hard_core_positions(box, 0.08, 1.2, rng)
        nums = rng.integers(1, 81, len(pos))
        energy = float(rng.uniform(80e3, 300e3))
        probe = bool(rng.integers(0, 2))
        jobs.append(dict(n=n, slices=slices, dz=dz, box=box, nums=nums, pos=pos, energy=energy, probe=probe))
    return jobs


def run_jobs(args, sk, L, engine, stream, torch, local):
    """The uneven batch of 256 jobs: the job table (fused form, jobs of a grid shape advancing together) against the
    same jobs run one after another in the plain form; potentials are built before the timed calls (all 256 jobs'
    potentials and transmissions take about 70 GB of device memory; --jobs-chunk bounds it). value = steps per second
    of the table's device span (from the call's start event, the incident waves included, to the last job's
    completion); the wall clock around each call (which adds the host's copies of the intensities into fresh arrays
    and varies with the host) is reported beside it, for both forms."""
    jobs = random_jobs(256, seed=1)
    chunk = args.jobs_chunk
    t_table, t_seq, done_table, dur_seq, steps, t_setup = 0.0, 0.0, [], [], 0, 0.0
    dev_table, dev_seq = 0.0, 0.0  # device spans of the calls [s]
    last_table = None
    for c0 in range(0, len(jobs), chunk):
        part = jobs[c0:c0 + chunk]
        table = sk.JobTable()
        pots = []
        t0 = time.perf_counter()
        for j in part:
            st = sk.AtomicStructure(j["box"], j["nums"], j["pos"])
            pot = sk.Potential(st, j["n"], j["n"], slice_thicknesses=[j["dz"]] * j["slices"])
            pot.handle(engine)
            pots.append(pot)
            if j["probe"]:
                pr = sk.Probe(sk.ElectronBeam(j["energy"]), pot.grid, sk.Aperture(20.0))
                table.add_probe(pot, pr, (j["box"][0] / 2, j["box"][1] / 2))
            else:
                table.add_plane_wave(pot, j["energy"])
            steps += j["slices"]
        torch.cuda.synchronize()
        t_setup += time.perf_counter() - t0
        fused = sk.ExecutionOptions(form=args.form if args.form != "plain" else "fused")
        table.run(options=fused, engine=engine)  # warm-up: transmissions, plans, propagators
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, done = table.run(options=fused, engine=engine)
        t_table += time.perf_counter() - t0
        done_table += list(done)
        dev_table += float(np.max(done)) / 1e3
        last_table = engine.last_table()  # one graph launch per table call: its kernels and shapes
        plain = sk.ExecutionOptions(form="plain")
        table.run(options=plain, engine=engine)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, done_p = table.run(options=plain, engine=engine)
        t_seq += time.perf_counter() - t0
        dev_seq += float(np.max(done_p)) / 1e3
        dp = np.sort(done_p)
        dur_seq += list(np.diff(np.concatenate([[0.0], dp])))
        del pots, table
    pct = lambda v, q: float(np.percentile(v, q))  # noqa: E731
    return {"metric": "probe.slice steps/s", "value": steps / dev_table, "ms_per_step": 1e3 * dev_table,
            "config": {"workload": "uneven batch: 256 jobs from seed 1, grids {256, 384, 500, 640}^2, 10-200 slices of "
                                   "1-2 A, cells 20-40 A, atoms at 0.08 A^-3 (hard core 1.2 A) with Z uniform in "
                                   "1-80, 80-300 keV, plane wave or 20 mrad probe, exit-wave intensities",
                       "form": args.form, "steps": steps, "chunks_of": chunk, "setup_s": t_setup},
            "jobs": {"table_device_s": dev_table, "sequential_plain_device_s": dev_seq,
                     "speedup_device": dev_seq / dev_table, "sequential_plain_steps_per_s": steps / dev_seq,
                     "table_wall_s": t_table, "sequential_plain_wall_s": t_seq, "speedup_wall": t_seq / t_table,
                     "table_completion_ms": {"p50": pct(done_table, 50), "p99": pct(done_table, 99)},
                     "sequential_job_ms": {"p50": pct(dur_seq, 50), "p99": pct(dur_seq, 99)},
                     "last_table_launch": last_table,
                     "timing": "device spans and completion times from each call's start event; wall clock around "
                               "each call (synchronising); sequential job times = gaps between completions"},
            "roofline": None, "cpu_baseline": None, "clocks": None, "gpu_launches": None}


def run_scanops(args, sk, L, engine, stream, torch, local):
    """Scan post-processing of a 4D-STEM measurement kept on the device: N x N positions (--post-scan, default 64) x
    128 x 128 binned values (float64; 537 MB at 64; synthetic patterns, each summing to 1), the Gaussian source size
    (sigma 0.5 A on 0.2 A scan pixels: 2.5 pixels, 21 taps per axis) then Poisson noise at 1e5 electrons per pattern
    (mean 6.1 per value: Knuth's sampler), in place; one step = a device copy of the measurement and both operations.
    The integrated centre of mass of a 256 x 256 COM scan is timed beside it. value = post-processed values per
    second."""
    import ctypes as C
    ns, nv = args.post_scan, 128
    count = ns * ns * nv * nv
    sigma, samp, dose = 0.5, 0.2, 1e5
    g = torch.Generator(device="cuda").manual_seed(1)
    base = torch.rand((ns * ns, nv * nv), dtype=torch.float64, device="cuda", generator=g)
    base /= base.sum(dim=1, keepdim=True)
    work = torch.empty_like(base)

    def run():
        work.copy_(base)
        p = C.c_void_p(work.data_ptr())
        L.check(engine.lib.simk_gaussian_source_size_device(engine.handle, ns, ns, nv * nv, sigma, sigma, samp, samp,
                                                            p, p))
        L.check(engine.lib.simk_poisson_noise_device(engine.handle, count, p, dose, 1, 7, p))

    ms, launches, clocks, kt = _time_scans(engine, run, args.steps, args.warmup, stream, torch, local,
                                           names=("gauss_axis", "poisson"))
    value = count * args.steps / (ms / 1e3)
    roof = _roofline({"gauss_axis": kt["gauss_axis"]}, 0, step_rule="16 B per value per axis pass (read + write)")
    total_ms = sum(v[0] for v in kt.values())
    roof["kernel_share"] = {k: round(v[0] / total_ms, 4) for k, v in kt.items() if v[1]}
    pois_ms, pois_n, _ = kt["poisson"]
    # iCOM of a 256 x 256 centre-of-mass scan (interleaved pairs, stride 2)
    com = torch.rand(256 * 256 * 2, dtype=torch.float64, device="cuda", generator=g) - 0.5
    icom = torch.empty(256 * 256, dtype=torch.float64, device="cuda")

    def run_icom():
        L.check(engine.lib.simk_integrate_gradient_device(engine.handle, 256, 256, 0.1, 0.1,
                                                          C.c_void_p(com.data_ptr()), C.c_void_p(com.data_ptr() + 8),
                                                          2, C.c_void_p(icom.data_ptr())))
    for _ in range(3):
        run_icom()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(20):
        run_icom()
    e1.record(stream)
    torch.cuda.synchronize()
    icom_ms = e0.elapsed_time(e1) / 20
    # end to end: host arrays through the package's ScanMeasurement methods (copies in and out each call)
    host = base.reshape(-1).cpu().numpy()
    m = sk.ScanMeasurement([ns, ns], [nv, nv], host)
    m.gaussianSourceSize(sigma, samplingX=samp, samplingY=samp, engine=engine)
    t0 = time.perf_counter()
    for _ in range(2):
        m.gaussianSourceSize(sigma, samplingX=samp, samplingY=samp, engine=engine).poissonNoise(dose, seed=7,
                                                                                              engine=engine)
    e2e_s = (time.perf_counter() - t0) / 2
    cpu = None
    if not args.no_cpu:
        # the oracle's float64 Gaussian filter on a bounded sample: every position, 256 values each
        from oracle import simk_oracle as O
        sample = host.reshape(ns, ns, nv * nv)[:, :, :256].copy()
        t0 = time.perf_counter()
        O.gaussian_source_size(sample, [ns, ns], sigma, sigma, samp, samp)
        dt = time.perf_counter() - t0
        cpu = {"value": sample.size / dt, "unit": "values/s", "cores": 1, "kind": "port",
               "sample": f"Gaussian source size only, {ns}x{ns} positions x 256 values ({dt:.2f} s), float64 NumPy "
                         "restatement of ScanMeasurement.gaussianSourceSize"}
    return {"metric": "post-processed values/s", "unit": "values/s", "value": value, "ms_per_step": ms / args.steps,
            "dtype": "f64",
            "config": {"workload": f"scan post-processing of a 4D-STEM measurement on the device: {ns}x{ns} positions "
                                   f"x 128x128 values (float64, {8 * count / 1e6:.0f} MB), Gaussian source size sigma "
                                   "0.5 A at 0.2 A scan pixels (21 taps per axis) + Poisson noise at 1e5 e per "
                                   "pattern, in place", "values": count,
                       "inputs": "larger than L2 at the default size (537 MB), no flush"},
            "roofline": roof, "poisson": {"avg_launch_ms": pois_ms / pois_n if pois_n else None,
                                          "values_per_s": count / (pois_ms / pois_n / 1e3) if pois_n else None},
            "icom_256x256_ms": icom_ms, "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": launches,
            "e2e": {"value": count / e2e_s, "unit": "values/s", "h2d_bytes_per_step": 8 * count * 2,
                    "d2h_bytes_per_step": 8 * count * 2}}


def run_tiling(args, sk, L, engine, stream, torch, local):
    """The headline workload's potential (SrTiO3 8x8x20, 512^2, 20 slices of 3.905 A) built two ways: atom by atom
    from the 6,400-atom crystal, and as one unit cell (64^2, one slice) tiled 8 x 8 x 20 on the device. Each step
    builds both from scratch (new handles); value = the tiled build's time in ms (lower is better). The tile kernel's
    roofline counts its 8-byte writes plus the cell's reads."""
    cell_box, cell_nums, cell_pos = srtio3(1, 1, 1)
    box, nums, pos = srtio3(8, 8, 20)
    cell = sk.AtomicStructure(cell_box, cell_nums, cell_pos)
    crystal = sk.AtomicStructure(box, nums, pos)

    def build_tiled():
        unit = sk.Potential(cell, NX // 8, NY // 8, slice_thickness=SLICE)
        t = unit.tiled(8, 8, 20)
        return t, t.handle(engine)

    def build_direct():
        p = sk.Potential(crystal, NX, NY, slice_thickness=SLICE)
        return p, p.handle(engine)

    for _ in range(max(1, args.warmup)):
        build_tiled()
        build_direct()
    torch.cuda.synchronize()
    times = {"tiled": [], "direct": []}
    for _ in range(args.steps):
        for name, fn in (("tiled", build_tiled), ("direct", build_direct)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            keep = fn()
            engine.synchronize()
            times[name].append(1e3 * (time.perf_counter() - t0))
            del keep
    engine.set_timing(True)
    engine.kernel_time("tile", reset=True)
    t, _ = build_tiled()
    engine.synchronize()
    kt = {"tile": engine.kernel_time("tile")}
    engine.set_timing(False)
    roof = _roofline(kt, 0, step_rule="8 B written per tiled value + 8 B per cell value read")
    vt = t.build(engine).values
    vd = sk.Potential(crystal, NX, NY, slice_thickness=SLICE).build(engine).values
    err = float(np.max(np.abs(vt - vd)) / np.max(np.abs(vd)))
    tiled_ms, direct_ms = statistics.median(times["tiled"]), statistics.median(times["direct"])
    return {"metric": "potential build ms", "unit": "ms", "value": tiled_ms, "ms_per_step": tiled_ms,
            "higher_is_better": False, "dtype": "f64",
            "config": {"workload": "the STEM workload's potential (SrTiO3 8x8x20, 512x512, 20 slices of 3.905 A): one "
                                   "cell on 64x64 tiled 8x8x20 on the device, against the 6,400-atom build",
                       "inputs": "42 MB written per build; wall clock around each build, synchronised"},
            "tiling": {"tiled_ms": tiled_ms, "direct_ms": direct_ms, "speedup": direct_ms / tiled_ms,
                       "rel_max_tiled_vs_direct": err},
            "roofline": roof, "cpu_baseline": None, "clocks": None, "gpu_launches": None}


def run_extra(args):
    import torch
    import simulatokit_b200 as sk
    from simulatokit_b200 import _lib as L
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if int(os.environ.get("RANK", "0")) != 0:
        return  # one GPU: these workloads have no replica mode
    torch.cuda.set_device(local)
    engine = sk.Engine.require(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    engine.set_stream(stream.cuda_stream)
    engine.apply(sk.ExecutionOptions(form=args.form, batch=args.batch, col_tile=args.col_tile, tma=not args.no_tma,
                                     autotune=args.autotune, tcgen05=args.tcgen05, composite=bool(args.composite)))
    fn = {"4dstem": run_4dstem, "surrogate": run_surrogate, "jobs": run_jobs, "scanops": run_scanops,
          "tiling": run_tiling}[args.workload]
    line = fn(args, sk, L, engine, stream, torch, local)
    for k, v in {"unit": "probe.slice steps/s", "dtype": "f32", "e2e": None}.items():
        line.setdefault(k, v)
    line.setdefault("higher_is_better", True)
    line.update({"n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "scaling": "weak", "vs_baseline": None,
                 "data": "synthetic"})
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------------------------------------------------

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="fused", choices=["plain", "fused", "bf16x3"])
    ap.add_argument("--batch", type=int, default=0)
    ap.add_argument("--col-tile", type=int, default=0)
    ap.add_argument("--no-tma", action="store_true")
    ap.add_argument("--autotune", action="store_true", help="time column tile, TMA passes and batch on first use")
    ap.add_argument("--cpu-positions", type=int, default=32)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the per-form comparison after the headline")
    ap.add_argument("--no-other-configs", action="store_true",
                    help="skip the 4D-STEM sample (2 configurations, fused and bf16x3) reported after the headline")
    ap.add_argument("--composite", type=int, default=1, choices=[0, 1],
                    help="fused passes at 3 or 5 times a power of two: 1 composite register engine, 0 shared-memory")
    ap.add_argument("--tcgen05", type=int, default=2, choices=[0, 1, 2],
                    help="bf16x3 engine: 2 tcgen05 stacked (six products a stage), 1 tcgen05 (twelve), 0 mma.sync")
    ap.add_argument("--workload", default="stem", choices=["stem", "4dstem", "surrogate", "jobs", "scanops", "tiling"],
                    help="stem: the headline STEM HAADF+BF scan; 4dstem, surrogate, jobs: the other configurations; "
                         "scanops: scan post-processing of a 4D-STEM measurement; tiling: the headline potential "
                         "built from a tiled unit cell")
    ap.add_argument("--sg-samples", type=int, default=10_000_000, help="surrogate workload: quadrature samples")
    ap.add_argument("--sg-steps", type=int, default=20000, help="surrogate workload: training steps")
    ap.add_argument("--jobs-chunk", type=int, default=256, help="jobs workload: jobs per table call")
    ap.add_argument("--configs", type=int, default=16, help="4dstem workload: frozen-phonon configurations")
    ap.add_argument("--scan", type=int, default=48, help="4dstem workload: scan positions per side")
    ap.add_argument("--post-scan", type=int, default=64, help="scanops workload: scan positions per side")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload != "stem":
        run_extra(args)
        return

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import ctypes as C

    import simulatokit_b200 as sk
    from simulatokit_b200 import _lib as L

    engine = sk.Engine.require(local)
    # a real (non-NULL) stream shared by torch's events and the library: the library maps NULL to its own stream
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    assert stream.cuda_stream != 0
    engine.set_stream(stream.cuda_stream)
    opts = sk.ExecutionOptions(form=args.form, batch=args.batch, col_tile=args.col_tile, tma=not args.no_tma,
                               autotune=args.autotune, tcgen05=args.tcgen05, composite=bool(args.composite))
    engine.apply(opts)

    box, nums, pos = srtio3(8, 8, 20)
    structure = sk.AtomicStructure(box, nums, pos)
    pot = sk.Potential(structure, NX, NY, slice_thickness=SLICE)
    assert pot.slice_count == 20
    beam = sk.ElectronBeam(ENERGY)
    probe = sk.Probe(beam, pot.grid, sk.Aperture(SEMIANGLE))
    dets = [sk.AnnularDetector(a, b) for _, a, b in DETECTORS]
    positions = scan_positions()
    n_pos = len(positions)
    steps_per_scan = n_pos * pot.slice_count

    # device-resident inputs and outputs
    h = pot.handle(engine)
    pos_dev = torch.tensor(positions, dtype=torch.float64, device="cuda")
    outs = [torch.zeros(n_pos, dtype=torch.float64, device="cuda") for _ in dets]
    harr = (C.c_void_p * 1)(h.handle)
    darr = (L.Detector_t * len(dets))(*[d.c() for d in dets])
    oarr = (C.c_void_p * len(outs))(*[o.data_ptr() for o in outs])
    pc = probe.c()

    def scan_once():
        L.check(engine.lib.simk_scan_device(engine.handle, C.byref(pc), 1, harr, n_pos, C.c_void_p(pos_dev.data_ptr()),
                                            len(dets), darr, oarr))

    for _ in range(max(3, args.warmup)):
        scan_once()
    torch.cuda.synchronize()

    def timed_region(with_kernel_timing: bool):
        engine.set_timing(with_kernel_timing)
        engine.kernel_time("line_fft", reset=True)
        engine.launch_count(reset=True)
        if dist:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clocks:
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(args.steps):
                scan_once()
            e1.record(stream)
            torch.cuda.synchronize()
        if dist:
            dist.barrier()
        return e0.elapsed_time(e1), engine.launch_count(), clocks

    # the headline: K scans with nothing else on the stream
    ms, launches, clocks = timed_region(False)
    # the same K scans again with CUDA events around every launch, for the per-kernel durations of the roofline
    ms_k, _, _ = timed_region(True)
    names = ["fused_rows", "fused_cols", "line_fft", "pointwise", "detect"]
    ktimes = {n: engine.kernel_time(n) for n in names}
    engine.set_timing(False)
    ms_max = slowest_rank(ms, dist, "cuda")
    value = whole_job_rate(steps_per_scan * args.steps, world, ms_max / 1e3)

    # dominant kernel: the largest total time
    dom = max(ktimes, key=lambda n: ktimes[n][0])
    dms, dn, dbytes = ktimes[dom]
    peak, peak_kind = measured_peaks()
    traffic, traffic_source = traffic_from_profiles(f"{dom}@{args.form}")
    achieved = (dbytes / dn) / (dms / dn / 1e3) / 1e9 if dn else None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                if peak_kind == "measured" else "fallback 6.65 TB/s",
                "traffic": traffic, "traffic_source": traffic_source,
                "algorithmic_bytes_per_launch": dbytes / dn if dn else None,
                "avg_launch_ms": dms / dn if dn else None,
                "kernel_share": {n: round(ktimes[n][0] / ms_k, 4) for n in names if ktimes[n][1]},
                "timing_pass_ratio": round(ms_k / ms, 4),
                "step_bytes_rule": "32*N bytes per probe.slice step (two read+write passes of the complex64 wave)",
                "step_roofline_frac": (value / world) * 32 * NX * NY / (peak * 1e9)}

    # e2e: the public API from host arrays, potential built on the device each call
    e2e_val = None
    h2d = d2h = 0
    if args.e2e_steps > 0:
        scan = sk.GridScan((4 * A0, 4 * A0), (5 * A0, 5 * A0), SCAN_N, SCAN_N)
        times = []
        for it in range(args.e2e_steps + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            p2 = sk.Potential(structure, NX, NY, slice_thickness=SLICE)
            res = sk.STEM.scan(probe, [p2], scan, dets, options=opts, engine=engine)
            torch.cuda.synchronize()
            if it > 0:
                times.append(time.perf_counter() - t0)
            del p2
        e2e_val = whole_job_rate(steps_per_scan, world, slowest_rank(statistics.median(times), dist, "cuda"))
        n_atoms = len(nums)
        h2d = n_atoms * (4 + 24 + 4) + 20 * 8 + n_pos * 16
        d2h = sum(n_pos * 8 for _ in dets)
        engine.apply(opts)
        engine.set_stream(stream.cuda_stream)

    # every form on the same scan (one timed scan each after a warm-up), for the metric's form comparison
    forms, form_values = {}, {}
    if rank == 0 and world == 1 and not args.no_forms:
        # bf16x3: the tcgen05 engine with six stacked products a stage (the form's default at this grid);
        # bf16x3_twelve: the same terms as twelve products; bf16x3_mma_sync: the warp-level mma.sync stages
        engines = {"bf16x3": 2, "bf16x3_twelve": 1, "bf16x3_mma_sync": 0}
        for f in ("plain", "fused", "bf16x3", "bf16x3_twelve", "bf16x3_mma_sync"):
            engine.apply(sk.ExecutionOptions(form=f.split("_")[0], batch=args.batch, col_tile=args.col_tile,
                                             tma=not args.no_tma, autotune=args.autotune,
                                             tcgen05=engines.get(f, 2)))
            engine.set_stream(stream.cuda_stream)
            scan_once()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            scan_once()
            e1.record(stream)
            torch.cuda.synchronize()
            fms = e0.elapsed_time(e1)
            forms[f] = {"value": steps_per_scan / (fms / 1e3), "ms_per_scan": fms}
            form_values[f] = [o.cpu().numpy().copy() for o in outs]
        engine.apply(opts)
        engine.set_stream(stream.cuda_stream)
        if "bf16x3" in forms and "fused" in forms and "plain" in forms:
            forms["bf16x3_over_fused"] = forms["bf16x3"]["value"] / forms["fused"]["value"]
            forms["bf16x3_over_plain"] = forms["bf16x3"]["value"] / forms["plain"]["value"]
            forms["fused_over_plain"] = forms["fused"]["value"] / forms["plain"]["value"]

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = host_threads()
        n_cpu = cpu_sample_size(args.cpu_positions, threads)
        v, dt, n, ref_vals = cpu_reference(n_cpu, threads, want_values=True)
        cpu = {"value": v, "unit": "probe.slice steps/s", "cores": threads, "kind": "port",
               "sample": CPU_SAMPLE.format(n=n, threads=threads) + f" ({dt:.1f} s)"}
        idx = sample_indices(n_cpu)
        for f, vals in form_values.items():
            errs = [float(np.linalg.norm(vals[d][idx] - ref_vals[d]) / np.linalg.norm(ref_vals[d]))
                    for d in range(len(dets))]
            forms[f]["rel_l2_vs_fp64"] = dict(zip([name for name, _, _ in DETECTORS], errs))
        if forms:
            forms["error_sample"] = f"detector values at the {n} CPU sample positions vs the C++ float64 restatement"

    # the 768^2 4D-STEM configuration on a 2-configuration sample, fused and bf16x3, reported beside the headline (one
    # GPU only; never fails the headline)
    other = None
    if rank == 0 and world == 1 and not args.no_other_configs:
        other = {}
        for f in ("fused", "bf16x3"):
            try:
                ns = argparse.Namespace(**vars(args))
                ns.configs, ns.scan, ns.steps, ns.warmup, ns.no_cpu, ns.form = 2, 48, 1, 1, True, f
                engine.apply(sk.ExecutionOptions(form=f))
                engine.set_stream(stream.cuda_stream)
                r = run_4dstem(ns, sk, L, engine, stream, torch, local)
                rf = r.get("roofline") or {}
                other[f"4dstem_2cfg_{f}"] = {"value": r["value"], "unit": "probe.slice steps/s",
                                             "ms_per_step": r["ms_per_step"], "roofline_frac": rf.get("frac"),
                                             "workload": r["config"]["workload"]}
            except Exception as exc:  # reported, not raised: the headline line must still print
                other[f"4dstem_2cfg_{f}"] = {"error": repr(exc)[:300]}

    if rank == 0:
        line = {"metric": "probe.slice steps/s", "value": value, "unit": "probe.slice steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": WORKLOAD, "form": args.form, "batch": args.batch, "col_tile": args.col_tile,
                           "tma": not args.no_tma, "autotune": args.autotune,
                           "positions": n_pos, "slices": 20,
                           "grid": [NX, NY], "replicas": world, "l2": "inputs larger than L2 (batch of waves up to "
                                                                     "1 GiB per launch)"},
                "roofline": roofline, "cpu_baseline": cpu, "forms": forms or None, "other_configs": other,
                "clocks": clocks.summary(), "gpu_launches": launches,
                "e2e": {"value": e2e_val, "unit": "probe.slice steps/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h}}
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
