#!/usr/bin/env python3
"""Benchmark: S(q) + partials frames/s on the precision-form workload.

Workload (the headline configuration): cubic box L = 220 A, N = 1,000,000 atoms,
3 types (fractions 0.5 / 0.3 / 0.2, shuffled), uniform base positions plus a
fresh Gaussian jitter (sigma 0.3 A) per frame, neutron weights b = 4.149, 5.803,
9.45 fm, q_max = 6 1/A (423^3 modes), nq 500, norm mean, partials on, NUFFT
tolerance 1e-6, FP32 spread / FFT / deconvolution with FP64 shell accumulation.
One step = one frame through the hot path.  Synthetic data, seeded.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun each rank runs its own frames (frames are independent units)
and the accumulators are summed once at the end; the rank timings are reduced
with MAX.  One JSON line is printed by rank 0.
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

METRIC = "S(q) frames/s at N=1M (FP32 spread/FFT + FP64 accumulation, partials)"
UNIT = "frames/s"
N_ATOMS = 1_000_000
BOX = 220.0
# --scale s shrinks the box by s at fixed density (profiling runs only)
SCALE = 1.0
FRACTIONS = (0.5, 0.3, 0.2)
B_NEUTRON = (4.149, 5.803, 9.45)
QMAX, NQ, EPS = 6.0, 500, 1e-6
JITTER = 0.3
SEED = 20240601


def workload_types(rng):
    # type_assignment of the reference generator: rounded counts, shuffled.
    counts = [int(round(f * N_ATOMS)) for f in FRACTIONS[:-1]]
    counts.append(N_ATOMS - sum(counts))
    types = np.repeat(np.arange(1, len(FRACTIONS) + 1, dtype=np.int32), counts)
    rng.shuffle(types)
    return types


def make_frames(nframes, seed):
    rng = np.random.default_rng(seed)
    types = workload_types(rng)
    base = rng.random((N_ATOMS, 3)) * BOX
    frames = np.empty((nframes, N_ATOMS, 3))
    for f in range(nframes):
        frames[f] = base + rng.normal(0.0, JITTER, (N_ATOMS, 3))
    return types, frames


def workload_config(extra=None):
    cfg = {"workload": "precision form: cubic L=220 A, N=1e6, 3 types 0.5/0.3/0.2, "
                       "uniform + per-frame N(0,0.3^2) jitter, neutron b=4.149/5.803/9.45 fm, "
                       "qmax 6 (423^3 modes), nq 500, norm mean, partials, eps 1e-6",
           "natoms": N_ATOMS, "box": BOX, "qmax": QMAX, "nq": NQ, "eps": EPS,
           "modes": [423, 423, 423], "l2": "inputs larger than L2 (fine grids > 126 MB)"}
    if extra:
        cfg.update(extra)
    return cfg


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples every 50 ms with their arrival time; started before
    the warm-up so that it is running when the timed region begins, and
    summarised over the samples that arrived inside that region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.idx = device_index
        self.proc = None
        self.lines = []
        self.window = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def wait_first(self, timeout=5.0):
        t0 = time.monotonic()
        while self.proc is not None and not self.lines and time.monotonic() - t0 < timeout:
            time.sleep(0.01)

    def mark(self, t0, t1):
        self.window = (t0, t1)

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.06)  # one more sample after the region
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        lines = self.lines
        if self.window is not None:
            t0, t1 = self.window
            inside = [x for x in lines if t0 <= x[0] <= t1 + 0.05]
            lines = inside if inside else lines[-1:]
        for _, line in lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# measured peaks
# ---------------------------------------------------------------------------
def hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def dram_traffic(kernel):
    """Per-launch DRAM bytes of a kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    try:
        for line in open(path):
            parts = line.split()
            if len(parts) >= 2 and not line.startswith("#") and parts[0] == kernel:
                return float(parts[1])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------
# reference arm: the CPU restatement of the reference's CPU path
# ---------------------------------------------------------------------------
def run_reference(args, rank, world):
    if rank != 0:
        return
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    types, frames = make_frames(1, SEED)
    w = O.Weights(kind=O.WEIGHT_NEUTRON, amp_const=np.array(B_NEUTRON))
    cell = np.eye(3) * BOX
    # one frame is ~10-30 s on a few host cores: run warm-up and steps on one
    # frame each, at most a bounded number of them
    t_est0 = time.perf_counter()
    O.nufft_cpu_sq([frames[0]], types, cell, np.zeros(3), w, 0.0, QMAX, NQ, eps=EPS,
                   sigma=1.25, workers=cores)
    t_one = time.perf_counter() - t_est0
    steps = max(1, min(args.steps, int(150.0 / max(t_one, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(steps):
        O.nufft_cpu_sq([frames[0]], types, cell, np.zeros(3), w, 0.0, QMAX, NQ, eps=EPS,
                       sigma=1.25, workers=cores)
    dt = time.perf_counter() - t0
    v = steps / dt
    sample = ("%d frame(s) of the workload through the CPU restatement of the reference's "
              "FINUFFT CPU path (ES spread C/OpenMP, pocketfft rfftn, deconvolve + shell sums), "
              "sigma 1.25, FP64" % steps)
    print(json.dumps({
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
        "warmup": 1, "ms_per_step": 1e3 * dt / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference", "config": workload_config({"parallelism": "cpu"}),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def cpu_baseline_sample():
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    types, frames = make_frames(1, SEED)
    w = O.Weights(kind=O.WEIGHT_NEUTRON, amp_const=np.array(B_NEUTRON))
    t0 = time.perf_counter()
    O.nufft_cpu_sq([frames[0]], types, np.eye(3) * BOX, np.zeros(3), w, 0.0, QMAX, NQ, eps=EPS,
                   sigma=1.25, workers=cores)
    dt = time.perf_counter() - t0
    return {"value": 1.0 / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "1 frame of the workload (N=1e6, 3 types, 423^3 modes) through the CPU "
                      "restatement of the reference's FINUFFT CPU path, sigma 1.25, FP64, "
                      "%d threads, %.1f s" % (cores, dt)}


def _max_over_ranks(x, dist, local_rank):
    if not dist:
        return x
    import torch
    import torch.distributed as td
    t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local_rank}")
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def precision_leg(types, dev, base, fbytes, W, K, stream, dist, world, local_rank):
    """The plain FP64 path on the same device-resident frames, at the benchmark's
    eps 1e-6 and at sqcalc's default eps 1e-9 (src/sqc_options.f90:87), and max
    |dS| of the FP32 path against FP64 at eps 1e-12 on two frames."""
    import torch
    from sqcalc_b200 import _lib

    def plan(prec, eps):
        return _lib.Plan(np.eye(3).reshape(9) * BOX, np.zeros(3), types,
                         weight=_lib.WEIGHT_NEUTRON, amp_const=np.array(B_NEUTRON), qmin=0.0,
                         qmax=QMAX, nq=NQ, norm=_lib.NORM_MEAN, partials=True, precision=prec,
                         eps=eps, device=local_rank, stream=stream.cuda_stream)

    def timed(eps):
        k = min(K, 10)
        p = plan(_lib.PREC_DOUBLE, eps)
        for f in range(W):
            p.accumulate((base + f * fbytes, 1), where=_lib.DEVICE)
        p.sync()
        if dist:
            import torch.distributed as td
            td.barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for f in range(W, W + k):
            p.accumulate((base + f * fbytes, 1), where=_lib.DEVICE)
        ev1.record(stream)
        torch.cuda.synchronize()
        t = _max_over_ranks(ev0.elapsed_time(ev1) * 1e-3, dist, local_rank)
        out = {"value": k * world / t, "unit": UNIT, "steps": k, "ms_per_step": 1e3 * t / k,
               "eps": eps, "upsampfac": p.info.upsampfac, "kernel_width": p.info.kernel_width,
               "fine_grid": list(p.info.nf)}
        p.close()
        return out

    fp64 = timed(EPS)
    fp64["sqcalc_default_eps"] = timed(1e-9)
    res = {}
    for name, prec, eps in (("fp32", _lib.PREC_SINGLE, EPS), ("fp64_ref", _lib.PREC_DOUBLE, 1e-12)):
        q = plan(prec, eps)
        for f in range(2):
            q.accumulate((base + f * fbytes, 1), where=_lib.DEVICE)
        s, sp, _, _ = q.finalize()
        res[name] = (s, sp)
        q.close()
    fp64["max_abs_dS_fp32"] = float(np.max(np.abs(res["fp32"][0] - res["fp64_ref"][0])))
    fp64["max_abs_dS_partials_fp32"] = float(np.max(np.abs(res["fp32"][1] - res["fp64_ref"][1])))
    fp64["dS_reference"] = "FP64 NUFFT at eps 1e-12 on the same 2 frames"
    return fp64


def reference_gpu_baseline(types, dev, W, K, stream, local_rank):
    """The reference's own GPU kernel on this GPU: cuFINUFFT built from the
    reference's vendored sources (external/finufft/src/cuda) for sm_100a by
    oracle/cufinufft.mk, called with sqcalc's options (src/sqc_gpu.f90:185-204:
    default opts, modeord 0, type 1, iflag +1, one transform per species) on the
    benchmark's frames: coordinates 2 pi s - pi of the wrapped fractional
    positions (:230-236) and one-hot species strengths, already on the device.
    Timed per frame: setpts + execute, the device part of the reference's frame
    (it then downloads the 3 x 423^3 mode cube and bins on the host).  FP32 at
    eps 1e-6 and FP64 at sqcalc's default eps 1e-9.  Beside each: this
    library's cuFINUFFT-shaped type-1 entry points (sqn_type1_*) on the same
    points and strengths, transform for transform."""
    import torch
    from oracle import cufinufft_ref as REF
    from sqcalc_b200 import _lib
    if not REF.available():
        return {"unavailable": "oracle/_ref/libcufinufft.so was not built"}
    modes = (423, 423, 423)
    species = sorted(set(int(t) for t in np.unique(types)))
    T = len(species)
    k = min(K, 5)
    nfr = min(dev.shape[0], 4)
    out = {"note": "device-only setpts + execute per frame, CUDA events on the launching "
                   "stream; sqcalc's options (type 1, iflag +1, modeord 0, ntransf 3, default "
                   "method); the same points and strengths for sqn_type1",
           "modes": list(modes), "ntransf": T, "steps": k}
    for fp64, eps in ((False, 1e-6), (True, 1e-9)):
        rdt = torch.float64 if fp64 else torch.float32
        cdt = torch.complex128 if fp64 else torch.complex64
        tid = torch.from_numpy(types.astype(np.int64)).cuda()
        c = torch.zeros((T, N_ATOMS), dtype=cdt, device="cuda")
        for a, t in enumerate(species):
            c[a][tid == t] = 1.0
        xyz = []
        for f in range(nfr):
            sfrac = torch.remainder(dev[f] / BOX, 1.0)
            xyz.append([(2 * np.pi * sfrac[:, d] - np.pi).to(rdt).contiguous() for d in range(3)])
        fk = torch.empty((T, modes[2], modes[1], modes[0]), dtype=cdt, device="cuda")
        torch.cuda.synchronize()
        res = {}
        with REF.Type1Plan(modes, T, eps, fp64, device=local_rank,
                           stream=stream.cuda_stream) as rp:
            def ref_frame(f):
                x = xyz[f % nfr]
                rp.setpts(N_ATOMS, x[0].data_ptr(), x[1].data_ptr(), x[2].data_ptr())
                rp.execute(c.data_ptr(), fk.data_ptr())
            res["cufinufft"] = _event_time(ref_frame, W, k, stream)
        with _lib.Type1Plan(modes, iflag=1, ntransf=T, eps=eps,
                            precision=_lib.PREC_DOUBLE if fp64 else _lib.PREC_SINGLE,
                            device=local_rank, stream=stream.cuda_stream) as op:
            def our_frame(f):
                op.setpts(*xyz[f % nfr])
                op.execute(c)
            res["sqn_type1"] = _event_time(our_frame, W, k, stream)
        del fk, c, xyz
        torch.cuda.empty_cache()
        name = "f64" if fp64 else "f32"
        for key, ms in res.items():
            out["%s_%s" % (key, name)] = {"frames_per_s": 1e3 / ms, "ms_per_frame": ms, "eps": eps}
    return out


def _event_time(step, W, k, stream):
    """ms per step of step(f) over k steps after W warm-up steps (CUDA events)."""
    import torch
    for f in range(W):
        step(f)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for f in range(W, W + k):
        step(f)
    ev1.record(stream)
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1) / k


def small_fp64_leg(W, K, stream, local_rank):
    """The CPU-runnable configuration (plain FP64 static S(q)): cubic L = 20 A,
    N = 8000, 2 types 2667 / 5333, i.i.d. uniform frames, unit weights, norm
    mean, partials, NUFFT tolerance 1e-9 (sqcalc's default), q_max 10 (65^3
    modes), nq 500.  The plan in FP64 and in FP32 with FP64 accumulation, frames
    device-resident; beside them the reference's cuFINUFFT (FP64, eps 1e-9) on
    the same frames (setpts + execute only, see reference_gpu_baseline)."""
    import torch
    from sqcalc_b200 import _lib
    rng = np.random.default_rng(SEED + 11)
    n, box, nfr = 8000, 20.0, 10
    types = np.repeat(np.array([1, 2], dtype=np.int32), [2667, n - 2667])
    rng.shuffle(types)
    frames = torch.from_numpy(rng.random((nfr, n, 3)) * box).cuda()
    k = max(K, 20)
    out = {"workload": "plain FP64 form: cubic L=20 A, N=8000, 2 types 2667/5333, uniform, "
                       "unit weights, norm mean, partials, eps 1e-9, qmax 10 (65^3 modes), nq 500",
           "steps": k}
    for name, prec in (("f64", _lib.PREC_DOUBLE), ("f32+f64acc", _lib.PREC_SINGLE)):
        with _lib.Plan(np.eye(3).reshape(9) * box, np.zeros(3), types, qmin=0.0, qmax=10.0,
                       nq=500, norm=_lib.NORM_MEAN, partials=True, precision=prec, eps=1e-9,
                       device=local_rank, stream=stream.cuda_stream) as p:
            fb = n * 3 * 8
            step = lambda f: p.accumulate((frames.data_ptr() + (f % nfr) * fb, 1),  # noqa: E731
                                          where=_lib.DEVICE)
            ms = _event_time(step, W, k, stream)
            out[name] = {"frames_per_s": 1e3 / ms, "ms_per_frame": ms,
                         "fine_grid": list(p.info.nf), "kernel_width": p.info.kernel_width,
                         "eps_used": p.info.eps_used}
    from oracle import cufinufft_ref as REF
    if REF.available():
        T = 2
        c = torch.zeros((T, n), dtype=torch.complex128, device="cuda")
        tid = torch.from_numpy(types.astype(np.int64)).cuda()
        for a in range(T):
            c[a][tid == a + 1] = 1.0
        xyz = [[(2 * np.pi * torch.remainder(frames[f][:, d] / box, 1.0) - np.pi).contiguous()
                for d in range(3)] for f in range(nfr)]
        fk = torch.empty((T, 65, 65, 65), dtype=torch.complex128, device="cuda")
        with REF.Type1Plan((65, 65, 65), T, 1e-9, True, device=local_rank,
                           stream=stream.cuda_stream) as rp:
            def ref_frame(f):
                x = xyz[f % nfr]
                rp.setpts(n, x[0].data_ptr(), x[1].data_ptr(), x[2].data_ptr())
                rp.execute(c.data_ptr(), fk.data_ptr())
            ms = _event_time(ref_frame, W, k, stream)
        out["reference_cufinufft_f64_device_only"] = {"frames_per_s": 1e3 / ms, "ms_per_frame": ms}
    return out


def solid_leg(W, K, stream, local_rank):
    """The structured-solid configuration: triclinic FCC crystal, a = 4 A,
    64^3 cells (N = 1,048,576), tilts xy = 5, xz = 3, 2 types alternating on the
    sublattices, Gaussian thermal displacement sigma 0.1 A, IT92 x-ray weights
    (Cu / Au), q_max 10 (817^3 modes: above the reference's 4e8 mode cap, which
    refuses this run), nq 500, FP32 spread / FFT with FP64 accumulation, eps
    1e-6, partials.  Frames device-resident."""
    import torch
    from sqcalc_b200 import _lib
    from sqcalc_b200.synthetic import fcc_solid
    from sqcalc_b200.weights import WeightScheme
    pos0, types, cell = fcc_solid(64)
    rng = torch.Generator(device="cuda").manual_seed(SEED + 13)
    base = torch.from_numpy(pos0).cuda()
    nfr = 4
    frames = torch.stack([base + 0.1 * torch.randn(base.shape, generator=rng, device="cuda",
                                                   dtype=torch.float64) for _ in range(nfr)])
    scheme = WeightScheme.from_options("xray", "1:Cu,2:Au")
    k = min(K, 10)
    with _lib.Plan(cell.reshape(9), np.zeros(3), types, ntypes=2, weight=_lib.WEIGHT_XRAY,
                   xray_coef=scheme.xray_rows(2), qmin=0.0, qmax=10.0, nq=500,
                   norm=_lib.NORM_MEAN, partials=True, precision=_lib.PREC_SINGLE, eps=1e-6,
                   max_grid_modes=-1, device=local_rank, stream=stream.cuda_stream) as p:
        fb = len(types) * 3 * 8
        step = lambda f: p.accumulate((frames.data_ptr() + (f % nfr) * fb, 1),  # noqa: E731
                                      where=_lib.DEVICE)
        ms = _event_time(step, W, k, stream)
        info = p.info
        out = {"workload": "structured solid: triclinic FCC a=4 A, 64^3 cells (N=1048576), "
                           "tilts xy=5 xz=3, 2 types on sublattices, thermal sigma 0.1 A, "
                           "IT92 x-ray (Cu/Au), qmax 10 (817^3 modes), nq 500, FP32+FP64acc, "
                           "eps 1e-6, partials",
               "frames_per_s": 1e3 / ms, "ms_per_frame": ms, "steps": k,
               "modes": list(info.modes), "fine_grid": list(info.nf),
               "kernel_width": info.kernel_width,
               "reference": "refuses this grid (817^3 modes above its 4e8 cap, "
                            "src/sqc_structure_factor.f90:340-345)"}
    del frames
    torch.cuda.empty_cache()
    return out


BATCH_SYSTEMS, BATCH_QMAX, BATCH_NQ, BATCH_FRAMES = 64, 8.0, 400, 20


def batched_leg(W, K, stream, dist, local_rank):
    """Batched form: 64 independent cubic systems, N ~ U[5k, 200k] at 0.08 A^-3,
    2 types 1:2, uniform positions, q_max 8, FP32 + FP64 accumulation, partials,
    each system's fine grid and kernel width chosen by the autotuner.  One step
    = one frame of every system = one CUDA graph launch, inside which the sort,
    the spread and the binning of all 64 systems run as one launch each and the
    systems' FFTs as parallel branches.  Reported beside it: the same plans
    launched one after another from the host without the graph."""
    import torch
    from sqcalc_b200 import _lib
    from sqcalc_b200.synthetic import batched_systems

    systems = batched_systems(BATCH_SYSTEMS, SEED + 3)
    kws = [dict(cell=np.eye(3).reshape(9) * box, origin=np.zeros(3), type_id=types, qmin=0.0,
                qmax=BATCH_QMAX, nq=BATCH_NQ, partials=True, precision=_lib.PREC_SINGLE,
                eps=EPS, device=local_rank, autotune=True) for _, box, types in systems]
    t0 = time.perf_counter()
    batch = _lib.Batch(kws, stream=stream.cuda_stream)
    t_create = time.perf_counter() - t0
    gen = torch.Generator(device=f"cuda:{local_rank}").manual_seed(SEED + 5)
    nfr = 4  # distinct i.i.d. frames per system, cycled
    dev = [torch.rand((nfr, n, 3), generator=gen, device=f"cuda:{local_rank}",
                      dtype=torch.float64) * box for n, box, _ in systems]
    torch.cuda.synchronize()
    step = lambda f: batch.accumulate([d[f % nfr].data_ptr() for d in dev],  # noqa: E731
                                      where=_lib.DEVICE, nframes=1)
    for f in range(W):
        step(f)
    batch.sync()
    k = min(K, BATCH_FRAMES)
    l0 = batch.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for f in range(k):
        step(W + f)
    ev1.record(stream)
    torch.cuda.synchronize()
    t = _max_over_ranks(ev0.elapsed_time(ev1) * 1e-3, dist, local_rank)
    launches = batch.launch_count() - l0
    # the same plans without the graph: host-issued launches, system after system
    batch.sync()
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for f in range(k):
        for v, d in zip(batch.plans, dev):
            v.accumulate((d[(W + f) % nfr].data_ptr(), 1), where=_lib.DEVICE)
    for v in batch.plans:
        v.sync()
    t_nograph = time.perf_counter() - t1
    natoms = sum(n for n, _, _ in systems)
    # fine-grid cells transformed per step (each system's transforms x nf1 nf2 nf3):
    # the unit the FFT and, with the atoms, the spread scale with; q_max 8 at
    # 0.08 A^-3 gives these systems ~2.8x the cells per atom of the single-system
    # workload, so atom-frames/s alone does not compare the two forms
    cells = sum(int(v.info.ntransforms) * int(np.prod(np.array(v.info.nf, dtype=np.int64)))
                for v in batch.plans)
    out = {"metric": "batched S(q) system-frames/s", "unit": "system-frames/s",
           "value": k * BATCH_SYSTEMS / t, "atom_frames_per_s": k * natoms / t,
           "grid_cells_per_s": k * cells / t, "grid_cells_per_step": cells,
           "ms_per_step": 1e3 * t / k, "steps": k, "systems": BATCH_SYSTEMS,
           "natoms_total": natoms, "graph_launches_per_step": 1,
           "gpu_launches_per_step": launches / k,
           "no_graph_ms_per_step_wall": 1e3 * t_nograph / k, "create_s": t_create,
           "multi_system_launches": batch.multi,
           "autotuned_systems": sum(int(v.info.autotuned) for v in batch.plans),
           "config": {"workload": "batched form: 64 cubic systems, N~U[5k,200k] at 0.08 A^-3, "
                                  "2 types 1:2, uniform, qmax 8, nq 400, partials, FP32+FP64acc, "
                                  "eps 1e-6, autotuned grids",
                      "fine_grids": sorted({int(v.info.nf[0]) for v in batch.plans})}}
    batch.close()
    return out


def ingest_leg(types, frames, stream, local_rank, nframes=4):
    """End to end from a LAMMPS text dump: the precision-form frames written
    as text (id type x y z, %.6f), then read by the library's multithreaded
    reader and streamed through sqn_accumulate_dump (the parse of frame f + 1
    overlaps the upload and transform of frame f).  Also times the reader
    alone on the same file."""
    import tempfile
    import torch
    from sqcalc_b200 import _lib

    nframes = min(nframes, len(frames))
    tmpdir = tempfile.mkdtemp(prefix="sqn_ingest_")
    path = os.path.join(tmpdir, "frames.dump")
    ids = np.arange(1, N_ATOMS + 1)
    with open(path, "w") as fh:
        for f in range(nframes):
            fh.write("ITEM: TIMESTEP\n%d\nITEM: NUMBER OF ATOMS\n%d\n"
                     "ITEM: BOX BOUNDS pp pp pp\n0 %r\n0 %r\n0 %r\nITEM: ATOMS id type x y z\n"
                     % (f, N_ATOMS, BOX, BOX, BOX))
            np.savetxt(fh, np.column_stack([ids, types, frames[f]]), fmt="%d %d %.6f %.6f %.6f")
    size = os.path.getsize(path)
    cores = os.cpu_count() or 1
    try:
        with _lib.DumpReader(path, nthreads=cores) as r:
            t0 = time.perf_counter()
            n = 0
            while r.next(capacity=N_ATOMS) is not None:
                n += 1
            t_read = time.perf_counter() - t0
        with _lib.Plan(np.eye(3).reshape(9) * BOX, np.zeros(3), types,
                       weight=_lib.WEIGHT_NEUTRON, amp_const=np.array(B_NEUTRON), qmin=0.0,
                       qmax=QMAX, nq=NQ, partials=True, precision=_lib.PREC_SINGLE, eps=EPS,
                       device=local_rank, stream=stream.cuda_stream) as p, \
                _lib.DumpReader(path, nthreads=cores) as r:
            p.accumulate_dump(r, max_frames=1)  # warm the plan and pin the buffers
            r.rewind()
            p.reset()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            done = p.accumulate_dump(r)
            t_all = time.perf_counter() - t0
    finally:
        os.remove(path)
        os.rmdir(tmpdir)
    return {"metric": "S(q) frames/s from a LAMMPS text dump (read + upload + transform)",
            "unit": "frames/s", "value": done / t_all, "frames": done,
            "reader_only_frames_per_s": n / t_read,
            "reader_gb_per_s": size / (nframes * 1e9) * n / t_read,
            "dump_bytes_per_frame": size // nframes, "threads": cores,
            "timing": "host wall clock around sqn_accumulate_dump (it syncs before returning)"}


GRAD_N, GRAD_BOX, GRAD_QMIN, GRAD_QMAX, GRAD_NQ = 100_000, 100.0, 0.5, 8.0, 375


def grad_leg(W, K, stream, dist, local_rank):
    """dS/dr evaluations/s on the differentiation form: cubic L = 100 A,
    N = 1e5, 2 types 1:2, loss sum_shells (S - S_target)^2 over q in [0.5, 8],
    S_target from a copy displaced by N(0, 0.2^2).  One evaluation = one
    sqn_sq_grad call with dL/dS: the weighted forward transform recomputed,
    three type-2 interpolations, S and the FP64 gradient returned.  Each plan's
    fine grid and kernel width are chosen by the autotuner, timing the gradient
    evaluation itself."""
    import torch
    from sqcalc_b200 import _lib

    rng = np.random.default_rng(SEED + 4)
    types = np.repeat([1, 2], [GRAD_N // 3, GRAD_N - GRAD_N // 3]).astype(np.int32)
    rng.shuffle(types)
    pos = rng.random((GRAD_N, 3)) * GRAD_BOX
    target_pos = pos + rng.normal(0.0, 0.2, pos.shape)
    d = torch.from_numpy(pos).to(f"cuda:{local_rank}")
    out = {"metric": "dS/dr evals/s", "unit": "evals/s",
           "config": {"workload": "differentiation form: cubic L=100 A, N=1e5, 2 types 1:2, "
                                  "uniform, loss over q in [0.5,8], S_target from a copy "
                                  "displaced by N(0,0.2^2)", "nq": GRAD_NQ}}
    k = min(K, 20)
    grads = {}
    for name, prec, eps in (("f32+f64acc", _lib.PREC_SINGLE, 1e-6), ("f64", _lib.PREC_DOUBLE, 1e-10)):
        with _lib.Plan(np.eye(3).reshape(9) * GRAD_BOX, np.zeros(3), types, qmin=GRAD_QMIN,
                       qmax=GRAD_QMAX, nq=GRAD_NQ, partials=False, precision=prec, eps=eps,
                       device=local_rank, stream=stream.cuda_stream, grad=True,
                       autotune=True) as p:
            S_t, _ = p.sq_grad(target_pos)
            S, _ = p.sq_grad(d)
            dLdS = 2.0 * (S - S_t)
            for _ in range(W):
                p.sq_grad(d, dLdS)
            torch.cuda.synchronize()
            l0 = p.launch_count()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            for _ in range(k):
                _, g = p.sq_grad(d, dLdS)
            ev1.record(stream)
            torch.cuda.synchronize()
            t = _max_over_ranks(ev0.elapsed_time(ev1) * 1e-3, dist, local_rank)
            grads[name] = g.cpu().numpy()
            out[name] = {"value": k / t, "ms_per_eval": 1e3 * t / k, "eps": eps, "steps": k,
                         "modes": list(p.modes), "fine_grid": list(p.info.nf),
                         "kernel_width": p.info.kernel_width, "autotuned": bool(p.info.autotuned),
                         "gpu_launches_per_eval": (p.launch_count() - l0) / k}
    # The headline is the FP64 adjoint: within 1e-6 relative of the FP64
    # direct-sum gradient (tests/test_gpu_grad.py measures ~1e-13).  The FP32
    # form is reported beside it with its measured deviation from FP64 on the
    # same positions and dL/dS (max |g32 - g64| / max |g64|).
    g64 = grads["f64"]
    out["f32+f64acc"]["max_rel_dev_vs_f64"] = float(
        np.max(np.abs(grads["f32+f64acc"] - g64)) / np.max(np.abs(g64)))
    out["value"] = out["f64"]["value"]
    out["value_form"] = "f64 (eps 1e-10), the form that meets 1e-6 of the FP64 direct-sum gradient"
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    from sqcalc_b200 import _lib, build

    build.build()
    torch.cuda.set_device(local_rank)
    dist = world > 1
    if dist:
        import torch.distributed as td
        td.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    K, W = args.steps, args.warmup
    # distinct frames, cycled through by the steps (each 24 MB, all of them far
    # larger than L2 together)
    NFR = min(K + W, 32)
    types, frames = make_frames(NFR, SEED + 7919 * rank)
    prec = _lib.PREC_SINGLE if args.precision == "single" else _lib.PREC_DOUBLE
    eps = EPS
    # A dedicated (non-default) stream: the plans run on it, so torch CUDA
    # events recorded on it bracket exactly the library's work.
    stream = torch.cuda.Stream(device=local_rank)
    torch.cuda.set_stream(stream)
    mk = lambda timing: _lib.Plan(np.eye(3).reshape(9) * BOX, np.zeros(3), types,  # noqa: E731
                                  weight=_lib.WEIGHT_NEUTRON, amp_const=np.array(B_NEUTRON),
                                  qmin=0.0, qmax=QMAX, nq=NQ, norm=_lib.NORM_MEAN,
                                  partials=True, precision=prec, eps=eps, device=local_rank,
                                  upsampfac=args.upsampfac, timing=timing,
                                  stream=stream.cuda_stream)

    # --- device-resident inputs: value --------------------------------------
    dev = torch.from_numpy(frames).to(f"cuda:{local_rank}")
    torch.cuda.synchronize()
    plan = mk(False)
    fbytes = N_ATOMS * 3 * 8
    base = dev.data_ptr()
    for f in range(W):
        plan.accumulate((base + (f % NFR) * fbytes, 1), where=_lib.DEVICE)
    plan.sync()
    if dist:
        td.barrier()
    torch.cuda.synchronize()
    launches0 = plan.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        clk.wait_first()
        t_wall = time.perf_counter()
        tm0 = time.monotonic()
        ev0.record(stream)
        for f in range(W, W + K):
            plan.accumulate((base + (f % NFR) * fbytes, 1), where=_lib.DEVICE)
        ev1.record(stream)
        torch.cuda.synchronize()
        clk.mark(tm0, time.monotonic())
        t_wall = time.perf_counter() - t_wall
    launches = plan.launch_count() - launches0
    info = plan.info
    elapsed = ev0.elapsed_time(ev1) * 1e-3
    if dist:
        t = torch.tensor([elapsed], dtype=torch.float64, device=f"cuda:{local_rank}")
        td.all_reduce(t, op=td.ReduceOp.MAX)
        elapsed = float(t.item())
    value = K * world / elapsed

    # --- per-stage device times (CUDA events inside the library) -------------
    tplan = mk(True)
    for f in range(W):
        tplan.accumulate((base + (f % NFR) * fbytes, 1), where=_lib.DEVICE)
    tplan.reset()
    for f in range(W, W + K):
        tplan.accumulate((base + (f % NFR) * fbytes, 1), where=_lib.DEVICE)
    st = tplan.stage_times()
    tplan.close()
    nfr = max(st["frames"], 1)
    stage_ms = {k: st[k] / nfr for k in ("sort_ms", "spread_ms", "fft_ms", "bin_ms")}

    # --- end to end through the C ABI with host buffers -------------------------
    pinned = torch.from_numpy(frames).pin_memory()
    pnum = torch.zeros(NQ, dtype=torch.float64).pin_memory()
    e2e_plan = mk(False)
    hbase = pinned.data_ptr()
    import ctypes
    L = _lib.load()
    for f in range(W):
        L.sqn_accumulate_frames(e2e_plan.handle, ctypes.c_void_p(hbase + (f % NFR) * fbytes), 1, _lib.HOST)
        e2e_plan.peek_num_async(pnum.data_ptr())
    e2e_plan.sync()
    if dist:
        td.barrier()
    torch.cuda.synchronize()
    ev0.record(stream)
    for f in range(W, W + K):
        rc = L.sqn_accumulate_frames(e2e_plan.handle, ctypes.c_void_p(hbase + (f % NFR) * fbytes), 1,
                                     _lib.HOST)
        _lib.check(rc, "sqn_accumulate_frames")
        e2e_plan.peek_num_async(pnum.data_ptr())
    e2e_plan.join()
    ev1.record(stream)
    torch.cuda.synchronize()
    e2e_t = ev0.elapsed_time(ev1) * 1e-3
    if dist:
        t = torch.tensor([e2e_t], dtype=torch.float64, device=f"cuda:{local_rank}")
        td.all_reduce(t, op=td.ReduceOp.MAX)
        e2e_t = float(t.item())
    e2e_value = K * world / e2e_t
    e2e_plan.close()

    # --- the plain FP64 path on the same frames, and max |dS| of FP32 ----------
    fp64 = precision_leg(types, dev, base, fbytes, W, K, stream, dist, world, local_rank)

    # --- the reference's own cuFINUFFT on this GPU (baseline) --------------------
    ref_gpu = None
    if world == 1 and not args.no_reference_gpu:
        ref_gpu = reference_gpu_baseline(types, dev, W, K, stream, local_rank)

    # --- the CPU-runnable FP64 configuration and the structured solid ----------
    small = solid = None
    if world == 1 and not args.no_configs:
        small = small_fp64_leg(W, K, stream, local_rank)
        solid = solid_leg(W, K, stream, local_rank)

    # --- dS/dr evaluations (differentiation form) -------------------------------
    grad = None if args.no_grad else grad_leg(W, K, stream, dist, local_rank)

    # --- ingest: from a LAMMPS text dump ------------------------------------------
    ingest = None if args.no_ingest else ingest_leg(types, frames, stream, local_rank)

    # --- batched form: many systems behind one CUDA graph -------------------------
    batched = None if args.no_batch else batched_leg(W, K, stream, dist, local_rank)

    # --- sharded frames: sum the FP64 accumulators once (one all-reduce) --------
    if dist:
        from sqcalc_b200.shard import reduce_plan
        reduce_plan(plan)
    plan.close()

    if rank == 0:
        # roofline of the dominant kernel of ours (spread or bin)
        peak, peak_kind = hbm_peak()
        ntr = info.ntransforms
        nf = list(info.nf)
        vol = nf[0] * nf[1] * nf[2]
        p = 4 if prec == _lib.PREC_SINGLE else 8
        c1 = nf[0] // 2 + 1
        spread_bytes = ntr * vol * p + N_ATOMS * (16 if p == 4 else 32)
        bin_bytes = ntr * (info.nmodes // 2) * 2 * p
        kern = "spread" if stage_ms["spread_ms"] >= stage_ms["bin_ms"] else "bin"
        kb = spread_bytes if kern == "spread" else bin_bytes
        kms = stage_ms["spread_ms"] if kern == "spread" else stage_ms["bin_ms"]
        achieved = kb / (kms * 1e-3) / 1e9
        frame_bytes = ntr * (3 * vol * p + (info.nmodes // 2) * 2 * p) + N_ATOMS * (24 + 1)
        # algorithmic bytes of each stage over its CUDA-event time
        m = list(info.modes)
        H1, M2, M3 = (m[0] - 1) // 2 + 1, m[1], m[2]
        if info.pruned_fft512:
            fft_bytes = ntr * (vol * p + 2 * nf[2] * nf[1] * H1 * 2 * p
                               + 2 * nf[2] * M2 * H1 * 2 * p + M3 * M2 * H1 * 2 * p)
        else:
            fft_bytes = ntr * (vol * p + vol // nf[0] * c1 * 2 * p)  # one-pass lower bound
        stage_roofline = {}
        for name, nbytes, ms in (("spread", spread_bytes, stage_ms["spread_ms"]),
                                 ("fft", fft_bytes, stage_ms["fft_ms"]),
                                 ("bin", bin_bytes, stage_ms["bin_ms"])):
            gbs = nbytes / (ms * 1e-3) / 1e9
            stage_roofline[name] = {"bytes": int(nbytes), "ms": ms, "gbs": gbs, "frac": gbs / peak}
        frame_ms = 1e3 * elapsed / K
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": 1e3 * elapsed / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64acc" if prec == _lib.PREC_SINGLE else "f64",
            "data": "synthetic (seeded uniform + Gaussian jitter)",
            "config": workload_config({
                "parallelism": "frames sharded over %d GPU(s)" % world,
                "upsampfac": info.upsampfac, "kernel_width": info.kernel_width,
                "fine_grid": nf, "nmodes_kept": info.nmodes, "ntransforms": ntr}),
            "roofline": {"bound": "hbm", "kernel": "k_spread" if kern == "spread" else "k_bin",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": dram_traffic("k_" + kern),
                         "algorithmic_bytes_per_launch": kb, "launch_ms": kms},
            "pipeline": {"bytes_per_frame": frame_bytes, "ms_per_frame": frame_ms,
                         "grid_cells_per_s": ntr * vol / (frame_ms * 1e-3),
                         "achieved_gbs": frame_bytes / (frame_ms * 1e-3) / 1e9,
                         "frac": frame_bytes / (frame_ms * 1e-3) / 1e9 / peak,
                         "stage_ms": stage_ms, "stage_roofline": stage_roofline,
                         "stage_roofline_note": "HBM roofline per stage (measured copy "
                                                "peak); fft = the pruned 512-point passes' "
                                                "reads and writes"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": fbytes,
                    "d2h_bytes_per_step": NQ * 8},
            "gpu_launches": launches,
            "gpu_launches_note": "own kernels per frame: prep, scan, scatter, spread, the "
                                 "three pruned 512-point FFT passes (512^3 grids; cuFFT "
                                 "kernels, not counted, otherwise) and bin",
            "fp64": fp64,
            "reference_gpu_baseline": ref_gpu,
            "plain_fp64_config": small,
            "solid_config": solid,
            "fp32_over_fp64": {
                "vs_own_fp64_eps1e-6": value / fp64["value"],
                "vs_own_fp64_sqcalc_eps1e-9": value / fp64["sqcalc_default_eps"]["value"],
                "vs_reference_cufinufft_fp64_eps1e-9": (
                    value / ref_gpu["cufinufft_f64"]["frames_per_s"]
                    if ref_gpu and "cufinufft_f64" in ref_gpu else None),
                "target": 10.0},
            "grad": grad,
            "batched": batched,
            "ingest": ingest,
            "clocks": clk.summary(),
            "wall_s": t_wall,
        }
        if world == 1 and not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline_sample()
        print(json.dumps(out), flush=True)
    if dist:
        td.barrier()
        td.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="single", choices=["single", "double"])
    ap.add_argument("--upsampfac", type=float, default=0.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-grad", action="store_true", help="skip the dS/dr leg")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the plain-FP64 (L=20, N=8000) and structured-solid legs")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's cuFINUFFT (oracle/_ref) on the GPU")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-systems leg")
    ap.add_argument("--no-ingest", action="store_true", help="skip the text-dump ingest leg")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="shrink the box by this factor at fixed density (profiling only)")
    args = ap.parse_args()
    if args.scale != 1.0:
        global N_ATOMS, BOX
        BOX = BOX * args.scale
        N_ATOMS = int(round(N_ATOMS * args.scale ** 3))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
