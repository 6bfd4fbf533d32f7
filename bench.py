#!/usr/bin/env python
"""Throughput benchmark of the emitter-wavefield direct sum on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the precision configuration of the direct sum): 50,000 emitters on
an fcc lattice (a = 0.36 nm) filling a 12 nm cube with 0.01 nm Gaussian
jitter, uniform phases, 8.0 keV, 1024 x 1024 detector with 50 um pixels at
0.2 m, 32 images with independent phase draws, near-field geometry, split
precision.  Inputs are synthetic (seeded Philox).  One step = one batched
forward of the 32 images (1.68e12 emitter-pixel pairs).

The JSON line carries the headline value (pairs/s with inputs resident in
HBM), the end-to-end figure through the public API (host emitters in, host
fields out), the forward+adjoint cost on the differentiation configuration,
the all-FP64 comparator, split-vs-FP64 error statistics, the MUFU roofline
and the CPU baseline (the oracle's C restatement on the host cores).

Multi-GPU (torchrun): images are independent, so every rank runs its own 32
images (weak scaling) with no data-path collective; timing is the max over
ranks.
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

E_EV = 8000.0
NDET = 1024
PIXEL = 50.0
DETZ = 2e5
N_EMIT = 50000
N_IMG = 32
SETTINGS = "nf split"
METRIC = "emitter-pixel pairs/s"
WORKLOAD = "fcc 50k emitters, 12 nm cube, 8 keV, 1024x1024 @ 50 um, 0.2 m, 32 images, near field, split precision"


def k_of(E):
    return 2 * np.pi / (1.24 / E)


def fcc_emitters(seed=1):
    g = np.random.Generator(np.random.Philox(seed))
    a = 3.6e-4
    m = int(np.ceil(0.012 / a))
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    cells = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), -1).reshape(-1, 1, 3)
    sites = ((cells + base[None]) * a).reshape(-1, 3)
    sites = sites[np.all(sites < 0.012, axis=1)] - 0.006
    pos = sites[g.choice(len(sites), N_EMIT, replace=False)] + g.normal(0, 1e-5, (N_EMIT, 3))
    return pos


def phases(seed, n_img=N_IMG):
    g = np.random.Generator(np.random.Philox(seed))
    return g.uniform(0, 2 * np.pi, (n_img, N_EMIT))


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def max_over_ranks(x, world):
    from idi_b200.simulation.shard import max_over_ranks as _max

    return _max(x) if world > 1 else x


def barrier(world):
    import torch

    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize()


# ---------------------------------------------------------------------------
# CPU baseline (the oracle's C restatement, all host cores)
# ---------------------------------------------------------------------------
def cpu_baseline(pos, ph, rows_target_s=12.0):
    import oracle

    k = k_of(E_EV)
    at = np.ascontiguousarray(np.concatenate([pos, ph[0][:, None]], 1))
    # calibrate on 2 detector rows, then size the sample to ~rows_target_s
    def run(rows):
        g = oracle.geometry([rows, NDET], PIXEL, DETZ, k, (0, 0), ((rows / 2 - NDET / 2) * PIXEL, 0.0))
        t0 = time.perf_counter()
        oracle.wavefield(g, oracle.NF, at)
        return time.perf_counter() - t0

    t_cal = run(2)
    rows = int(max(2, min(NDET, round(2 * rows_target_s / max(t_cal, 1e-3)))))
    dt = run(rows)
    pairs = rows * NDET * N_EMIT
    return {"value": pairs / dt, "unit": "pairs/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{rows} detector rows x {NDET} px x {N_EMIT} emitters of image 0 "
                      f"({pairs:.3g} pairs, {dt:.1f} s), FP64 near field, OpenMP over rows"}


def c2_oracle_windows(out, pos, ph, k, w=64, seed=9):
    """Split-precision intensities of the timed step (all images) against the
    FP64 CPU oracle on a w x w window of every image, at a seeded position per
    image.  The window's detector offset places its pixels exactly on the
    full detector's (integer multiples of the pixel size), so both compute
    the same points."""
    import oracle

    g = np.random.Generator(np.random.Philox(seed))
    I_s, I_o = [], []
    t0 = time.perf_counter()
    for b in range(out.shape[0]):
        ix0, iy0 = (int(v) for v in g.integers(0, NDET - w + 1, 2))
        og = oracle.geometry([w, w], PIXEL, DETZ, k, (0, 0),
                             ((ix0 - NDET // 2 + w // 2) * PIXEL, (iy0 - NDET // 2 + w // 2) * PIXEL))
        at = np.ascontiguousarray(np.concatenate([pos, ph[b][:, None]], 1))
        I_o.append(np.abs(oracle.wavefield(og, oracle.NF, at)) ** 2)
        E = out[b, ix0:ix0 + w, iy0:iy0 + w].cpu().numpy()
        I_s.append(np.abs(E) ** 2)
    dt = time.perf_counter() - t0
    st = error_stats(np.stack(I_s), np.stack(I_o))
    st.update({"windows": f"{out.shape[0]} images x {w}x{w} px at seeded positions", "oracle_s": dt,
               "compare": "split (the timed step's output) vs FP64 CPU oracle (reference rounding sequence)"})
    return st


def summarize_targets(line, t):
    """The target figures (C2 rate, SFU fraction, split/FP64 speed-up and error,
    end-to-end rate, forward+adjoint ratio, batched rate and balance, time
    path) in one compact object, last on the line."""
    def r4(x):
        return None if x is None else float(f"{x:.4g}")

    out = {"c2_pairs_per_s": r4(t["c2_pairs_per_s"]), "c2_sfu_frac": r4(t["c2_sfu_frac"])}
    fp64 = line.get("fp64", {}).get("value")
    if fp64:
        out["c2_split_over_fp64"] = r4(t["c2_pairs_per_s"] / fp64)
    acc = line.get("accuracy_c2_vs_cpu_oracle")
    if acc:
        out["c2_err_vs_cpu_oracle"] = {"max_rel_masked": r4(acc["max_rel_masked"]),
                                       "max_rel_to_mean": r4(acc["max_rel_to_mean"]), "pixels": acc["pixels"]}
    if "e2e" in line:
        out["e2e_pairs_per_s"] = r4(line["e2e"]["value"])
    fb = line.get("fwd_bwd")
    if fb:
        out["c4_fwd_bwd_over_fwd"] = r4(fb["ratio"])
    bt = line.get("batched_uneven")
    if bt:
        out["c3_pairs_per_s"] = r4(bt["pairs_per_s"])
        out["c3_imbalance"] = r4(bt["load_imbalance_max_over_mean_cta_busy"])
    tp = line.get("time_path")
    if tp:
        out["c5_pairs_per_s"] = r4(tp["pairs_per_s"])
        if "roofline" in tp:
            out["c5_frac"] = r4(tp["roofline"]["frac"])
    return out


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle

    pos = fcc_emitters()
    ph = phases(2, 1)
    k = k_of(E_EV)
    at = np.ascontiguousarray(np.concatenate([pos, ph[0][:, None]], 1))
    rows = 8
    g = oracle.geometry([rows, NDET], PIXEL, DETZ, k, (0, 0), ((rows / 2 - NDET / 2) * PIXEL, 0.0))
    for _ in range(args.warmup):
        oracle.wavefield(g, oracle.NF, at)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.wavefield(g, oracle.NF, at)
    dt = (time.perf_counter() - t0) / args.steps
    pairs = rows * NDET * N_EMIT
    v = pairs / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "pairs/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded Philox)", "config": {"workload": WORKLOAD},
        "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": f"per step: {rows} rows x {NDET} px x {N_EMIT} emitters of image 0, "
                                   "FP64 near field (the oracle's C restatement of idi/simulation/cpu.py)"},
        "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    gpu_point = reference_gpu_kernels(pos, ph[0], k)
    if gpu_point is not None:
        line["reference_gpu"] = gpu_point
    print(json.dumps(line), flush=True)
    return 0


def reference_gpu_kernels(pos, ph0, k):
    """The reference's own GPU kernels, wfkerneld (FP64) and wfkernelf (FP32,
    with the near-field distance in FP64) of idi/simulation/sim.cu, compiled
    from the reference tree for sm_100a into oracle/_ref and launched with the
    reference's 16x16 blocks: one image of the workload, near field, timed
    with CUDA events (best of 3 after a warm-up).  None where oracle/_ref was
    not built or no GPU is present."""
    import ctypes

    lib = os.path.join(ROOT, "oracle", "_ref", "libref_wf.so")
    try:
        import torch

        if not (os.path.exists(lib) and torch.cuda.is_available()):
            return None
        L = ctypes.CDLL(lib)
    except (ImportError, OSError):
        return None
    L.ref_wf_launch.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_float] * 5 + \
                               [ctypes.c_int] * 3 + [ctypes.c_void_p]
    L.ref_wf_launch.restype = ctypes.c_int
    at = np.ascontiguousarray(np.concatenate([pos, ph0[:, None]], 1))
    res = {"workload": f"1 image: {N_EMIT} emitters x {NDET}x{NDET}, near field (sim.cu -Dusenf -Dnodist)"}
    pairs = N_EMIT * NDET * NDET
    for label, single in (("wfkerneld_fp64", 0), ("wfkernelf_fp32", 1)):
        d_at = torch.from_numpy(at.astype(np.float32) if single else at).cuda()
        out = torch.empty((NDET, NDET), dtype=torch.complex64 if single else torch.complex128, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream

        def launch():
            st = L.ref_wf_launch(single, out.data_ptr(), d_at.data_ptr(), 0.0, 0.0, DETZ, PIXEL, k, NDET, NDET,
                                 N_EMIT, stream)
            if st != 0:
                raise RuntimeError(f"reference kernel launch failed ({st})")

        ms = timed_fn(torch)(launch, reps=3)
        res[label] = {"ms": ms, "pairs_per_s": pairs / (ms * 1e-3)}
    return res


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip e2e/fwd+bwd/fp64/accuracy legs")
    ap.add_argument("--case", default="full", choices=["full", "small"],
                    help="small: 8 images on a 512x512 detector (profiling-sized capture of the same kernel)")
    ap.add_argument("--no-tune", action="store_true", help="use the default kernel shape instead of autotuning")
    ap.add_argument("--config", default=None, help='kernel shape as JSON, e.g. {"threads":256,"pixels_per_thread":4}')
    ap.add_argument("--leg", default="main",
                    choices=["main", "fwd_bwd", "time", "batched", "detector", "emitters", "qcorr", "accuracy"],
                    help="run one secondary leg alone (for profiling) instead of the headline measurement")
    args = ap.parse_args()
    global N_IMG, NDET
    global WORKLOAD
    if args.case == "small":
        N_IMG, NDET = 8, 512
        WORKLOAD = WORKLOAD.replace("1024x1024", "512x512").replace("32 images", "8 images")
    if args.impl == "reference":
        return reference_arm(args)
    if args.leg != "main":
        return single_leg(args)
    if args.warmup < 3:
        args.warmup = 3

    import torch

    rank, world, local = dist_init()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    from idi_b200 import _native as nat
    from idi_b200.simulation import _core, cuda, simobj

    k = k_of(E_EV)
    pos = fcc_emitters()
    ph = phases(1000 + rank, N_IMG)
    atoms_h = np.concatenate([np.concatenate([pos, p[:, None]], 1) for p in ph])
    atoms = torch.from_numpy(np.ascontiguousarray(atoms_h)).to(dev)
    offsets = np.arange(N_IMG + 1, dtype=np.int64) * N_EMIT
    flags, precision, _ = _core.parse_settings(SETTINGS)
    geom = _core.make_geom(NDET, PIXEL, DETZ, k, flags=flags)
    out = torch.empty((N_IMG, NDET, NDET), dtype=torch.complex128, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    pairs_per_step = N_IMG * N_EMIT * NDET * NDET

    if args.config:
        cfg = json.loads(args.config)
    elif args.no_tune:
        cfg = None
    else:
        nt = min(2, N_IMG)
        cfg = _core.tune(atoms[: nt * N_EMIT], offsets[: nt + 1], geom, precision, nat.OUT_C128)

    def step():
        _core.forward(atoms, offsets, geom, precision, nat.OUT_C128, out=out, config=cfg)

    for _ in range(args.warmup):
        flush.fill_(1)
        step()
    barrier(world)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        barrier(world)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        for i in range(args.steps):
            flush.fill_(1)
            ev[i][0].record()
            step()
            ev[i][1].record()
        t1.record()
        barrier(world)
    total_ms = t0.elapsed_time(t1)
    kern_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = max_over_ranks(total_ms, world)
    _core.workspace_error(dev)
    ms_per_step = total_ms / args.steps
    value = pairs_per_step * world / (ms_per_step * 1e-3)
    kern_avg = sum(kern_ms) / len(kern_ms)

    # MUFU roofline: the split kernel issues one sin and one cos per pair
    mufu = _core.microbench("mufu_sincos", dev)
    achieved_mufu = 2.0 * pairs_per_step / (kern_avg * 1e-3)
    clocks = clk.summary()
    traffic = None
    try:  # DRAM bytes per launch from the committed ncu capture, scaled to this launch
        with open(os.path.join(ROOT, "profiles", "fwd_split_traffic.json")) as f:
            cap = json.load(f)
        traffic = (cap["dram_bytes_read"] + cap["dram_bytes_write"]) * (N_IMG * N_EMIT) / (
            cap["images"] * cap["emitters_per_image"])
    except (OSError, KeyError, ValueError):
        pass
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    nominal_mufu = sms * 16 * (clocks["sm_max_mhz"] or 1965.0) * 1e6

    line = {
        "metric": METRIC,
        "value": value,
        "unit": "pairs/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 phase / f32 sincos+sum",
        "data": "synthetic (seeded Philox)",
        "config": {"workload": WORKLOAD, "images": N_IMG, "emitters": N_EMIT, "detector": [NDET, NDET],
                   "settings": SETTINGS, "parallelism": f"images per rank, {world} rank(s)",
                   "l2": "flushed between steps (256 MiB write)", "kernel_shape": cfg},
        # per step: prep_split_kernel, the pixel-run kernel, and the per-pixel and exact near-field
        # kernels (both return at once on this workload)
        "gpu_launches": 4 * args.steps,
        "clocks": clocks,
        "roofline": {"bound": "sfu", "achieved": achieved_mufu / 1e9, "peak": mufu / 1e9, "unit": "Gop/s (MUFU)",
                     "frac": achieved_mufu / mufu, "frac_of_nominal": achieved_mufu / nominal_mufu,
                     "peak_source": "measured: in-repo MUFU sin/cos microbenchmark (idiwf_microbench kind 0)",
                     "ops_per_pair": 2, "kernel_ms": kern_avg, "traffic": traffic,
                     "traffic_unit": "bytes per launch (ncu capture of 8 images, scaled by emitter records)"},
    }
    targets = {"c2_pairs_per_s": value, "c2_sfu_frac": achieved_mufu / mufu}
    if not args.no_extras and rank == 0:
        line.update(extras(args, torch, dev, _core, nat, cuda, simobj, pos, ph, k, geom, atoms, offsets, cfg))
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        try:
            line["cpu_baseline"] = cpu_baseline(pos, ph)
            # C2's split error against the FP64 CPU oracle: windows of every image
            line["accuracy_c2_vs_cpu_oracle"] = c2_oracle_windows(out, pos, ph, k)
        except Exception as e:  # the oracle library may be missing on a stripped box
            line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
    if rank == 0:
        line["targets"] = summarize_targets(line, targets)
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def extras(args, torch, dev, _core, nat, cuda, simobj, pos, ph, k, geom, atoms, offsets, cfg):
    res = {}
    # --- end to end through the public API: host emitters in, host fields out
    obj = simobj.fixed(E_EV, pos, phases=ph)
    cuda.simulate(2, obj, NDET, PIXEL, DETZ, k, settings=SETTINGS, verbose=False)  # warm
    n_e2e = min(args.steps, 2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        cuda.simulate(N_IMG, obj, NDET, PIXEL, DETZ, k, settings=SETTINGS, verbose=False)
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / n_e2e
    pairs = N_IMG * N_EMIT * NDET * NDET
    res["e2e"] = {"value": pairs / dt, "unit": "pairs/s", "h2d_bytes_per_step": N_IMG * N_EMIT * 32,
                  "d2h_bytes_per_step": N_IMG * NDET * NDET * 16,
                  "call": "idi_b200.simulation.cuda.simulate(32, simobject, 1024, 50, 2e5, k, settings='nf split')"}

    # --- all-FP64 comparator on 2 images of the same batch
    timed = timed_fn(torch)

    at2 = atoms[: 2 * N_EMIT]
    off2 = offsets[:3]
    ms64 = timed(lambda: _core.forward(at2, off2, geom, nat.DOUBLE, nat.OUT_C128), reps=2)
    v64 = 2 * N_EMIT * NDET * NDET / (ms64 * 1e-3)
    res["fp64"] = {"value": v64, "unit": "pairs/s", "images": 2, "ms": ms64}

    # --- accuracy on 2 full images: split and the reference-sequence FP64
    #     kernel, both against the cancellation-free FP64 kernel ("truth")
    Es = _core.forward(at2, off2, geom, nat.SPLIT, nat.OUT_C128, config=cfg)
    Ed = _core.forward(at2, off2, geom, nat.DOUBLE, nat.OUT_C128)
    geom_acc = _core.make_geom(NDET, PIXEL, DETZ, k, flags=nat.NF | nat.ACCURATE)
    Ea = _core.forward(at2, off2, geom_acc, nat.DOUBLE, nat.OUT_C128)
    Is = (Es.real ** 2 + Es.imag ** 2).cpu().numpy()
    Id = (Ed.real ** 2 + Ed.imag ** 2).cpu().numpy()
    Ia = (Ea.real ** 2 + Ea.imag ** 2).cpu().numpy()

    def stats(I, Iref, name):
        mean = Iref.mean()
        d = np.abs(I - Iref)
        mask = Iref >= 1e-3 * mean
        rel = d[mask] / Iref[mask]
        hist, edges = np.histogram(np.log10(np.maximum(rel, 1e-12)), bins=np.arange(-12, 0.5, 1.0))
        return {"compare": name, "pixels": int(Iref.size), "max_rel_masked": float(rel.max()),
                "max_rel_to_mean": float(d.max() / mean), "p50": float(np.percentile(rel, 50)),
                "p99": float(np.percentile(rel, 99)), "p9999": float(np.percentile(rel, 99.99)),
                "mask": "I_ref >= 1e-3 mean",
                "log10_rel_hist": {f"{int(e)}": int(h) for e, h in zip(edges[:-1], hist)}}

    res["accuracy_split_vs_fp64"] = stats(Is, Id, "split vs FP64 (reference rounding sequence)")
    res["accuracy_vs_truth"] = {"split": stats(Is, Ia, "split vs cancellation-free FP64"),
                                "fp64_reference_sequence": stats(Id, Ia, "FP64 reference sequence vs cancellation-free FP64")}
    del Es, Ed, Ea

    res["detector"] = detector_leg(torch, dev, _core, nat, args, cuda=cuda, simobj=simobj, pos=pos, ph=ph, k=k)
    res["emitters"] = emitters_leg(torch, dev, _core, nat, args)
    res["qcorr"] = qcorr_leg(torch, dev, args)
    res["accuracy_per_config"] = accuracy_leg(torch, dev, _core, nat)
    res["fwd_bwd"] = fwd_bwd_leg(torch, dev, _core, nat, timed)
    res["batched_uneven"] = batched_leg(torch, dev, _core, nat)
    res["time_path"] = time_leg(torch, dev, _core, nat, args)
    return res


def timed_fn(torch):
    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        best = 1e30
        for _ in range(reps):
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            best = min(best, a.elapsed_time(b))
        return best
    return timed


def fwd_bwd_leg(torch, dev, _core, nat, timed):
    """Forward + adjoint on the differentiation configuration: 10,000 emitters
    in a 15 nm sphere, 512x512 @ 75 um, 0.1 m, 6.4 keV, near field; target =
    intensities after a 0.05 nm Gaussian displacement; L = sum (I - T)^2."""
    g = np.random.Generator(np.random.Philox(7))
    n4 = 10000
    t = g.uniform(-1, 1, n4)
    p = g.uniform(0, 2 * np.pi, n4)
    u = 0.015 * g.uniform(0, 1, n4) ** (1 / 3)
    s = np.sqrt(1 - t ** 2)
    pos4 = np.stack([u * t, u * s * np.sin(p), u * s * np.cos(p)], -1)
    ph4 = g.uniform(0, 2 * np.pi, n4)
    k4 = k_of(6400.0)
    geom4 = _core.make_geom(512, 75.0, 1e5, k4, flags=nat.NF)
    a4 = torch.from_numpy(np.concatenate([pos4, ph4[:, None]], 1)).to(dev)
    T4 = _core.forward(torch.from_numpy(np.concatenate([pos4 + g.normal(0, 5e-5, pos4.shape), ph4[:, None]], 1)).to(dev),
                       [0, n4], geom4, nat.SPLIT, nat.OUT_I64)
    off4 = [0, n4]

    def fwd():
        return _core.forward(a4, off4, geom4, nat.SPLIT, nat.OUT_C128)

    def fwd_bwd():
        E = fwd()
        I = E.real ** 2 + E.imag ** 2
        return _core.backward(a4, off4, geom4, E, (2 * (I - T4)).contiguous())

    ms_f = timed(fwd, reps=5)
    ms_fb = timed(fwd_bwd, reps=5)
    pairs4 = n4 * 512 * 512
    return {"workload": "10k emitters, 15 nm sphere, 512x512 @ 75 um, 0.1 m, 6.4 keV, near field",
            "fwd_ms": ms_f, "fwd_bwd_ms": ms_fb, "ratio": ms_fb / ms_f,
            "fwd_pairs_per_s": pairs4 / (ms_f * 1e-3), "fwd_bwd_pairs_per_s": pairs4 / (ms_fb * 1e-3)}


def single_leg(args):
    import torch

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    from idi_b200 import _native as nat
    from idi_b200.simulation import _core

    if args.leg == "fwd_bwd":
        out = fwd_bwd_leg(torch, dev, _core, nat, timed_fn(torch))
    elif args.leg == "time":
        out = time_leg(torch, dev, _core, nat, args)
    elif args.leg == "detector":
        out = detector_leg(torch, dev, _core, nat, args)
    elif args.leg == "emitters":
        out = emitters_leg(torch, dev, _core, nat, args)
    elif args.leg == "qcorr":
        out = qcorr_leg(torch, dev, args)
    elif args.leg == "accuracy":
        out = accuracy_leg(torch, dev, _core, nat)
    else:
        out = batched_leg(torch, dev, _core, nat)
    print(json.dumps({"leg": args.leg, **out}), flush=True)
    return 0


def sphere_points(g, n, r):
    t = g.uniform(-1, 1, n)
    p = g.uniform(0, 2 * np.pi, n)
    u = r * g.uniform(0, 1, n) ** (1 / 3)
    s = np.sqrt(1 - t ** 2)
    return np.stack([u * t, u * s * np.sin(p), u * s * np.cos(p)], -1)


def batched_leg(torch, dev, _core, nat):
    """256 images, emitter counts log-uniform in [1e3, 1e5], sphere radii
    uniform in [5, 25] nm, amplitudes uniform in [0.5, 1.5] (float32),
    512x512 @ 75 um, 0.1 m, 6.4 keV, near field, split precision: one
    persistent launch per batch, captured in a CUDA graph, shape autotuned."""
    from idi_b200.simulation.batch import BatchPlan

    g = np.random.Generator(np.random.Philox(33))
    counts = np.floor(np.exp(g.uniform(np.log(1e3), np.log(1e5), 256))).astype(np.int64)
    radii = g.uniform(0.005, 0.025, 256)
    at = np.concatenate([np.concatenate([sphere_points(g, int(c), r), g.uniform(0, 2 * np.pi, (int(c), 1))], 1)
                         for c, r in zip(counts, radii)])
    amp = g.uniform(0.5, 1.5, at.shape[0]).astype(np.float32)
    geom = _core.make_geom(512, 75.0, 1e5, k_of(6400.0), flags=nat.NF)
    plan = BatchPlan(counts, geom, nat.SPLIT, nat.OUT_I64, amplitudes="float32", device=dev)
    d_at = torch.from_numpy(at).to(dev)
    d_amp = torch.from_numpy(amp).to(dev)
    plan.run(d_at, d_amp)  # autotune + capture
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 2
    a.record()
    for _ in range(reps):
        plan.run()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / reps
    plan.check()
    busy = plan.cta_times().astype(np.float64)
    pairs = int(counts.sum()) * 512 * 512
    out = {"workload": "256 images, N log-uniform [1e3, 1e5], r in [5, 25] nm, a in [0.5, 1.5] f32, "
                       "512x512 @ 75 um, 0.1 m, 6.4 keV, near field, split, CUDA graph",
           "emitters": int(counts.sum()), "pairs_per_step": pairs, "ms": ms, "pairs_per_s": pairs / (ms * 1e-3),
           "kernel_shape": plan.config,
           "load_imbalance_max_over_mean_cta_busy": float(busy.max() / busy.mean()) if busy.size else None,
           "ctas": int(busy.size)}
    plan.close()
    return out


def time_leg(torch, dev, _core, nat, args):
    """20,000 emitters in a 10 nm sphere, emission times Gaussian (5 fs FWHM),
    tau = 2 fs, c = 0.3 um/fs, 256x256 @ 75 um, 0.1 m, 6.4 keV, 4 images."""
    import oracle

    g = np.random.Generator(np.random.Philox(44))
    n, nimg = 20000, 4
    geom = _core.make_geom(256, 75.0, 1e5, k_of(6400.0))
    pos = sphere_points(g, n, 0.01)
    imgs = []
    for _ in range(nimg):
        at = np.concatenate([pos, g.uniform(0, 2 * np.pi, (n, 1))], 1)
        t = g.normal(0, 5.0 / 2.35, n)
        imgs.append((torch.from_numpy(at).to(dev), torch.from_numpy(t).to(dev), at, t))
    _core.time_forward(imgs[0][0], imgs[0][1], geom, 0.3, 2.0)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for d_at, d_t, _, _ in imgs:
        _core.time_forward(d_at, d_t, geom, 0.3, 2.0)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    pairs = nimg * n * 256 * 256
    out = {"workload": "20k emitters, 10 nm sphere, 5 fs FWHM emission, tau 2 fs, 256x256 @ 75 um, 0.1 m, 4 images",
           "ms": ms, "pairs_per_s": pairs / (ms * 1e-3)}
    # issue roofline: thread instructions per pair (ncu count of the same kernel,
    # committed with its summary) against 4 warp instructions per clock per SM
    try:
        with open(os.path.join(ROOT, "profiles", "time_kernel_ff_20k_256.json")) as f:
            ipp = float(json.load(f)["thread_instructions_per_pair"])
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
                mhz, src = float(json.load(f)["sm_max_mhz"]), "MEASURED_PEAKS.json sm_max_mhz"
        except (OSError, KeyError, ValueError):
            mhz, src = 1965.0, "clocks.max.sm of the B200"
        peak = 4 * 32 * sms * mhz * 1e6
        achieved = out["pairs_per_s"] * ipp
        out["roofline"] = {"bound": "issue", "achieved": achieved / 1e9, "peak": peak / 1e9,
                           "unit": "G thread-instructions/s", "frac": achieved / peak, "instructions_per_pair": ipp,
                           "peak_source": f"4 warp instructions per clock per SM at {mhz:g} MHz ({src})",
                           "instructions_source": "ncu instruction count, profiles/time_kernel_ff_20k_256.md"}
    except (OSError, KeyError, ValueError):
        pass
    # above the on-chip table: 200,000 emitters, 64x64 detector, one image
    nl = 200000
    posl = sphere_points(g, nl, 0.01)
    atl = torch.from_numpy(np.concatenate([posl, g.uniform(0, 2 * np.pi, (nl, 1))], 1)).to(dev)
    tl = torch.from_numpy(g.normal(0, 5.0 / 2.35, nl)).to(dev)
    geoml = _core.make_geom(64, 75.0, 1e5, k_of(6400.0))
    msl = timed_fn(torch)(lambda: _core.time_forward(atl, tl, geoml, 0.3, 2.0), reps=2)
    out["large_n"] = {"workload": "200k emitters, 64x64, one image (workspace-resident sort)", "ms": msl,
                      "pairs_per_s": nl * 64 * 64 / (msl * 1e-3)}
    if not args.no_cpu_baseline:
        # CPU: the oracle's C restatement of time.py on a row-block sample of image 0
        rows = 2
        og = oracle.geometry([rows, 256], 75.0, 1e5, k_of(6400.0))
        t0 = time.perf_counter()
        oracle.time_image(og, 0, imgs[0][2], imgs[0][3], 0.3, 2.0)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": rows * 256 * n / dt, "unit": "pairs/s", "cores": os.cpu_count(),
                               "kind": "port", "sample": f"{rows} rows x 256 px x {n} emitters of image 0"}
    return out


def hbm_peak():
    """Measured HBM copy bandwidth (GB/s) and where it came from."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json copy bandwidth)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback (earlier measurement on this GPU type)"


def detector_leg(torch, dev, _core, nat, args, cuda=None, simobj=None, pos=None, ph=None, k=None):
    """Detector stage at the headline output size: 32 images x 1024 x 1024
    float64 intensities (268 MB, larger than L2), exponentially distributed
    like speckle.  Poisson photons with 1e5 and 1e9 expected photons per image
    (rates ~0.1: inversion; ~1000: PTRS) into uint32 counts; charge sharing
    (s = 0.5 px, w = 1, generated draws) of the 1e5-photon counts into float64.
    HBM roofline: photons move 20 B per pixel (two reads of the intensity and
    the count write), charge sharing 12 B (count read, float64 write)."""
    nimg, nd = N_IMG, NDET
    npix = nimg * nd * nd
    gen = torch.Generator(device=dev)
    gen.manual_seed(5)
    I = -torch.log1p(-torch.rand((nimg, nd, nd), dtype=torch.float64, device=dev, generator=gen))
    cnt = torch.empty((nimg, nd, nd), dtype=torch.uint32, device=dev)
    shared = torch.empty((nimg, nd, nd), dtype=torch.float64, device=dev)
    peak, peak_src = hbm_peak()
    timed = timed_fn(torch)
    out = {"workload": f"{nimg} images x {nd}x{nd} float64 intensities (exponential), uint32 counts",
           "hbm_peak_gbs": peak, "peak_source": peak_src}
    for label, nph in (("photons_1e5", 1e5), ("photons_1e9", 1e9)):
        ms = timed(lambda: _core.photons(I, nph, (1, 2), 0, dtype=torch.uint32, out=cnt), reps=5)
        gbs = 20.0 * npix / (ms * 1e-3) / 1e9
        out[label] = {"ms": ms, "pixels_per_s": npix / (ms * 1e-3), "achieved_gbs": gbs, "frac": gbs / peak,
                      "bytes_per_pixel": 20, "launches": 2}
    _core.workspace_error(dev, "photons")
    _core.photons(I, 1e5, (1, 2), 0, dtype=torch.uint32, out=cnt)
    photons_per_image = float(cnt.to(torch.float64).sum().item()) / nimg
    ms = timed(lambda: _core.chargesharing(cnt, 0.5, 0.0, (3, 4), 0, out=shared), reps=5)
    gbs = 12.0 * npix / (ms * 1e-3) / 1e9
    out["chargesharing_s0.5"] = {"ms": ms, "pixels_per_s": npix / (ms * 1e-3), "achieved_gbs": gbs,
                                 "frac": gbs / peak, "bytes_per_pixel": 12, "photons_per_image": photons_per_image}
    _core.workspace_error(dev, "charge")
    del I, shared
    if cuda is not None:
        # end to end through the public API: host emitters in, host uint32 counts out
        obj = simobj.fixed(E_EV, pos, phases=ph)
        cuda.simulate_photons(2, obj, NDET, PIXEL, DETZ, 1e5, k, settings=SETTINGS, verbose=False, rng=1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cuda.simulate_photons(N_IMG, obj, NDET, PIXEL, DETZ, 1e5, k, settings=SETTINGS, verbose=False, rng=1)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        out["e2e_simulate_photons"] = {
            "value": N_IMG * N_EMIT * NDET * NDET / dt, "unit": "pairs/s", "s": dt,
            "h2d_bytes_per_step": N_IMG * N_EMIT * 32, "d2h_bytes_per_step": N_IMG * NDET * NDET * 4,
            "call": "simulate_photons(32, simobject, 1024, 50, 2e5, 1e5, k, settings='nf split')"}
    if not args.no_cpu_baseline:
        # the reference's randomphotons on the host is numpy's Generator.poisson
        # of p * (N / sum p) (common.py:17): timed on 2 images of the same size
        h = np.random.default_rng(5).exponential(1.0, (2, nd, nd))
        t0 = time.perf_counter()
        np.random.default_rng(1).poisson(h * (1e5 / h.sum(axis=(-2, -1), keepdims=True)))
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": h.size / dt, "unit": "pixels/s", "cores": 1, "kind": "port",
                               "sample": f"numpy Generator.poisson of 2 x {nd}x{nd} rates ~0.1 (common.py:17)"}
    return out


def emitters_leg(torch, dev, _core, nat, args):
    """Emitter sources drawn on the device.  Crystal: the fcc lattice of the
    headline workload (a = 0.36 nm, 34^3 cells = 157,216 sites filling 12 nm),
    50,000 sites per image without replacement, random phases, 32 images,
    with and without a random orientation per image.  Sphere: 2,000 emitters
    in 10 nm, 8 images (the small CPU-runnable configuration)."""
    import warnings

    from idi_b200.simulation import simobj

    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        c = simobj.fcc(E_EV, N_EMIT, 3.6e-4, repeats=[34, 34, 34], seed=1)
    sites = torch.from_numpy(c._allpos.astype(np.float64)).to(dev)
    timed = timed_fn(torch)
    out = {"workload": "fcc 157,216 sites -> 50,000 per image x 32 images; sphere 2,000 x 8 images"}
    for label, orient in (("crystal_fixed", nat.ORIENT_FIXED), ("crystal_random_orientation", nat.ORIENT_RANDOM)):
        desc = _core.emitters_desc(nat.EMIT_SITES, sites=sites, orientation=orient)
        buf = torch.empty((N_IMG * N_EMIT, 4), dtype=torch.float64, device=dev)
        ms = timed(lambda: _core.emitters(desc, N_IMG, N_EMIT, (1, 2), 0, 0, dev, out=buf), reps=5)
        out[label] = {"ms": ms, "emitters_per_s": N_IMG * N_EMIT / (ms * 1e-3),
                      "sites_per_s": N_IMG * sites.shape[0] / (ms * 1e-3), "launches": 3}
    desc = _core.emitters_desc(nat.EMIT_SPHERE, r=0.01)
    ms = timed(lambda: _core.emitters(desc, 8, 2000, (1, 2), 0, 0, dev), reps=5)
    out["sphere"] = {"ms": ms, "emitters_per_s": 8 * 2000 / (ms * 1e-3), "launches": 1}
    # end to end on the small configuration: simulate() of 64 images of a
    # 2,000-emitter sphere (10 nm), 256x256 @ 75 um, 0.1 m, 6.4 keV, split,
    # with the emitters drawn on the host (get2) and on the device
    from idi_b200.simulation import cuda as sim

    e2e = {}
    for label, ondevice in (("host_draws", False), ("device_draws", True)):
        obj = simobj.sphere(6400.0, 2000, 0.01, rng=np.random.default_rng(1), seed=1)
        obj.ondevice = ondevice
        sim.simulate(8, obj, 256, 75.0, 1e5, settings="split", verbose=False)  # warm
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim.simulate(64, obj, 256, 75.0, 1e5, settings="split", verbose=False)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        e2e[label] = {"s": dt, "images_per_s": 64 / dt, "pairs_per_s": 64 * 2000 * 256 * 256 / dt}
    out["e2e_small_config"] = e2e
    if not args.no_cpu_baseline:
        # the reference's host draw per image (simobj.py:446-487 and 50-60):
        # numpy choice without replacement of 50,000 of the 157,216 sites
        # and uniform phases, timed on 4 images
        rng = np.random.default_rng(1)
        allpos = c._allpos
        t0 = time.perf_counter()
        for _ in range(4):
            idx = rng.choice(len(allpos), N_EMIT, replace=False)
            np.concatenate([allpos[idx], rng.uniform(0, 2 * np.pi, (N_EMIT, 1))], 1)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": 4 * N_EMIT / dt, "unit": "emitters/s", "cores": 1, "kind": "port",
                               "sample": "numpy choice(157216, 50000, replace=False) + phases, 4 images"}
    return out


def error_stats(I, I_ref, floor=1e-3):
    """Per-pixel intensity error of I against I_ref: max |dI|/I_ref over pixels
    with I_ref >= floor * mean, max |dI| / mean over all, percentiles."""
    mean = float(I_ref.mean())
    d = np.abs(I - I_ref)
    mask = I_ref >= floor * mean
    rel = d[mask] / I_ref[mask]
    return {"pixels": int(I_ref.size), "max_rel_masked": float(rel.max()), "max_rel_to_mean": float(d.max() / mean),
            "p50": float(np.percentile(rel, 50)), "p99": float(np.percentile(rel, 99)),
            "mask": f"I_ref >= {floor:g} mean"}


def accuracy_leg(torch, dev, _core, nat):
    """Split-precision intensity error against the FP64 kernel for every
    direct-sum configuration (the FP64 kernel reproduces the reference's FP64
    CPU kernel to the last bits of sin/cos; the tests pin it to the reference's
    outputs).  C1: 2,000 emitters in a 10 nm sphere, 256^2 @ 75 um, 0.1 m,
    6.4 keV, 8 images (near and far field).  C3: 8 images of the uneven batch
    (the largest and smallest emitter counts among them), amplitudes in
    [0.5, 1.5] float32, 512^2.  C4: 10,000 emitters in 15 nm, 512^2, near field.
    (C2 is the accuracy_* entries of the headline record; the time path, C5,
    is checked against the oracle in the tests: 1e-10, bit-exact order.)"""
    out = {}

    def compare(atoms, offsets, geom_flags, ndet, ps, dz, k, amps=None):
        at = torch.from_numpy(np.ascontiguousarray(atoms)).to(dev)
        am = None if amps is None else torch.from_numpy(np.ascontiguousarray(amps)).to(dev)
        g = _core.make_geom(ndet, ps, dz, k, flags=geom_flags)
        Is = _core.forward(at, offsets, g, nat.SPLIT, nat.OUT_I64, amplitudes=am).cpu().numpy()
        Id = _core.forward(at, offsets, g, nat.DOUBLE, nat.OUT_I64, amplitudes=am).cpu().numpy()
        return error_stats(Is, Id)

    g = np.random.Generator(np.random.Philox(101))
    pos = sphere_points(g, 2000, 0.01)
    at1 = np.concatenate([np.concatenate([pos, g.uniform(0, 2 * np.pi, (2000, 1))], 1) for _ in range(8)])
    off1 = np.arange(9) * 2000
    k64 = k_of(6400.0)
    out["C1_far_field"] = compare(at1, off1, 0, 256, 75.0, 1e5, k64)
    out["C1_near_field"] = compare(at1, off1, nat.NF, 256, 75.0, 1e5, k64)
    g = np.random.Generator(np.random.Philox(33))
    counts = np.floor(np.exp(g.uniform(np.log(1e3), np.log(1e5), 256))).astype(np.int64)
    pick = np.argsort(counts)[np.linspace(0, 255, 8).astype(int)]
    rows, amps = [], []
    for i in pick:
        c = int(counts[i])
        rows.append(np.concatenate([sphere_points(g, c, g.uniform(0.005, 0.025)), g.uniform(0, 2 * np.pi, (c, 1))], 1))
        amps.append(g.uniform(0.5, 1.5, c).astype(np.float32))
    off3 = np.concatenate([[0], np.cumsum([r.shape[0] for r in rows])])
    out["C3_subset"] = compare(np.concatenate(rows), off3, nat.NF, 512, 75.0, 1e5, k64, np.concatenate(amps))
    out["C3_subset"]["emitters"] = [int(counts[i]) for i in pick]
    g = np.random.Generator(np.random.Philox(7))
    pos4 = sphere_points(g, 10000, 0.015)
    at4 = np.concatenate([pos4, g.uniform(0, 2 * np.pi, (10000, 1))], 1)
    out["C4"] = compare(at4, [0, 10000], nat.NF, 512, 75.0, 1e5, k64)
    return out


def qcorr_pairs(nr, nc, row_offsets, col_offsets):
    """Pixel pairs the correlators visit: rows r, r + dr (dr in
    [0, row_offsets)), columns c, c + dc (|dc| <= col_offsets)."""
    rows = sum(max(0, nr - dr) for dr in range(row_offsets))
    cols = sum(max(0, nc - abs(dc)) for dc in range(-col_offsets, col_offsets + 1))
    return rows * cols


def qcorr_leg(torch, dev, args):
    """Correlation of speckle images (exponential intensities): direct radial,
    512 x 512 at z = 2000 px, 256 bins, 4 images; direct 3d, 512 x 512 at
    z = 2000 px, maxq 128, 2 images (one unit = one pixel pair); FFT
    autocorrelation of 8 x 1024 x 1024."""
    from idi_b200.reconstruction import _geometry, cucor, cucorrad

    g = np.random.default_rng(3)
    out = {"workload": "radial: 4 x 512x512, z 2000 px, 256 bins; 3d: 2 x 512x512, z 2000 px, maxq 128"}
    imgs = torch.from_numpy(g.exponential(1.0, (4, 512, 512)).astype(np.float32)).to(dev)
    timed = timed_fn(torch)
    with cucorrad.corrfunction((512, 512), 2000.0, 256, return_gpu=True) as f:
        ms = timed(lambda: f(imgs), reps=3)
    pairs = 4 * qcorr_pairs(512, 512, 256, 256)
    out["radial"] = {"ms": ms, "pairs_per_s": pairs / (ms * 1e-3), "pairs": pairs}
    with cucor.corrfunction((512, 512), 2000.0, 128) as f3:
        ms3 = timed(lambda: f3(imgs[:2]), reps=2)
    pairs3 = 2 * qcorr_pairs(512, 512, 128, 127)
    out["3d"] = {"ms": ms3, "pairs_per_s": pairs3 / (ms3 * 1e-3), "pairs": pairs3,
                 "note": "includes the device-to-host copy of the float64 volume, as the reference's corr()"}
    from idi_b200.reconstruction import cusimple

    stack = torch.from_numpy(g.exponential(1.0, (8, 1024, 1024))).to(dev)
    msf = timed(lambda: cusimple.corr(stack, returngpu=True), reps=3)
    # the same autocorrelation through cuFFT's transforms and this library's
    # power / crop kernels (the path other shapes take)
    msc = timed(lambda: cusimple._crop(cusimple._autocorr(stack, 2, [2048, 2048]), 2, [1024, 1024]), reps=3)
    out["fft_corr"] = {"ms": msf, "images_per_s": 8 / (msf * 1e-3), "cufft_path_ms": msc,
                       "workload": "cusimple.corr of 8 x 1024x1024 float64 (2048^2 transforms), on the device; "
                                   "hand-written FFTs (power-of-two shape)"}
    # a general shape: fastlen(2000) = 2000 = 5^3 2^4, mixed-radix passes
    stack_g = torch.from_numpy(g.exponential(1.0, (8, 1000, 1000))).to(dev)
    msg = timed(lambda: cusimple.corr(stack_g, returngpu=True), reps=3)
    msgc = timed(lambda: cusimple._crop(cusimple._autocorr(stack_g, 2, [2000, 2000]), 2, [1000, 1000]), reps=3)
    out["fft_corr_general"] = {"ms": msg, "images_per_s": 8 / (msg * 1e-3), "cufft_path_ms": msgc,
                               "workload": "cusimple.corr of 8 x 1000x1000 float64 (2000^2 transforms, radices "
                                           "5, 8, 2), on the device; hand-written FFTs"}
    if not args.no_cpu_baseline:
        import oracle

        # the oracle's restatement of the reference kernel (one thread) on the
        # first 2 reference rows of image 0
        sub = imgs[0].cpu().numpy()
        q = _geometry.q_rows((512, 512), 2000.0)
        rows = 2
        # pairs whose reference row is 0 or 1 need target rows up to 1 + 255
        t0 = time.perf_counter()
        oracle.qcorr_radial(q[: (rows + 255) * 512], sub[: rows + 255], 256)
        dt = time.perf_counter() - t0
        sample = qcorr_pairs(rows + 255, 512, 256, 256)
        out["cpu_baseline"] = {"value": sample / dt, "unit": "pairs/s", "cores": 1, "kind": "port",
                               "sample": f"radial restatement on a {rows + 255} x 512 strip of image 0"}
    return out


if __name__ == "__main__":
    sys.exit(main())
