#!/usr/bin/env python
"""Batched STEM ADF multislice throughput on B200 (probe·slices/s).

Workload (one GPU): cubic perovskite supercell (a = 3.905 Å, Sr/Ti/O) tiled 10x10x20 (10,000 atoms),
512x512 grid, 300 kV probe with 24 mrad convergence, Cs = 1 um, C1 = 0, 64x64 probe positions on a
0.2 Å raster, 40 slices of 1.9525 Å, ADF detector 70-200 mrad, frozen phonons with isotropic Gaussian
displacements u_rms = 0.08 Å (seeded). The complex64 engine (FP64 phase arguments and accumulation).

A step is one frozen-phonon configuration: bin the atoms, build and band-limit the 40 transmission
functions, generate the 4096 probes and propagate them through all 40 slices with the fused FFT passes,
and accumulate the ADF image (FP64, Kahan). The default K = 10 steps is the full 10-configuration job.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU (torchrun, one rank per GPU): every rank runs K configurations of its own (weak scaling); the
averaged images are combined with one NCCL reduction at the end (the reference merges per-device
results in SimulationManager::updateImages).

--impl reference times the CPU restatement of the reference's double-precision path (the reference's
OpenCL build cannot be compiled or run here) on the host cores, on a bounded sample of the same
workload per step, reported in the same unit.
"""
import argparse
import ctypes as C
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

METRIC = "STEM probe·slices/s at 512² FP32 vs plain FP64 GPU; adjoint/forward time ratio"
UNIT = "probe·slices/s"
WORKLOAD = "stem_adf_perovskite_10x10x20_512x512_64x64probes_40slices_phonon_u0.08"
# DRAM bytes per wave of one launch of each step kernel at 512^2 FP32 (ncu dram__bytes_read.sum +
# dram__bytes_write.sum over one launch of the timed configuration, divided by its waves), measured at this
# workload's autotuned batch of 2048 waves on this build's kernels (plain row pass, per-pair-barrier persistent
# column pass); a kernel change needs a new capture
NCU_DRAM_BYTES_PER_WAVE = {"row_step": (2954996480 + 2893525504) / 2048, "col_step": (3021943552 + 2895444480) / 2048}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="mslice", choices=["mslice", "reference"])
    p.add_argument("--batch", type=int, default=0, help="probes propagated together (0 = engine default)")
    p.add_argument("--scan", type=int, default=64)
    p.add_argument("--variants", default=None,
                   help="column:row step-kernel variants (mslice_set_step_variant) instead of the autotuner's, e.g. 1:1")
    p.add_argument("--no-baseline", action="store_true", help="skip the CPU baseline and plain-FP64 legs")
    p.add_argument("--cpu-probes", type=int, default=32, help="probes in the bounded CPU sample")
    p.add_argument("--sizes", default="256,384,512,768,1024,1536,2048,3072,4096,8192",
                   help="grids of the sizes leg (comma-separated)")
    p.add_argument("--only", default=None, choices=["adjoint", "cbed3d", "uneven", "cufft", "sizes"],
                   help="run one extra leg alone and print its JSON (for profiling it)")
    p.add_argument("--cbed-nz", type=int, default=60, help="FCC cells along z of the cbed3d leg (60: 120 slices)")
    return p.parse_args()


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))


def workload(scan=64, double_precision=False):
    from cltem_b200 import config
    s, st = config.perovskite_stem(n=(10, 10, 20), resolution=512, scan=scan, double_precision=double_precision)
    return s, st


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:  # noqa: BLE001
        return 6650.0, "fallback 6.65 TB/s"


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples of one GPU during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.proc = None
        self.lines = []

    def start(self):
        try:
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
            if self.uuid:
                cmd += ["-i", self.uuid]
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:  # noqa: BLE001
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:  # noqa: BLE001
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, pw, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
                pw.append(float(f[3]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(pw) if pw else None, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------------------------------
# CPU legs (oracle): the baseline beside our line, and the whole reference arm
# ---------------------------------------------------------------------------------------------------
def cpu_sample(n_probes, double_precision, seed=0):
    """Time the CPU restatement on a bounded sample of one configuration of the workload: the transmission
    build of all 40 slices, then n_probes probes through all slices (OpenMP over the probes). Both parts are
    measured; `value` combines them into the rate of a whole 4096-probe configuration (one build, 4096 probes),
    the unit the GPU arm's step is quoted in, and `sample_rate` is the sample's own probe·slices per second."""
    from oracle import bind as ob
    from cltem_b200.params import load_default
    from cltem_b200.structure import phonon_configs
    s, st = workload()
    conf = phonon_configs(st, 1, 0.08, seed=1000 + seed)[0]
    osim = ob.OracleSim(s.cfg, load_default("kirkland"), double_precision=double_precision)
    osim.set_atoms(conf)
    t0 = time.perf_counter()
    osim.build_transmission()
    t1 = time.perf_counter()
    npx = s.cfg.stem_pixels_x * s.cfg.stem_pixels_y
    rng = np.random.default_rng(seed)
    pix = np.sort(rng.choice(npx, size=n_probes, replace=False)).astype(np.int32)
    osim.stem(pix)
    t2 = time.perf_counter()
    S = osim.geo.n_slices
    per_probe = (t2 - t1) / n_probes
    return {"value": npx * S / ((t1 - t0) + per_probe * npx), "sample_rate": n_probes * S / (t2 - t0),
            "build_s": t1 - t0, "propagate_s": t2 - t1, "per_probe_s": per_probe, "sample_s": t2 - t0,
            "probes": n_probes, "slices": S, "configs": 1}


def ref_kernel_leg(seed=0):
    """The reference's own compiled double-precision kernels (oracle/_ref/libref.so, its kernels/*_d.cl built
    for the CPU) beside the restatement, on one slice of the workload's projected potential (the one kernel of
    the path that is not an FFT): seconds per slice for each. The reference kernel runs each 16x16 work group
    as a team of 256 threads, one group after another, as its OpenCL CPU device would; the restatement uses
    OpenMP over pixels. None where the reference kernels were not built."""
    from oracle import bind as ob
    from oracle import ref_bind as rb
    if not rb.available():
        return None
    from cltem_b200.params import load_default
    from cltem_b200.structure import phonon_configs
    s, st = workload(double_precision=True)
    p = load_default("kirkland")
    conf = phonon_configs(st, 1, 0.08, seed=1000 + seed)[0]
    o = ob.OracleSim(s.cfg, p, double_precision=True)
    o.set_atoms(conf)
    g = o.geo
    a = o.sorted_atoms(len(conf))
    k = g.n_slices // 2
    ia = np.array([p.form, p.i_per_atom, s.cfg.resolution, s.cfg.resolution, k, g.n_slices, g.blocks_x, g.blocks_y,
                   g.load_blocks_x, g.load_blocks_y, g.load_blocks_z, s.cfg.full3d_integrals], np.int32)
    da = np.array([g.dz, g.real_scale, g.full_x[1], g.full_x[0], g.full_y[1], g.full_y[0], g.sigma, g.sim_x[0],
                   g.sim_y[0], s.cfg.beam_tilt, s.cfg.beam_azimuth], np.float64)
    out = np.zeros(2 * s.cfg.resolution ** 2)
    vals = np.ascontiguousarray(p.values)
    t0 = time.perf_counter()
    rb.lib().ref_transmission_projected_d(rb.d(out), rb.d(a["x"]), rb.d(a["y"]), rb.d(a["z"]), rb.i(a["Z"]), rb.d(vals),
                                          rb.i(ia), rb.d(da), rb.i(a["block_start"]))
    t1 = time.perf_counter()
    o.build_transmission()   # the oracle's potentials of every slice (its per-slice time is the mean)
    t2 = time.perf_counter()
    mine = o.transmission(k, band_limited=False)
    same = bool(np.array_equal(rb.cplx(out, mine.shape), mine))
    return {"kernel": "transmission_potentials_projected_d, one 512x512 slice of the workload", "reference_s": t1 - t0,
            "restatement_s": (t2 - t1) / g.n_slices, "restatement_note": f"mean over the {g.n_slices} slices of one "
            "build (band limit included)", "identical_output": same}


def cufft_leg(batch=512, steps=20, warmup=3, n=512):
    """The same multislice step built from cuFFT (through torch.fft) and elementwise kernels, timed for
    comparison with the fused passes: per probe·slice, psi <- IFFT2(P * FFT2(T * psi)) on a batch of n² complex64
    waves (1 GiB at 512 waves of 512², larger than L2); neither transform scales, as the fused passes fold the
    scale into P. Device time with CUDA events after warm-up."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(7)
    w = torch.randn(batch, n, n, dtype=torch.complex64, device="cuda", generator=g)
    T = torch.exp(1j * torch.rand(n, n, device="cuda", generator=g)).to(torch.complex64)
    P = (torch.exp(1j * torch.rand(n, n, device="cuda", generator=g)) / (n * n)).to(torch.complex64)
    buf = torch.empty_like(w)

    def step():
        w.mul_(T)
        torch.fft.fft2(w, out=buf)
        buf.mul_(P)
        torch.fft.ifft2(buf, norm="forward", out=w)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        step()
    b.record()
    b.synchronize()
    ms = a.elapsed_time(b) / steps
    del w, buf
    torch.cuda.empty_cache()
    return {"value": batch / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms,
            "sample": f"{steps} steps of {batch} waves of {n}² complex64 after {warmup} untimed",
            "kernels": "torch.fft.fft2 / ifft2 (cuFFT C2C) + 2 elementwise multiplies per step"}


def cpu_baseline_leg(n_probes):
    from oracle import bind as ob
    threads = ob.num_threads()
    r = cpu_sample(n_probes, double_precision=False)
    return {"value": r["value"], "unit": UNIT, "cores": threads, "kind": "port",
            "sample": (f"CPU oracle (C++/OpenMP restatement of the reference path, FP32 instantiation) on one phonon "
                       f"configuration: transmission build of {r['slices']} slices ({r['build_s']:.2f} s, measured) + "
                       f"{n_probes} of 4096 probes through all slices ({r['propagate_s']:.2f} s, measured, "
                       f"{r['per_probe_s']:.3f} s a probe), combined into the rate of a whole 4096-probe configuration; "
                       f"the same sample the reference arm times per step"),
            "build_s": r["build_s"], "per_probe_s": r["per_probe_s"], "sample_s": r["sample_s"],
            "sample_rate": r["sample_rate"], "threads": threads, "reference_kernels": ref_kernel_leg()}


def workload_config(probes, slices, steps):
    """The workload both arms time (the same keys and values in both lines; each arm's engine details are under
    the line's "engine" key)."""
    return {"workload": WORKLOAD, "grid": 512, "probes": probes, "slices": slices, "phonon_configs_per_gpu": steps,
            "precision": "complex64 waves and FFTs; FP64 phase arguments, offsets and Kahan accumulation",
            "l2": "inputs larger than L2 (per configuration: 4096 waves x 2 MiB + 40 transmission slices x 2 MiB)"}


def run_reference(args):
    rank, local, world = dist_env()
    if world > 1 and rank != 0:
        return 0
    from oracle import bind as ob
    ob.lib()
    threads = ob.num_threads()
    n_probes = args.cpu_probes
    # the workload's precision (FP32, the reference's _f path), as the GPU arm
    for w in range(args.warmup):   # untimed: a tiny sample
        cpu_sample(1, double_precision=False, seed=100 + w)
    runs = []
    t0 = time.perf_counter()
    for k in range(args.steps):
        runs.append(cpu_sample(n_probes, double_precision=False, seed=k))
    wall = time.perf_counter() - t0
    value = statistics.mean(r["value"] for r in runs)
    S = runs[0]["slices"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * wall / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(4096, S, args.steps),
        "engine": {"parallelism": "host threads (OpenMP over probes)", "sample_wall_s": wall},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": (f"per step (timed): transmission build of {S} slices + {n_probes} of 4096 probes "
                                    f"through all slices of one phonon configuration, FP32 (the reference's _f path); "
                                    f"value = the measured build and per-probe times combined into the rate of a whole "
                                    f"4096-probe configuration; the reference's OpenCL CPU-device build needs OpenCL "
                                    f"headers/ICD and clFFT, absent here"),
                         "build_s": statistics.mean(r["build_s"] for r in runs),
                         "per_probe_s": statistics.mean(r["per_probe_s"] for r in runs),
                         "sample_rate": statistics.mean(r["sample_rate"] for r in runs),
                         "reference_kernels": ref_kernel_leg()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------------------------------
def adjoint_leg(ctx, ext, warmup):
    """Differentiable CTEM (perovskite 8x8x16, 512^2, 32 slices, FP32): device time of the image loss
    (forward) and of loss + gradients by the adjoint with sqrt(N) checkpointing."""
    import torch
    from cltem_b200 import config
    from cltem_b200.engine import Simulation
    from cltem_b200.structure import phonon_configs
    s, st = config.perovskite_dctem()
    ts, _ = config.perovskite_dctem()
    ts.cfg.C10 = s.cfg.C10 + 30.0
    tsim = Simulation(ctx, ts.cfg)
    tsim.set_atoms(phonon_configs(st, 1, 0.05, seed=77)[0])
    target = tsim.ctem()[2][0]
    tsim.close()
    sim = Simulation(ctx, s.cfg)
    sim.set_atoms(st)

    def timed(fn, reps=3):
        for _ in range(max(1, warmup)):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(ext)
        for _ in range(reps):
            fn()
        b.record(ext)
        b.synchronize()
        return a.elapsed_time(b) / reps

    t_fwd = timed(lambda: sim.ctem_loss(target))
    t_adj = timed(lambda: sim.ctem_loss_grad(target, len(st), checkpoint_every=0))
    t_adj1 = timed(lambda: sim.ctem_loss_grad(target, len(st), checkpoint_every=1))
    sim.close()
    return {"workload": "ctem_perovskite_8x8x16_512x512_32slices_fp32", "forward_ms": t_fwd,
            "loss_and_grad_ms": t_adj, "ratio": t_adj / t_fwd, "checkpoint": "every ceil(sqrt(32)) = 6 slices",
            "loss_and_grad_ms_store_all": t_adj1, "ratio_store_all": t_adj1 / t_fwd,
            "note": "ratio = (forward + adjoint with checkpoint recomputation) / forward, both including the "
                    "transmission build of the 32 slices"}


def parity_leg(ctx, sim, confs, avg_image, n_pixels=8, seed=31):
    """Correctness of the headline run, outside the timed region, on n_pixels seeded scan pixels: the FP32
    engine's image of the first timed configuration (staged and run again through the same batches and
    graphs) against the FP64 CPU oracle, and the FP32 image averaged over every timed configuration against
    the FP64 engine averaged over the same configurations (relative L2 over the pixels)."""
    from oracle import bind as ob
    from cltem_b200.engine import Simulation
    from cltem_b200.params import load_default
    avg32 = np.asarray(avg_image).reshape(-1)
    npx = sim.cfg.stem_pixels_x * sim.cfg.stem_pixels_y
    pix = np.sort(np.random.default_rng(seed).choice(npx, n_pixels, replace=False)).astype(np.int32)
    sim.stage(confs[:1])
    sim.run_staged()
    one32 = sim.staged_result().reshape(-1)
    t0 = time.perf_counter()
    o = ob.OracleSim(sim.cfg, load_default("kirkland"), double_precision=True)
    o.set_atoms(confs[0])
    o.build_transmission()
    ref = o.stem(pix).reshape(-1)
    t_oracle = time.perf_counter() - t0
    s64, _ = workload(double_precision=True)
    sim64 = Simulation(ctx, s64.cfg)
    acc = np.zeros(n_pixels)
    for c in confs:
        sim64.set_atoms(c)
        acc += sim64.stem(pix).reshape(-1)
    sim64.close()
    acc /= len(confs)
    rl2 = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    return {"pixels": pix.tolist(), "fp32_vs_fp64_oracle_config0": rl2(one32[pix], ref),
            "fp32_avg_vs_fp64_engine_avg": rl2(avg32[pix], acc), "configs_averaged": len(confs),
            "tolerance": 1e-5, "oracle_s": t_oracle}


def full3d_evaluations(sim, n_atoms, S, N):
    """Atom-sample evaluations of one full-3D potential build (the unit the CBED full-3D throughput is quoted
    in): for every binned atom, the pixels within 8 Å in xy times the (slice, sub-slice sample) pairs of the
    slices that load the atom's z bin (k +- load_blocks_z) whose sample lies at most 3 Å above it (the one-sided
    test of transmission_potentials_full_3d_f.cl:263), counted on the host from the binned atoms (no beam tilt,
    so the xy test does not depend on the sample)."""
    g = sim.geo
    a = sim.sorted_atoms(n_atoms)
    nb = g.blocks_x * g.blocks_y
    kz_all = (np.searchsorted(a["block_start"], np.arange(len(a["x"])), side="right") - 1) // nb
    dx, x0, y0 = g.real_scale, g.sim_x[0], g.sim_y[0]
    rows = np.arange(-int(8 / dx) - 2, int(8 / dx) + 3)
    I = sim.cfg.full3d_integrals
    total = 0.0
    for c0 in range(0, len(kz_all), 4096):
        ax, ay, az, kz = a["x"][c0:c0 + 4096], a["y"][c0:c0 + 4096], a["z"][c0:c0 + 4096], kz_all[c0:c0 + 4096]
        # pixels of the disk |r - r_a| <= 8 inside the grid, row by row
        iy = np.floor((ay - y0) / dx).astype(np.int64)[:, None] + rows[None, :]
        ry = (y0 + iy * dx) - ay[:, None]
        h2 = 64.0 - ry * ry
        ok = (h2 >= 0) & (iy >= 0) & (iy < N)
        h = np.sqrt(np.where(ok, h2, 0.0))
        lo = np.maximum(np.ceil((ax[:, None] - h - x0) / dx), 0)
        hi = np.minimum(np.floor((ax[:, None] + h - x0) / dx), N - 1)
        px = np.where(ok & (hi >= lo), hi - lo + 1, 0).sum(axis=1)
        pairs = np.zeros(len(kz))
        for off in range(-g.load_blocks_z, g.load_blocks_z + 1):
            k = kz + off
            valid = (k >= 0) & (k < S)
            cz = g.z_lims[0] + (S - k) * g.dz
            for hh in range(I + 1):
                pairs += valid & ((cz - hh * g.dz / I) - az <= 3.0)
        total += float((px * pairs).sum())
    return total


def cbed3d_leg(ctx, ext, nz=60):
    """CBED through the full-3D Lobato potential (FCC Au 20x20x60 cells, 96,000 atoms, 1024^2, 120 slices,
    4 sub-slices, FP32): one phonon configuration (u_rms 0.09 Å) of the 50; the potential build is the bound."""
    import torch
    from cltem_b200 import config
    from cltem_b200.engine import Simulation
    from cltem_b200.params import load_default
    from cltem_b200.structure import phonon_configs
    s, st = config.fcc_cbed(n=(20, 20, nz))
    ctx.load_params(load_default("lobato"))
    sim = Simulation(ctx, s.cfg)
    S, N = sim.geo.n_slices, s.cfg.resolution
    confs = phonon_configs(st, 2, 0.09, seed=90)
    sim.stage(confs[:1])
    sim.run_staged()                        # warm-up (sort, 120-slice build, 120 steps)
    sim.stage(confs[1:])
    sim.profile(True)
    sim.profile_read(reset=True)
    torch.cuda.synchronize()
    sim.run_staged()
    prof = sim.profile_read()
    sim.profile(False)
    t = sim.last_timing()
    sim.set_atoms(confs[1])
    ev = full3d_evaluations(sim, len(st), S, N)
    pot_ms = prof["potential"][0]
    sim.close()
    ctx.load_params(load_default("kirkland"))
    return {"workload": f"cbed_full3d_lobato_fcc_20x20x{nz}_1024x1024_{S}slices_4subslices_fp32",
            "atom_sample_evaluations": ev, "potential_ms": pot_ms,
            "evaluations_per_s": ev / (pot_ms * 1e-3), "config_ms": t["total_ms"],
            "build_ms": t["build_ms"], "propagate_ms": t["propagate_ms"],
            "projected_50_configs_s": 50 * t["total_ms"] * 1e-3,
            "note": "one configuration of the 50; evaluations counted on the host from the binned atoms"}


def sizes_leg(ctx, sizes, dp=False, n_atoms=30, seed=11, tune=True, variants=None):
    """The step kernels at each grid: FP32 (or FP64) STEM of about 1 GiB of waves (at most 1024 probes)
    through 7 slices of 0.25 Å over a 400 Å field holding a few seeded atoms; device time per probe·slice of
    the row and column passes (the column figure includes the last step of each batch, which carries the
    detector reduction), from the engine's per-kernel event timing of the third of three runs. With `tune` the
    autotuner picks each grid's probe batch and step kernels first (as a STEM run of that grid would), and
    the figures are also given per pixel, relative to 512². `variants` = (column, row) fixes the step kernels
    instead (mslice_set_step_variant; the indices are per grid), with the engine's default batch."""
    import torch
    from cltem_b200 import config
    from cltem_b200.engine import Simulation
    from cltem_b200.structure import Structure
    rng = np.random.default_rng(seed)
    st = Structure(rng.choice([8, 22, 38], n_atoms).astype(np.int32), rng.uniform(-40, 40, n_atoms),
                   rng.uniform(-40, 40, n_atoms), rng.uniform(0.2, 1.7, n_atoms))
    out = {}
    for res in sizes:
        s, _ = config.perovskite_stem(n=(1, 1, 1), resolution=res, scan=1, double_precision=dp)
        c = s.cfg
        c.allow_any_resolution = 1
        c.stem_area[:] = [0.0, 0.2, 0.0, 0.2]
        c.padding_xy = 192.0
        c.slice_thickness, c.slice_offset = 0.25, 0.125
        npr = min(1024, max(4, (1 << 30) // (res * res * (16 if dp else 8))))
        k = int(np.ceil(np.sqrt(npr)))
        c.stem_pixels_x = c.stem_pixels_y = k
        s.attach_structure(st)
        sim = Simulation(ctx, c)
        sim.set_atoms(st)
        tuned = None
        if variants is not None:
            sim.set_step_variant(*variants)
        elif tune:
            cands = [b for b in (2, 4, 8, 16, 32, 64, 128, 256, 512, 1024) if b <= npr]
            tuned = sim.tune_batch(cands)
        pix = np.arange(npr, dtype=np.int32)
        sim.stem(pix)
        sim.stem(pix)
        torch.cuda.synchronize()
        sim.profile(True)
        sim.profile_read(reset=True)
        sim.stem(pix)
        torch.cuda.synchronize()
        p = sim.profile_read()
        sim.profile(False)
        S = sim.geo.n_slices
        row_us, col_us = 1e3 * p["row_step"][0] / (npr * S), 1e3 * p["col_step"][0] / (npr * S)
        out[str(res)] = {"probes": npr, "slices": S, "row_us_per_probe_slice": row_us,
                         "col_us_per_probe_slice": col_us, "ps_per_pixel": 1e6 * (row_us + col_us) / (res * res)}
        if tuned or variants is not None:
            tn = sim.tuning()
            out[str(res)].update({"batch": tuned[0] if tuned else tn["batch"], "column": sim.step_variant_name(0, tn["col_variant"]),
                                  "row": sim.step_variant_name(1, tn["row_variant"])})
        sim.close()
    if "512" in out:
        for v in out.values():
            v["per_pixel_vs_512"] = v["ps_per_pixel"] / out["512"]["ps_per_pixel"]
    return {"workload": f"stem_sparse_400A_{'fp64' if dp else 'fp32'}", "sizes": out}


def uneven_leg(ctx, n_cells=48, n_configs=4, seed=2024, streams=4):
    """Uneven batched STEM: 48 seeded perovskite / FCC cells (4-16 cells laterally, 10-80 slices, grids
    256-1024, 80-300 kV, 16-32 mrad, 16x16 probes, 4 phonon configurations each), FP32, each grid with the
    autotuned probe batch and step kernels. The cells are dealt round-robin to `streams` contexts (one CUDA stream
    each); every cell's staged run is one graph launch queued with mslice_stem_run_staged_async, so cells on
    different streams overlap. Setup (tuning, staging) and one untimed run per cell (the graph capture) come
    first; the value is probe·slices of all cells over the device time from the first launch to the last
    completion (CUDA events joined across the streams)."""
    import torch
    from cltem_b200 import config
    from cltem_b200.engine import Context, Simulation
    from cltem_b200.params import load_default
    from cltem_b200.structure import phonon_configs
    rng = np.random.default_rng(seed)
    ctxs = [ctx] + [Context(ctx.device) for _ in range(streams - 1)]
    for c in ctxs[1:]:
        c.load_params(load_default("kirkland"))
    total_ps, setup_s, batches, grids, sims = 0.0, 0.0, {}, {}, []
    for i in range(n_cells):
        s, st = config.uneven_stem_cell(rng)
        t0 = time.perf_counter()
        c = ctxs[i % streams]
        sim = Simulation(c, s.cfg)
        b, _ = sim.tune_batch()   # cached after the first cell of a grid
        batches[s.cfg.resolution] = b
        sim.stage(phonon_configs(st, n_configs, 0.08, seed=seed + i))
        sim.run_staged()          # untimed: captures the cell's run graph
        setup_s += time.perf_counter() - t0
        total_ps += 256 * sim.geo.n_slices * n_configs
        grids[s.cfg.resolution] = grids.get(s.cfg.resolution, 0) + 1
        sims.append(sim)
    torch.cuda.synchronize()
    strm = [torch.cuda.ExternalStream(c.stream(), device=torch.device("cuda", ctx.device)) for c in ctxs]
    start, final = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(strm[0])
    for st_ in strm[1:]:
        st_.wait_event(start)
    for sim in sims:
        sim.run_staged_async()
    for st_ in strm[1:]:
        e = torch.cuda.Event()
        e.record(st_)
        strm[0].wait_event(e)
    final.record(strm[0])
    final.synchronize()
    ms = start.elapsed_time(final)
    serial_ms = 0.0
    for sim in sims:
        sim.wait()
        serial_ms += sim.last_timing()["total_ms"]
        sim.close()
    for c in ctxs[1:]:
        c.close()
    return {"workload": f"uneven_stem_{n_cells}cells_16x16probes_{n_configs}configs_fp32", "value": total_ps / (ms * 1e-3),
            "unit": UNIT, "probe_slices": total_ps, "device_ms": ms, "streams": streams,
            "sum_of_cell_ms": serial_ms, "host_setup_s": setup_s, "cells_per_grid": grids,
            "autotuned_batch_per_grid": batches}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.warmup < 3:
        print("warning: the timing rules ask for >= 3 warm-up steps", file=sys.stderr)
    rank, local, world = dist_env()
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if args.only:   # one extra leg alone (1 GPU)
        from cltem_b200.engine import Context
        from cltem_b200.params import load_default
        ctx = Context(local)
        ctx.load_params(load_default("kirkland"))
        ext = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", local))
        leg = {"adjoint": lambda: adjoint_leg(ctx, ext, args.warmup), "cbed3d": lambda: cbed3d_leg(ctx, ext, args.cbed_nz),
               "uneven": lambda: uneven_leg(ctx), "cufft": lambda: cufft_leg(),
               "sizes": lambda: sizes_leg(ctx, [int(v) for v in args.sizes.split(",")],
                                          variants=tuple(int(v) for v in args.variants.split(":")) if args.variants else None)}[args.only]()
        print(json.dumps({"leg": args.only, **leg}))
        return 0
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    from cltem_b200.engine import Context, Simulation
    from cltem_b200.params import load_default
    from cltem_b200.structure import phonon_configs, concat_configs

    s, st = workload(scan=args.scan)
    if args.batch:
        s.cfg.probe_batch = args.batch
    ctx = Context(local)
    ctx.load_params(load_default("kirkland"))
    sim = Simulation(ctx, s.cfg)
    tuned = None
    if not args.batch:   # the probe batch from the autotuner (untimed; cached per device, grid and precision)
        tuned = sim.tune_batch()
    if args.variants:
        cv, rv = (int(v) for v in args.variants.split(":"))
        sim.set_step_variant(cv, rv)
    tn = sim.tuning()
    step_kernels = {
        "column": sim.step_variant_name(0, tn["col_variant"]),
        "row": sim.step_variant_name(1, tn["row_variant"]),
        "column_candidates": [sim.step_variant_name(0, v) for v in range(tn["col_variants"])],
        "chosen_by": "--variants" if args.variants else ("autotuner (mslice_tune_batch)" if not args.batch else "defaults")}
    S = sim.geo.n_slices
    npx = s.cfg.stem_pixels_x * s.cfg.stem_pixels_y
    N = 512 * 512
    ext = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", local))

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    # warm-up: W configurations (untimed)
    warm = phonon_configs(st, args.warmup, 0.08, seed=10_000 + rank)
    sim.stage(warm)
    sim.run_staged()
    # timed: K configurations staged in HBM before the timed region (inputs resident); one untimed run of the
    # same staged layout captures the whole run into one CUDA graph, so the timed run is a single graph launch
    confs = phonon_configs(st, args.steps, 0.08, seed=rank)
    sim.stage(confs)
    sim.run_staged()
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
        uuid = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
    except Exception:  # noqa: BLE001
        uuid = None
    clocks = ClockSampler(uuid)
    sim.profile(True)
    sim.profile_read(reset=True)
    l0 = ctx.launch_count()
    barrier()
    clocks.start()
    time.sleep(0.4)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    sim.run_staged()
    e1.record(ext)
    e1.synchronize()
    barrier()
    clk = clocks.stop()
    launches = ctx.launch_count() - l0
    prof = sim.profile_read()
    sim.profile(False)
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    img = sim.staged_result()
    img_local = img.copy()   # this rank's average (the parity leg checks it)
    # one exchange step: merge the per-rank image sums and weights (SimulationManager::updateImages)
    from cltem_b200.distributed import merge_average
    img = merge_average(img * args.steps, args.steps, device=torch.device("cuda", local))

    probe_slices = npx * S * args.steps * world
    value = probe_slices / (ms_max / 1000.0)

    # roofline of the dominant kernel (by device time) from the live event timings
    # algorithmic bytes per kernel, the per-unit model of the multislice step: per probe·slice the row pass
    # reads psi and T and writes psi (24 N bytes, complex64), the column pass reads and writes psi (16 N).
    # The engine moves fewer: columns outside the propagator's cut are never read or written; its own count
    # of the bytes each launch must move is reported beside ("design_bytes").
    row_ms, row_n, row_dbytes = prof["row_step"]
    col_ms, col_n, col_dbytes = prof["col_step"]
    units = npx * S * args.steps              # probe·slices on this rank
    row_bytes, col_bytes = 24.0 * N * units, 16.0 * N * units
    dom = ("row_step", row_bytes, row_ms, row_n) if row_ms >= col_ms else ("col_step", col_bytes, col_ms, col_n)
    peak, peak_src = peaks()
    achieved = dom[1] / (dom[2] / 1000.0) / 1e9
    # DRAM bytes per wave from one ncu capture of this build's step kernels, scaled to this run's launches
    per_wave = NCU_DRAM_BYTES_PER_WAVE.get(dom[0])
    traffic = per_wave * (npx * S * args.steps) / max(dom[3], 1) if per_wave else None
    roofline = {"bound": "hbm", "kernel": dom[0], "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                "algorithmic_bytes_per_launch": dom[1] / max(dom[3], 1), "avg_launch_ms": dom[2] / max(dom[3], 1),
                "pair_achieved_gbs": (row_bytes + col_bytes) / ((row_ms + col_ms) / 1000.0) / 1e9,
                "pair_frac": (row_bytes + col_bytes) / ((row_ms + col_ms) / 1000.0) / 1e9 / peak,
                "design_bytes": {"row_step": row_dbytes, "col_step": col_dbytes},
                "design_pair_gbs": (row_dbytes + col_dbytes) / ((row_ms + col_ms) / 1000.0) / 1e9,
                "kernel_ms": {k: v[0] for k, v in prof.items()}, "kernel_launches": {k: v[1] for k, v in prof.items()},
                "kernel_bytes": {k: v[2] for k, v in prof.items()}}

    # end to end through the public API: one configuration per step from pinned host memory, result back
    e2e = None
    if rank == 0 or world > 1:
        cnt, Z, x, y, z = concat_configs(confs[:1])
        pinned = [torch.from_numpy(a).pin_memory() for a in (Z, x, y, z)]
        out = torch.zeros(sim.result_size(), dtype=torch.float64).pin_memory()
        cnt_arr = np.ascontiguousarray(cnt)
        lib = ctx.lib
        ptr = lambda tns, ty: C.cast(C.c_void_p(tns.data_ptr()), C.POINTER(ty))
        e2e_confs = phonon_configs(st, min(args.steps, 3), 0.08, seed=50_000 + rank)
        barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(ext)
        for c in e2e_confs:
            _, Zc, xc, yc, zc = concat_configs([c])
            for dst, src in zip(pinned, (Zc, xc, yc, zc)):
                dst.numpy()[:] = src
            rc = lib.mslice_stem_simulate(sim.h, 1, cnt_arr.ctypes.data_as(C.POINTER(C.c_size_t)), ptr(pinned[0], C.c_int),
                                          ptr(pinned[1], C.c_double), ptr(pinned[2], C.c_double), ptr(pinned[3], C.c_double),
                                          ptr(out, C.c_double), out.numel())
            assert rc == 0, lib.mslice_last_error()
        f1.record(ext)
        f1.synchronize()
        ms_e2e = f0.elapsed_time(f1)
        te = torch.tensor([ms_e2e], device="cuda")
        if world > 1:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        ms_e2e = float(te.item())
        h2d = int(sum(p.numel() * p.element_size() for p in pinned))
        e2e = {"value": npx * S * len(e2e_confs) * world / (ms_e2e / 1000.0), "unit": UNIT,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": int(out.numel() * 8),
               "steps": len(e2e_confs), "ms_per_step": ms_e2e / len(e2e_confs)}

    parity = None
    if rank == 0 and not args.no_baseline:
        parity = parity_leg(ctx, sim, confs, img_local)

    adjoint = cbed3d = uneven = None
    if rank == 0 and world == 1 and not args.no_baseline:
        adjoint = adjoint_leg(ctx, ext, args.warmup)
        cbed3d = cbed3d_leg(ctx, ext)
        uneven = uneven_leg(ctx)

    cpu = plain = cufft = None
    if rank == 0 and world == 1 and not args.no_baseline:
        # plain per-probe FP64 GPU path (the reference's unfused order with cuFFT Z2Z) on a sample
        sd, std_ = workload(double_precision=True)
        simd = Simulation(ctx, sd.cfg)
        simd.set_atoms(confs[0])
        simd.build_transmission()
        pix = np.arange(16, dtype=np.int32)
        simd.stem_plain(pix[:1])   # untimed: allocates the path's buffers and cuFFT plan, which later calls reuse
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(ext)
        simd.stem_plain(pix)
        g1.record(ext)
        g1.synchronize()
        pms = g0.elapsed_time(g1)
        pv = len(pix) * S / (pms / 1000.0)
        # the fused FP64 engine on the same configuration (one batch of 512 probes): the design's gain at the
        # reference's own precision
        fpix = np.arange(512, dtype=np.int32)
        for _ in range(2):   # untimed warm-up: batch buffers and the batches' CUDA-graph capture
            simd.stem(fpix)
        torch.cuda.synchronize()
        g0.record(ext)
        for _ in range(3):
            simd.stem(fpix)
        g1.record(ext)
        g1.synchronize()
        fv = 3 * len(fpix) * S / (g0.elapsed_time(g1) / 1000.0)
        plain = {"value": pv, "unit": UNIT, "sample": f"{len(pix)} probes x {S} slices, FP64, one probe at a time",
                 "fused_fp32_over_plain_fp64": value / pv,
                 "fused_fp64": {"value": fv, "unit": UNIT, "sample": f"3 runs of {len(fpix)} probes x {S} slices after 2 untimed",
                                "fused_fp64_over_plain_fp64": fv / pv}}
        simd.close()
        cufft = cufft_leg()
        cufft["fused_fp32_over_cufft"] = value / cufft["value"]
        cpu = cpu_baseline_leg(args.cpu_probes)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": workload_config(npx, S, args.steps),
            "engine": {"probe_batch": sim.cfg.probe_batch or (f"{tuned[0]} (autotuned: {tuned[1]:.0f} waves/s per slice step)" if tuned else "engine default"),
                       "step_kernels": step_kernels,
                       "parallelism": f"dp{world} (phonon configurations sharded over GPUs)"},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "plain_fp64_gpu": plain,
            "cufft_fp32_step": cufft,
            "adjoint_forward_ratio": adjoint["ratio"] if adjoint else None,
            "adjoint": adjoint,
            "cbed_full3d": cbed3d,
            "uneven_stem": uneven,
            "e2e": e2e,
            "parity": parity,
            "gpu_launches": launches,
            "clocks": clk,
        }
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
