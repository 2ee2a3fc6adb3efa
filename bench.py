#!/usr/bin/env python
"""Benchmark: pixels/s of the Milne-Eddington inversion on B200.

Workload (one "step"): invert the 256x256-pixel, 30-wavelength, PSF-convolved,
9-free-parameter cube (benchmark configuration 1; Fe I 6173.3354 A, grid
-350..375 mA in 25 mA steps, Gaussian PSF FWHM 60 mA through the 1 mA table
route, sigma = 1e-3 noise, <= 50 LM iterations) with the FP32 batched form.
Synthetic data: seeded atmospheres whose profiles are synthesized by the
reference's own mil_sinrf (its C sources built with REAL = double under oracle/,
outside every timed region), plus seeded N(0, 1e-3) noise; both arms invert the
same cube.  Cubes above 4 GB (configuration 4) are synthesized on the device by
this library's FP64 path instead.

JSON line (rank 0):
  value    pixels/s with the cube resident in HBM (CUDA-event time of the
           inversion kernel; L2 flushed between steps)
  e2e      pixels/s through the public call (Inverter.invert -> pm_invert_batch)
           with the cube and the result arrays in pinned host memory, timed by the
           wall clock around the call: the host->device copy of the cube and the
           device->host transfer of models, chi^2 and iterations (stored by the
           kernel into the pinned arrays, or copied back) are inside it
  plain    the FP64 plain form on the same cube (eigen solve, and Cholesky)
  roofline FP32-pipe fraction from the frozen flop model (below: add/sub/mul/div 1,
           FMA 2, transcendentals 0, per pixel and iteration)
  cpu_baseline  the reference's own C hot path (oracle/_ref, float build,
           -O3) on every host core, forked slabs like pmilos' Scatterv

--impl reference: the reference's own C hot path (oracle/_ref, REAL = float, -O3)
on every host core, one forked process per contiguous slab (pmilos' Scatterv
partition), inverting the whole cube each step; rank 0 only.  This arm loads no
library of this package.
Multi-GPU (torchrun): every rank inverts its own cube (weak scaling, replicas:
pixels are independent, there is no collective on the data path); time is the
max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "p-milos_b200"))

# ---- frozen flop model (per pixel; counted from the reference statements) ----
F_VOIGT = 100


def flop_model(nl: int, taps: int, K: int, psf: bool, stray: bool):
    F_syn = nl * (3 * F_VOIGT + 100) + (8 * nl * taps if psf else 0) + (12 * nl if stray else 0)
    F_rf = 870 * nl + (8 * nl * taps * (K - 1) if psf else 0) + (4 * nl * K if stray else 0)
    F_ne = 4 * nl * (K * K + 3 * K)
    F_chi = 20 * nl
    F_solve = 9 * K ** 3 + 4 * K ** 2
    return dict(F_syn=F_syn, F_rf=F_rf, F_ne=F_ne, F_chi=F_chi, F_solve=F_solve)


def flops(fm, pixels, iterations, accepted):
    fp32 = pixels * (fm["F_syn"] + fm["F_rf"] + fm["F_ne"] + fm["F_chi"]) + iterations * (
        fm["F_syn"] + fm["F_chi"]) + accepted * (fm["F_rf"] + fm["F_ne"])
    fp64 = iterations * fm["F_solve"]
    return fp32, fp64


# ---- clocks sampled during the timed region ----
class ClockSampler:
    """nvidia-smi sampling every 100 ms while the timed region runs."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.lines = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=10)
            except Exception:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        rows = [[x.strip() for x in l.split(",")] for l in self.lines]
        rows = [r for r in rows if len(r) == 7]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [v for v in (num(r[0]) for r in rows) if v is not None]
        mx = [v for v in (num(r[1]) for r in rows) if v is not None]
        pw = [v for v in (num(r[2]) for r in rows) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[3 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(pw) if pw else None, "reasons": reasons, "samples": len(rows)}


# ---- the reference's own code on the host cores (input synthesis, CPU baseline, reference arm) ----
_W = {}


def load_specs():
    """pmilos_b200/specs.py loaded by file path: the workload definitions
    without importing the package (the reference arm maps no library of it)."""
    import importlib.util

    path = os.path.join(ROOT, "p-milos_b200", "pmilos_b200", "specs.py")
    spec = importlib.util.spec_from_file_location("pm_bench_specs", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class RefWorkload:
    """A benchmark configuration built with numpy and the reference's own host
    routines (interpolationLinearPSF / fgauss_WL through oracle/_ref)."""

    def __init__(self, cfg: int, npix: int | None):
        import pyoracle as po

        S = load_specs()
        self.cfg = cfg
        ini, step, fin, self.lambda0 = S.grid_spec(cfg)
        self.offs, self.lam = S.grid_from_malla(ini, step, fin, self.lambda0)
        self.cuantic = np.array([1.0, *S.TRIPLET])
        self.npix = npix or S.DEFAULT_NPIX[cfg]
        self.seed = cfg
        self.nterms, self.fix, self.guess = S.nterms_fix_guess(cfg)
        self.noise = (1.0 / S.SN) ** 2
        self.miter = 50
        flavour = "f64" if po.reference_available("f64") else None
        lib = po.Reference if flavour else po.Restatement
        self.synth_kind = "reference" if flavour else "port"
        route = S.psf_route(cfg)
        self.psf = None
        if route is not None:
            helper = po.Reference(po.LineSetup(self.lam, self.lambda0, self.cuantic, None, self.nterms), "f64") \
                if flavour else None
            if route[0] == "table":
                x, y = S.gaussian_psf_table(route[1])
                self.psf = helper.interp_psf(x, y, self.offs, 0.0) if helper else None
            else:
                nl = self.lam.size
                self.psf = helper.fgauss_wl(route[1], self.lam[1] - self.lam[0], self.lam[0], self.lam[nl // 2], nl) \
                    if helper else None
            if self.psf is None:
                raise RuntimeError("the reference build (oracle/_ref) is needed for the PSF route")
        self.slight = None
        if cfg == 2:  # stray light: the synthesis of a B = 0 atmosphere
            one = lib(po.LineSetup(self.lam, self.lambda0, self.cuantic, self.psf, self.nterms), "f64")
            self.slight = one.synth(S.QUIET_SUN_B0, None, fix=self.fix, rf=False)[0].astype(np.float32)
        self.specs = S

    @property
    def nl(self) -> int:
        return int(self.lam.size)

    def setup_args(self):
        return (self.lam, self.lambda0, self.cuantic, self.psf, self.nterms)


def _worker_init(lib, lam, lambda0, cq, psf, nterms):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po

    setup = po.LineSetup(lam, lambda0, cq, psf, nterms)
    if lib.startswith("port_"):
        _W["ref"] = po.Restatement(setup, lib[5:])
    else:
        _W["ref"] = po.Reference(setup, lib)


def _worker_synth(args):
    truth, slight, fix = args
    ref = _W["ref"]
    sl = None if slight is None else np.asarray(slight, dtype=np.float64)
    return np.array([ref.synth(m, sl, fix=fix, rf=False)[0] for m in truth], dtype=np.float32)


def _worker_invert(args):
    obs, guess, fix, noise, slight = args
    t0 = time.perf_counter()
    _W["ref"].invert(obs, guess, fix=fix, noise=noise, slight=slight, want_spectra=False)
    return time.perf_counter() - t0


def reference_cube(rw: RefWorkload, seed: int, cores: int):
    """Seeded observed cube [npix][4][nl] float32 of configuration rw.cfg: truth
    atmospheres from specs.truth_models, profiles synthesized by the reference's
    mil_sinrf (REAL = double) on `cores` spawned processes, then N(0, 1e-3) noise
    from the same generator."""
    import multiprocessing as mp

    rng = np.random.default_rng(seed)
    truth = rw.specs.truth_models(rw.cfg, rw.npix, rng)
    lib = "f64" if rw.synth_kind == "reference" else "port_f64"
    parts = np.array_split(truth, max(1, min(cores, rw.npix // 256 or 1)))
    with mp.get_context("spawn").Pool(min(cores, len(parts)), initializer=_worker_init,
                                      initargs=(lib, *rw.setup_args())) as pool:
        obs = np.concatenate(pool.map(_worker_synth, [(t, rw.slight, rw.fix) for t in parts]))
    obs = obs + rng.normal(0.0, rw.specs.NOISE_SIGMA, obs.shape).astype(np.float32)
    return np.ascontiguousarray(obs, dtype=np.float32)


class ReferencePool:
    """The reference's inversion (oracle/_ref float build, -O3: the reference
    makefile's default REAL = float) on `cores` spawned processes; each call
    inverts contiguous slabs, one per process (pmilos.c:1181-1205)."""

    def __init__(self, rw: RefWorkload, cores: int):
        import multiprocessing as mp

        import pyoracle as po

        self.kind = "reference" if po.reference_available("f32_fast") else "port"
        lib = "f32_fast" if self.kind == "reference" else "port_f32"
        self.rw, self.cores = rw, cores
        self.noise32 = float(np.float32(np.float32(1.0 / rw.specs.SN) ** 2))
        self.pool = mp.get_context("spawn").Pool(cores, initializer=_worker_init, initargs=(lib, *rw.setup_args()))

    def run(self, obs: np.ndarray) -> tuple:
        """Invert obs on every process; returns (wall s, slowest slab s)."""
        rw = self.rw
        slabs = np.array_split(obs, self.cores)
        t0 = time.perf_counter()
        per = self.pool.map(_worker_invert, [(sl, rw.guess, rw.fix, self.noise32, rw.slight) for sl in slabs])
        return time.perf_counter() - t0, max(per)

    def close(self):
        self.pool.close()
        self.pool.join()


def cpu_baseline(rw: RefWorkload, obs, sample_pixels: int, cores: int):
    """The reference's inversion on `cores` processes over a bounded sample of
    the cube (contiguous slabs).  Returns (pixels/s, info)."""
    n = min(sample_pixels, obs.shape[0])
    ref = ReferencePool(rw, cores)
    try:
        ref.run(obs[:2 * cores])  # warm-up
        wall, slab = ref.run(obs[:n])
    finally:
        ref.close()
    info = {"kind": ref.kind, "cores": cores, "sample": f"{n} pixels of the workload in {cores} contiguous slabs",
            "wall_s": round(wall, 3), "max_slab_s": round(slab, 3)}
    return n / wall, info


def _mem_available() -> int:
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---- cube ingest ----
def bench_ingest(args, rank: int):
    """pm_fits_reorder on a 512 x 512 x 4 x 112 float32 cube (470 MB) written in
    three axis orders; bytes/s = 2 x data block (read + write) per launch."""
    import ctypes

    import torch

    import pmilos_b200 as pm
    from pmilos_b200.files import cube_fits_bytes

    size = {"R": 512, "C": 512, "L": 112, "S": 4}
    role = {"R": "HPLN-TAN", "C": "HPLT-TAN", "L": "WAVE-GRI", "S": "STOKES"}
    L = pm.load_library()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    hbm_peak = json.load(open(peaks_path))["hbm_gbs"] if os.path.exists(peaks_path) else 6650.0
    rows = {}
    e2e = None
    for order in ("LSRC", "LRSC", "RCLS"):
        dims = [size[r] for r in order]
        data = np.random.default_rng(1).standard_normal(dims[::-1], dtype=np.float32)
        raw = cube_fits_bytes(data, [role[r] for r in order])
        info = pm._fits_struct(np.frombuffer(raw, dtype=np.uint8))
        o, n = int(info.data_offset), int(info.data_bytes)
        host = torch.from_numpy(np.frombuffer(raw, dtype=np.uint8)[o:o + n].copy()).pin_memory()
        dev = host.to("cuda")
        out = torch.empty((int(info.npix), 4, int(info.nlambda)), dtype=torch.float32, device="cuda")
        st = torch.cuda.current_stream().cuda_stream

        def launch():
            rc = L.pm_fits_reorder(ctypes.byref(info), dev.data_ptr(), out.data_ptr(), ctypes.c_void_p(st))
            if rc != 0:
                raise RuntimeError(L.pm_last_error().decode())

        for _ in range(max(3, args.warmup)):
            launch()
        ts, te = [], []
        for _ in range(args.steps):
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            launch()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
            # end to end: the data block from pinned host memory, then the reorder
            e0.record()
            dev.copy_(host, non_blocking=True)
            launch()
            e1.record()
            torch.cuda.synchronize()
            te.append(e0.elapsed_time(e1))
        ms, ms_e2e = float(np.median(ts)), float(np.median(te))
        rows[order] = {"ms": ms, "gbs": 2 * n / ms / 1e6, "frac": 2 * n / ms / 1e6 / hbm_peak,
                       "e2e_ms": ms_e2e, "bytes_per_launch": 2 * n}
        if order == "LSRC":
            e2e = n / ms_e2e / 1e6
    v = rows["LSRC"]
    if rank == 0:
        print(json.dumps({
            "metric": "FITS cube ingest (byte swap + reorder) on 1 B200", "value": v["gbs"], "unit": "GB/s",
            "n_gpus": 1, "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": v["ms"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": "512 x 512 pixels x 4 Stokes x 112 wavelengths float32 (470 MB), axis orders "
                                   "(wavelength, Stokes, rows, columns) = the reference's default, "
                                   "(wavelength, rows, Stokes, columns), (rows, columns, wavelength, Stokes)",
                       "l2": "flushed between timed launches (256 MiB write)"},
            "e2e": {"value": e2e, "unit": "GB/s of data block", "h2d_bytes_per_step": rows["LSRC"]["bytes_per_launch"] // 2,
                    "d2h_bytes_per_step": 0},
            "roofline": {"bound": "hbm", "achieved": v["gbs"], "peak": hbm_peak, "unit": "GB/s", "frac": v["frac"],
                         "traffic": None, "peak_source": "MEASURED_PEAKS.json hbm_gbs"},
            "orders": rows, "gpu_launches": len(rows) * (args.steps * 2 + max(3, args.warmup))}), flush=True)


# ---- served stream (configuration 3) ----
SIZES = (256 * 256, 512 * 512, 1024 * 1024, 2048 * 2048)


def bench_served(args, rank: int, world: int, metric: str):
    """Poisson stream of scans (mean 20/s) through pm_server: each scan a cube of
    256^2..2048^2 pixels on one of the 6/15/30-point grids, FP32; then the first
    --plain-requests scans of the same schedule on a plain FP64 server."""
    import torch

    import pmilos_b200 as pm
    from pmilos_b200 import workloads

    # N > 1: replicas, every rank serves its own stream (no collective)
    line = pm.LineData(workloads.FE6173, workloads.TRIPLET)
    specs = [workloads.config(3, npix=1, grid=g) for g in range(3)]

    def grids(precision):
        return [pm.Grid(lam=w.lam, psf=w.psf, guess=w.guess, noise=w.noise, fix=w.fix, nterms=9,
                        precision=precision) for w in specs]

    rng = np.random.default_rng(3 + 1000 * rank)
    n = args.requests + args.warmup
    arrivals = np.cumsum(rng.exponential(1.0 / 20.0, n))
    sizes = rng.choice(len(SIZES), n)
    which = rng.choice(3, n)
    # one pinned cube per (size, grid): synthesized on the device, FP64, seeded
    pool = {}
    for si, g in sorted(set(zip(sizes.tolist(), which.tolist()))):
        w = workloads.config(3, npix=SIZES[si], grid=g)
        with pm.Inverter(w.line, w.lam, w.psf, noise=w.noise, fix=w.fix, nterms=9, precision=pm.PREC_FP64) as inv64:
            d = workloads.synthesize_device(w, inv64, seed=100 * si + g + 1000 * rank)
        h = torch.empty(tuple(d.shape), dtype=torch.float32, pin_memory=True)
        h.copy_(d)
        del d
        pool[(si, g)] = h.numpy()
    torch.cuda.empty_cache()

    def run(precision, count, rate_scale=1.0):
        """Replay scans warmup..warmup+count of the schedule, arrival times
        scaled by 1/rate_scale (rate_scale < 1: a lighter load than 20 scans/s)."""
        infos = []
        with pm.Server(line, grids(precision), hbm_budget_bytes=int(args.budget_gb * (1 << 30)), max_inflight=64,
                       linger_ms=5.0) as srv:
            for i in range(min(args.warmup, count)):  # warm-up scans (untimed): smallest cube of each grid
                srv.wait(srv.submit(int(which[i]), pool[(0, int(which[i]))] if (0, int(which[i])) in pool else
                                    pool[(int(sizes[i]), int(which[i]))]))
            t0 = time.perf_counter()
            ids = []
            for i in range(args.warmup, args.warmup + count):
                dt = t0 + (arrivals[i] - arrivals[args.warmup]) / rate_scale - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
                ids.append(srv.submit(int(which[i]), pool[(int(sizes[i]), int(which[i]))], want_status=False))
            for sid in ids:
                r = srv.wait(sid)
                infos.append(r["info"])
            st = srv.stats()
        first = min(x["submit_ms"] for x in infos)
        last = max(x["done_ms"] for x in infos)
        lat = np.array([x["done_ms"] - x["submit_ms"] for x in infos])
        svc = np.array([x["done_ms"] - x["admit_ms"] for x in infos])
        queue = np.array([x["admit_ms"] - x["submit_ms"] for x in infos])
        pix = sum(x["npix"] for x in infos)
        its = sum(x["iterations"] for x in infos)
        span = (arrivals[args.warmup + count - 1] - arrivals[args.warmup]) / rate_scale
        return {"pixels_per_s": pix / ((last - first) / 1000.0), "pixels": int(pix), "scans": len(infos),
                "offered_pixels_per_s": pix / span if span > 0 else None,
                "arrival_rate_scans_per_s": 20.0 * rate_scale,
                "wall_ms": last - first, "latency_p50_ms": float(np.percentile(lat, 50)),
                "latency_p99_ms": float(np.percentile(lat, 99)), "latency_max_ms": float(lat.max()),
                "service_p50_ms": float(np.percentile(svc, 50)), "service_p99_ms": float(np.percentile(svc, 99)),
                "queue_p50_ms": float(np.percentile(queue, 50)), "queue_p99_ms": float(np.percentile(queue, 99)),
                "kernel_launches": st["kernel_launches"], "prepass_launches": st["prepass_launches"],
                "arena_peak_gib": st["arena_peak_bytes"] / 2**30,
                "iterations_per_pixel": its / pix}

    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        fp32 = run(pm.PREC_FP32, args.requests)
    # the same scans offered below capacity (arrivals slowed to half the rate the
    # first run served): latency without a backlog
    light = None
    if args.light_load:
        scale = 0.5 * fp32["pixels_per_s"] / fp32["offered_pixels_per_s"]
        light = run(pm.PREC_FP32, args.requests, rate_scale=min(1.0, scale))
    plain = run(pm.PREC_FP64, min(args.plain_requests, args.requests)) if args.plain_requests > 0 else None
    h2d = sum(pool[(int(sizes[i]), int(which[i]))].nbytes for i in range(args.warmup, n)) / args.requests
    d2h = sum(SIZES[int(sizes[i])] for i in range(args.warmup, n)) * (11 * 8 + 4 + 4) / args.requests
    cfg_desc = {"workload": "served stream: Poisson scans (mean 20/s), cubes of 256^2..2048^2 pixels on 6/15/30-point "
                            "grids around Fe I 6173.3354 A, 60 mA PSF, 9 free parameters, config-2 atmosphere mix",
                "scans": args.requests, "hbm_budget_gib": args.budget_gb, "parallelism": f"replicas x{world}",
                "l2": "scan cubes (up to 2 GB) exceed L2; no flush"}
    if rank == 0:
        print(json.dumps({
            "metric": metric + " (served stream)", "value": fp32["pixels_per_s"], "unit": "pixels/s",
            "n_gpus": world, "steps": args.requests, "warmup": args.warmup,
            "ms_per_step": fp32["wall_ms"] / args.requests, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": cfg_desc,
            "e2e": {"value": fp32["pixels_per_s"], "unit": "pixels/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "note": "host clock from each scan's submit (host buffers) to its results in host memory"},
            "latency_ms": {"p50": fp32["latency_p50_ms"], "p99": fp32["latency_p99_ms"],
                           "max": fp32["latency_max_ms"], "service_p50": fp32["service_p50_ms"],
                           "service_p99": fp32["service_p99_ms"],
                           "note": "latency: submit -> results in host memory; service: admit -> results"},
            "offered_pixels_per_s": fp32["offered_pixels_per_s"],
            "served_fp32": fp32, "served_fp32_light_load": light, "plain_fp64": plain, "clocks": clk.summary(),
            "gpu_launches": fp32["kernel_launches"] + fp32["prepass_launches"]}), flush=True)


# ---- the batch configurations: description, inputs, reference arm ----
def describe(rw: RefWorkload, gpus: int) -> dict:
    psf_desc = "no PSF" if rw.psf is None else "Gaussian PSF"
    stray_desc = ", stray light mixed at alpha~U(0.7,1)" if rw.cfg == 2 else ""
    return {"workload": f"ME inversion, benchmark configuration {rw.cfg}: {rw.npix} pixels "
                        f"({int(np.sqrt(rw.npix))}^2) x 4 Stokes x {rw.nl} wavelengths, Fe I {rw.lambda0} A, "
                        f"{psf_desc}{stray_desc}, {rw.nterms} free parameters, <= {rw.miter} LM iterations",
            "pixels_per_step": rw.npix, "nlambda": rw.nl, "nterms": rw.nterms,
            "parallelism": f"replicas x{gpus}", "l2": "flushed between timed steps (256 MiB write)"}


def data_desc(rw: RefWorkload, on_device: bool) -> str:
    if on_device:
        return ("synthetic: seeded atmospheres drawn on the device, profiles synthesized by this library's FP64 "
                "path, N(0, 1e-3) noise")
    who = "the reference's mil_sinrf (REAL = double)" if rw.synth_kind == "reference" else \
        "the oracle's restatement of mil_sinrf (FP64)"
    return f"synthetic: seeded atmospheres (seed {rw.seed}), profiles synthesized by {who}, N(0, 1e-3) noise"


def reference_arm(args, rank: int, metric: str):
    """--impl reference: the reference's own C hot path on every host core,
    inverting the whole cube (configurations 0-2; a bounded sample of the 30 GB
    configuration 4) every step, one process per contiguous slab."""
    if rank != 0:
        return
    if args.ingest or args.config == 3:
        why = "the reference has no serving mode" if args.config == 3 else "the reference reads FITS on the host"
        print(json.dumps({"impl": "reference", "unavailable": why}), flush=True)
        return
    cores = host_cores()
    rw = RefWorkload(args.config, args.npix)
    cfg_desc = describe(rw, args.gpus)
    whole = rw.npix * rw.nl * 16 <= (4 << 30)
    if not whole:
        rw.npix = args.cpu_sample or 200 * cores  # a bounded sample of the same distributions
    obs = reference_cube(rw, rw.seed, cores)
    ref = ReferencePool(rw, cores)
    walls = []
    try:
        for _ in range(args.warmup + args.steps):
            walls.append(ref.run(obs)[0])
    finally:
        ref.close()
    t = float(np.mean(walls[args.warmup:]))
    val = rw.npix / t
    sample = (f"the whole cube ({rw.npix} pixels) every step, {cores} contiguous slabs" if whole else
              f"{rw.npix} pixels of the workload's distributions every step, {cores} contiguous slabs")
    print(json.dumps({"metric": metric, "value": val, "unit": "pixels/s", "impl": "reference",
                      "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                      "ms_per_step": 1000.0 * t, "higher_is_better": True, "scaling": "weak",
                      "vs_baseline": None, "dtype": "f32", "data": data_desc(rw, False), "config": cfg_desc,
                      "cpu_baseline": {"value": val, "unit": "pixels/s", "cores": cores, "kind": ref.kind,
                                       "sample": sample},
                      "e2e": {"value": val, "unit": "pixels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
          flush=True)


# ---- main ----
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=1)
    ap.add_argument("--npix", type=int, default=None)
    ap.add_argument("--cpu-sample", type=int, default=None, help="pixels timed on the CPU baseline")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--plain-npix", type=int, default=None,
                    help="pixels of the cube the plain FP64 forms invert (default: all, or 2^18 above 2^20)")
    ap.add_argument("--requests", type=int, default=48, help="served stream (configuration 3): scans timed")
    ap.add_argument("--plain-requests", type=int, default=12,
                    help="served stream: scans of the same schedule timed on the plain FP64 server")
    ap.add_argument("--budget-gb", type=float, default=24.0, help="served stream: device arena of the server")
    ap.add_argument("--light-load", type=int, default=1,
                    help="served stream: also replay the scans at half the served rate (1) or not (0)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch tuning")
    ap.add_argument("--tuning", default=None, help="variant,warps_per_block: this launch tuning, no autotuning")
    ap.add_argument("--ingest", action="store_true",
                    help="time the FITS cube ingest (512x512 pixels x 112 wavelengths, three axis orders)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    metric = "pixels/s inverted on 1 B200"
    # the reference's own code (oracle/): input synthesis, CPU baseline, reference arm
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    if args.impl == "reference":
        return reference_arm(args, rank, metric)

    rw = None
    if not args.ingest and args.config != 3:
        # inputs first (spawned CPU processes, before any CUDA call)
        rw = RefWorkload(args.config, args.npix)
        cfg_desc = describe(rw, args.gpus)
        big = rw.npix * rw.nl * 16 > (4 << 30)
        obs = None if big else reference_cube(rw, rw.seed + 1000 * rank, max(1, host_cores() // world))

    import torch

    import pmilos_b200 as pm
    from pmilos_b200 import workloads

    torch.cuda.set_device(local)
    if args.ingest:
        return bench_ingest(args, rank)
    if args.config == 3:
        return bench_served(args, rank, world, metric)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    w = workloads.config(args.config, npix=args.npix)
    w.slight = rw.slight  # the reference's synthesis of the B = 0 atmosphere (configuration 2)
    inv32 = pm.Inverter(w.line, w.lam, w.psf, noise=w.noise, fix=w.fix, nterms=w.nterms, precision=pm.PREC_FP32)
    inv64 = pm.Inverter(w.line, w.lam, w.psf, noise=w.noise, fix=w.fix, nterms=w.nterms, precision=pm.PREC_FP64)
    if obs is None:
        # cubes above 4 GB are drawn and synthesized on the device, in chunks
        obs_d = workloads.synthesize_device(w, inv64, seed=w.seed + 1000 * rank)
    else:
        obs_d = torch.as_tensor(obs, device="cuda")
    sl_h = None if w.slight is None else np.ascontiguousarray(w.slight, dtype=np.float32)
    sl_d = None if sl_h is None else torch.as_tensor(sl_h, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    # the project's autotuner picks the launch tuning on a sample of this cube (untimed)
    if args.tuning:
        v, wpb = (int(x) for x in args.tuning.split(","))
        inv32.tuning = {"variant": v, "warps_per_block": wpb}
    elif not args.no_autotune:
        ns = min(w.npix, 65536)  # configurations 0-2: the whole cube (a smaller one has a different tail)
        sample = torch.from_numpy(np.ascontiguousarray(obs[:ns])) if obs is not None else obs_d[:ns].cpu()
        sample = sample.pin_memory()  # pinned, as e2e's input
        inv32.autotune(sample.numpy(), w.guess, slight=sl_h, reps=3)
        del sample
    tuning = inv32.tuning

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def step_device(inv, cube=None):
        flush.fill_(1)  # L2 flush outside the timed kernel
        r = inv.invert(obs_d if cube is None else cube, w.guess, slight=sl_d, want_spectra=False,
                       want_status=False)
        s = inv.stats()
        return r, s

    for _ in range(args.warmup):
        step_device(inv32)
    barrier()
    kms, iters, acc, launches = [], 0, 0, 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            r, s = step_device(inv32)
            kms.append(s["kernel_ms"])
            iters += s["iterations"]
            acc += s["accepted"]
            launches += 2  # classical-estimates pre-pass + inversion kernel
        barrier()
    ms = float(np.mean(kms))
    if dist is not None:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * w.npix / (ms / 1000.0)

    # e2e: host buffers (pinned) through the C ABI; copies inside the timed region
    e2e_v, e2e_note = None, None
    cube_bytes = obs_d.numel() * 4
    room = obs is not None or _mem_available() >= 3 * cube_bytes
    if dist is not None:  # every rank takes the same branch (the e2e leg has a collective)
        f = torch.tensor([1 if room else 0], device="cuda", dtype=torch.int32)
        dist.all_reduce(f, op=dist.ReduceOp.MIN)
        room = bool(f.item())
    if not args.no_e2e and not room:
        e2e_note = f"not measured: {cube_bytes / 2**30:.1f} GiB cube, host memory available {_mem_available() / 2**30:.1f} GiB"
    elif not args.no_e2e:
        if obs is None:
            pinned = torch.empty(tuple(obs_d.shape), dtype=torch.float32, pin_memory=True)
            pinned.copy_(obs_d)
        else:
            pinned = torch.from_numpy(obs).pin_memory()
        obs_pinned = pinned.numpy()
        # result arrays in pinned host memory, allocated once (as a host's scan loop would)
        res = {"models": torch.empty((w.npix, 11), dtype=torch.float64, pin_memory=True).numpy(),
               "chisq": torch.empty(w.npix, dtype=torch.float32, pin_memory=True).numpy(),
               "iters": torch.empty(w.npix, dtype=torch.int32, pin_memory=True).numpy()}
        for _ in range(max(1, args.warmup)):
            inv32.invert(obs_pinned, w.guess, slight=sl_h, want_spectra=False, want_status=False, out=res)
        e2e_ms = []
        for _ in range(args.steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            t0 = time.perf_counter()  # wall clock around the public call: copies, kernel, results in host memory
            inv32.invert(obs_pinned, w.guess, slight=sl_h, want_spectra=False, want_status=False, out=res)
            e2e_ms.append((time.perf_counter() - t0) * 1000.0)
        if dist is not None:
            t = torch.tensor([float(np.mean(e2e_ms))], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = [float(t.item())]
        e2e_v = world * w.npix / (float(np.mean(e2e_ms)) / 1000.0)
        del obs_pinned, pinned, res
    h2d = cube_bytes
    d2h = w.npix * (11 * 8 + 4 + 4)

    # plain FP64 forms on the same cube (fewer steps: slower)
    plain = {}
    if not args.no_plain:
        pn = args.plain_npix or (w.npix if w.npix <= (1 << 20) else (1 << 18))
        sub = obs_d[:pn]
        for name, solver in (("fp64_eigen", pm.SOLVE_EIGEN), ("fp64_cholesky", pm.SOLVE_CHOLESKY)):
            with pm.Inverter(w.line, w.lam, w.psf, noise=w.noise, fix=w.fix, nterms=w.nterms,
                             precision=pm.PREC_FP64, solver=solver) as inv:
                step_device(inv, sub)
                t = []
                for _ in range(max(1, min(2, args.steps))):
                    t.append(step_device(inv, sub)[1]["kernel_ms"])
                plain[name] = {"value": pn / (float(np.mean(t)) / 1000.0), "unit": "pixels/s",
                               "ms_per_step": float(np.mean(t)), "pixels": pn}

    # taps per output: every tap for one-warp grids (the reference's direct
    # convolution), the support above 1e-18 of the peak on multi-warp grids
    taps = w.nl if w.nl <= 32 else workloads.psf_support(w.psf)
    fm = flop_model(w.nl, taps, w.nterms, w.psf is not None, w.slight is not None)
    f32, f64 = flops(fm, w.npix * args.steps, iters, acc)
    kernel_s = sum(kms) / 1000.0
    clocks = clk.summary()
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    peak_fp32 = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12  # TFLOP/s, FP32 vector pipe at the sampled clock
    achieved = f32 / kernel_s / 1e12
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    hbm_peak = json.load(open(peaks_path))["hbm_gbs"] if os.path.exists(peaks_path) else 6650.0
    hbm_bytes = w.npix * args.steps * (16 * w.nl + 11 * 8 + 8)
    # DRAM bytes per pixel of the FP32 inversion kernel from one ncu capture of a
    # cube of the same workload, scaled to this launch by its pixel count: 353.9 MB
    # for 524,288 pixels of the 30-point grid (lock-step kernel, 16-warp blocks,
    # dram__bytes_read.sum + dram__bytes_write.sum), 132.7 MB for 65,536 pixels of
    # the 112-point grid
    traffic = {1: 675.0, 4: 2025.0}.get(args.config) if w.nl in (30, 112) else None
    traffic = traffic * w.npix if traffic else None
    roofline = {"bound": "fp32", "achieved": round(achieved, 3), "peak": round(peak_fp32, 2), "unit": "TFLOP/s",
                "frac": round(achieved / peak_fp32, 4), "traffic": traffic,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per pixel, scaled",
                "peak_source": f"148 SMs x 128 FP32 lanes x 2 x sampled SM clock {sm_mhz:.0f} MHz (nominal; no "
                               "measured FP32-pipe peak in MEASURED_PEAKS.json)",
                "flops_per_pixel_fp32": round(f32 / (w.npix * args.steps)),
                "flops_per_pixel_fp64": round(f64 / (w.npix * args.steps)),
                "iterations_per_pixel": iters / (w.npix * args.steps),
                "accepted_per_pixel": acc / (w.npix * args.steps),
                "hbm": {"achieved_gbs": round(hbm_bytes / kernel_s / 1e9, 3), "peak_gbs": hbm_peak,
                        "frac": round(hbm_bytes / kernel_s / 1e9 / hbm_peak, 6)}}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cores = host_cores()
        n = args.cpu_sample or min(w.npix, (1500 if w.nl <= 32 else 200) * cores)
        sample = obs if obs is not None else obs_d[:n].cpu().numpy()
        v, info = cpu_baseline(rw, sample, n, cores)
        cpu = {"value": v, "unit": "pixels/s", "cores": info["cores"], "kind": info["kind"],
               "sample": info["sample"]}

    if rank == 0:
        print(json.dumps({
            "metric": metric, "value": value, "unit": "pixels/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": data_desc(rw, obs is None), "config": cfg_desc,
            "tuning": tuning,
            "e2e": {"value": e2e_v, "unit": "pixels/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    **({"note": e2e_note} if e2e_note else {})},
            "plain": plain, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
            "gpu_launches": launches}), flush=True)
    inv32.close()
    inv64.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
