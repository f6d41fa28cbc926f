"""Benchmark: get_apr (+ particle sampling) on the 2048x2048x512 uint16 volume,
then APR isotropic 3x3x3 and 5x5x5 convolution over its particles.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0.  A step is one get_apr + sample_image pass over one
seeded synthetic volume (background 100, 60000 Gaussian blobs sigma U[2,8] px,
amplitude U[500,6000], Poisson noise; APR parameters lambda=3, E=0.1,
Ip_th=0, sigma_th=50, grad_th=10; ImageType float by default, because with
ImageType uint16 the reference's B-spline overflow check throws on this
volume).  ``value`` is whole-job
GVox/s with the input resident in HBM; ``e2e`` is the same through the
host-buffer C ABI (image host->device and particles device->host inside the
timed region).  Under torchrun every rank converts its own volume (different
seed): the volumes are independent, so scaling is weak and no collective runs
on the data path.  The input (4 GiB) is larger than L2, so no L2 flush is
needed between steps.
"""
import argparse
import ctypes as C
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

SHAPE = (512, 2048, 2048)  # z, x, y
BLOBS = 60000
SIGMA = (2.0, 8.0)
AMP = (500.0, 6000.0)
BG = 100.0
PARAMS = dict(lambda_=3.0, rel_error=0.1, Ip_th=0.0, sigma_th=50.0, grad_th=10.0)
METRIC = "get_apr GVox/s + APR conv Gpart/s vs HBM roofline; RL time-to-1e-3 learned vs plain"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for n, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
            except Exception:
                pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(value, world, device):
    """The slowest rank's time: every rank of a weak-scaling run converts its
    own volume, and the job is as fast as its slowest rank."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def volume_seed(rank):
    """Each rank converts a different seeded volume of the same model."""
    return 1000 + rank


def lib_params():
    import libapr_b200 as A
    p = A.APRParameters()
    for k, v in PARAMS.items():
        setattr(p, k, v)
    return p


SINGLE_KERNEL_STAGES = ("bspline_y", "bspline_x", "bspline_z", "gradient_ds", "inv_bspline", "levels")

# DRAM bytes per full-resolution voxel of one launch, from one ncu capture of
# the 128x1024x1024 case (dram__bytes_read.sum + dram__bytes_write.sum divided
# by its voxels; the traffic grows in proportion to the volume)
TRAFFIC_PER_VOXEL = {
    "gradient_ds": ((537.159424e6 + 120.076288e6) / (128 * 1024 * 1024),
                    "ncu, 128x1024x1024 float capture scaled by voxels "
                    "(profiles/grad_ds_kernel_float_128x1024x1024.md)"),
    "bspline_y": ((468.568e6 + 496.170496e6) / (128 * 1024 * 1024),
                  "ncu, 128x1024x1024 float capture scaled by voxels "
                  "(profiles/iir_tma_kernels_float_128x1024x1024.md)"),
    "bspline_x": ((1019.727e6 + 544.518400e6) / (128 * 1024 * 1024),
                  "ncu, 128x1024x1024 float capture scaled by voxels "
                  "(profiles/iir_tma_kernels_float_128x1024x1024.md)"),
    "bspline_z": ((644.672e6 + 544.285184e6) / (128 * 1024 * 1024),
                  "ncu, 128x1024x1024 float capture scaled by voxels "
                  "(profiles/iir_tma_kernels_float_128x1024x1024.md)"),
}


def algorithmic_bytes(stage, N, Nd, P, T, its=2):
    """Minimum HBM bytes of one launch of a stage (its = bytes per ImageType
    value: 2 for uint16, 4 for float)."""
    return {
        "bspline_y": (2 + its) * N, "bspline_x": 2 * its * N, "bspline_z": 2 * its * N,
        "gradient_ds": its * N + (its + 8) * Nd, "inv_bspline": 8 * Nd, "local_intensity_scale": 8 * Nd,
        "levels": 14 * Nd, "offset": 2 * N, "sample_image": 2 * N + 4 * P,
        "convolve": 10 * P + 10 * T, "fill_tree_mean": 6 * P + 6 * T,
    }.get(stage)


def workload_config(image_type, P, world):
    """The workload description both arms print (the reference arm converts
    the rank-0 volume of the same generator and parameters)."""
    z, x, y = SHAPE
    return {"workload": "get_apr + sample_image, uint16 %dx%dx%d (y,x,z) blob volume, 60000 blobs per "
                        "2048x2048x512, one volume per process" % (y, x, z),
            "image_type": image_type, **PARAMS, "particles": P,
            "l2": "input 4 GiB > L2, no flush needed",
            "parallelism": "independent volume per GPU" if world > 1 else "one volume"}


def cpu_baseline(host_img, image_type):
    """The reference's own CPU get_apr + sample_image (oracle/_ref, Release
    flags -O3 -ffast-math) on the whole volume the GPU converted, all host
    threads, one run."""
    from oracle import bind as B
    if not B.ref_available(fast=True):
        return None
    p = B.make_params(**PARAMS)
    t0 = time.perf_counter()
    e, r = B.ref_get_apr(host_img, p, image_type, staged=False, fast=True)
    if e != 0:
        return {"value": None, "unit": "GVox/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": "reference get_apr failed with status %d" % e}
    r.sample(host_img)
    t = time.perf_counter() - t0
    del r
    return {"value": host_img.size / t / 1e9, "unit": "GVox/s", "cores": os.cpu_count(), "kind": "reference",
            "sample": "get_apr + sample_image on the whole %dx%dx%d volume the GPU converted, one run"
                      % host_img.shape[::-1], "seconds": t}


def parity_full_volume(A, host_img, dev_img, image_type, rel_tol=1e-5):
    """Outside the timed region: the GPU's get_apr on the benchmark volume
    against the reference's own CPU code built with strict IEEE flags
    (oracle/_ref/libaprref.so) on the same bytes -- linear access structure,
    uint16 intensities, the down-sampled level of every cell (a differing
    level is a flip) -- and the number of cells whose level argument lies
    within rel_tol of a level boundary (LocalParticleCellSet.hpp:129-171)."""
    from oracle import bind as B
    if not B.ref_available():
        return {"skipped": "oracle/_ref/libaprref.so not built"}
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = None
    if avail is not None and avail < 40e9:
        return {"skipped": "%.0f GB of host memory available, the reference run needs about 40" % (avail / 1e9)}
    conv = A.APRConverter(image_type)
    conv.par = lib_params()
    conv.keep_intermediates(True)
    apr = A.APR()
    conv.get_apr(apr, dev_img)
    near, active = conv.level_margins(rel_tol)
    z, x, y = host_img.shape
    ds = ((z + 1) // 2, (x + 1) // 2, (y + 1) // 2)
    it = 1 if image_type == "uint16" else 0
    t0 = time.perf_counter()
    e, ref = B.ref_get_apr(host_img, B.make_params(**PARAMS), it, staged=True)
    t_ref = time.perf_counter() - t0
    if e != 0:
        return {"reference_status": e}
    flips = int(np.count_nonzero(conv.intermediate(6, ds) != ref.intermediate(6)))
    acc = ref.access()
    lx, xe, yv = apr.linear_access()
    structure = bool(np.array_equal(lx, acc.level_xz) and np.array_equal(xe, acc.xz_end)
                     and np.array_equal(yv, acc.y_vec))
    del lx, xe, yv
    P = acc.P
    del acc
    parts = A.ParticleData().sample_image(apr, host_img).data
    same_parts = bool(np.array_equal(parts[:P], ref.sample(host_img)[:P]))
    del parts, ref
    apr._free()
    return {"reference": "oracle/_ref/libaprref.so: the reference's get_apr_cpu + sample_image compiled from "
                         "its headers with strict IEEE flags, on the same bytes",
            "structure_equal": structure, "intensities_equal": same_parts, "level_flips": flips,
            "near_threshold_cells": near, "cells_at_level_1_or_more": active, "rel_tol": rel_tol,
            "particles": P, "reference_seconds": t_ref}


def run_reference(args):
    """--impl reference: the reference's own CPU implementation (LibAPR's
    get_apr_cpu + sample_image compiled from its headers at its Release flags,
    oracle/_ref/libaprref_fast.so, OpenMP on every host core) on the rank-0
    volume of the benchmark, rendered on the host by the generator's CPU twin
    (the same bytes the device generator writes); rank 0 only.  Nothing of
    the library is loaded."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
    from oracle import bind as B
    if not B.ref_available(fast=True):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built (needs the LibAPR tree)"}))
        return 0
    t0 = time.perf_counter()
    img = B.blob_volume_cpu(SHAPE, BLOBS, SIGMA, AMP, BG, volume_seed(0))
    t_gen = time.perf_counter() - t0
    p = B.make_params(**PARAMS)
    it = 1 if args.image_type == "uint16" else 0
    times, P = [], None
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        e, r = B.ref_get_apr(img, p, it, staged=False, fast=True)
        if e != 0:
            print(json.dumps({"impl": "reference", "unavailable": "reference get_apr failed with status %d" % e}))
            return 0
        r.sample(img)
        dt = time.perf_counter() - t0
        if P is None:
            P = r.access().P
        del r
        if i >= args.warmup:
            times.append(dt)
    t = sum(times) / len(times)
    v = img.size / t / 1e9
    line = {"metric": METRIC, "value": v, "unit": "GVox/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.image_type == "float" else "u16", "data": "synthetic",
            "config": workload_config(args.image_type, P, 1),
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "GVox/s", "cores": os.cpu_count(), "kind": "reference",
                             "sample": "the whole %dx%dx%d volume per step: LibAPR's CPU get_apr_cpu + "
                                       "sample_image at its Release flags (-O3 -ffast-math), OpenMP on all host "
                                       "cores; volume rendered on the host (%.1f s) by the generator's CPU twin, "
                                       "bit-identical to the device generator" % (SHAPE[2], SHAPE[1], SHAPE[0], t_gen)},
            "e2e": {"value": v, "unit": "GVox/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


BATCH_AXES = (64, 96, 128, 192, 256, 384, 512)


def batch_shapes(n=96, seed=2024):
    """Seeded uneven volumes: every axis from BATCH_AXES, z <= 256, blob
    density uniform in [1e-5, 5e-4] per voxel."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        z = int(rng.choice([a for a in BATCH_AXES if a <= 256]))
        x = int(rng.choice(BATCH_AXES))
        y = int(rng.choice(BATCH_AXES))
        dens = float(rng.uniform(1e-5, 5e-4))
        out.append(((z, x, y), max(1, int(round(dens * z * x * y)))))
    return out


def bench_batch(A, L, _lib, torch, stream, sptr, args):
    """96 volumes through the blocked converter (z tiles of 128 planes, 16 ghost
    planes) in one batch call, beside one whole-volume get_apr per volume."""
    shapes = batch_shapes()
    vols = []
    for i, (shp, nb) in enumerate(shapes):
        t = torch.empty(shp, dtype=torch.int16, device="cuda")
        A.synth_blobs_device(t, nb, SIGMA, AMP, BG, seed=5000 + i, stream=stream)
        vols.append(t)
    torch.cuda.synchronize()
    conv = A.APRConverterBatch("float", z_block_size=128, ghost_z=16)
    conv.par = lib_params()
    plain = A.APRConverter("float")
    plain.par = lib_params()
    nvox = sum(int(v.numel()) for v in vols)
    par = plain.par.c()

    def run_batch():
        aprs = conv.get_apr_batch(vols, stream=stream)
        return sum(a.total_number_particles() for a in aprs)

    def run_plain():
        P = 0
        for v in vols:
            h = C.c_void_p()
            z, x, y = v.shape
            _lib.check(L.aprb_get_apr_device(plain._h, C.byref(par), C.c_void_p(v.data_ptr()), y, x, z, sptr,
                                             C.byref(h)))
            info = _lib.aprb_apr_info()
            L.aprb_apr_get_info(h, C.byref(info))
            P += int(info.total_number_particles)
            L.aprb_apr_free(h)
        return P

    res = {}
    for name, fn in (("batch", run_batch), ("per_volume", run_plain)):
        for _ in range(max(1, args.warmup - 1)):
            fn()
        torch.cuda.synchronize()
        reps = 2
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            P = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        res[name] = {"ms": ms, "value": nvox / (ms / 1e3) / 1e9, "unit": "GVox/s", "particles": P}
    res["volumes"] = len(vols)
    res["voxels"] = nvox
    res["workload"] = ("96 seeded uint16 blob volumes, axes from %s with z <= 256, blob density U[1e-5, 5e-4]; "
                       "batch: blocked converter, z tiles 128 + ghost 16; per_volume: whole-volume get_apr, "
                       "one call per volume; ImageType float" % (BATCH_AXES,))
    del vols
    return res


RL_BLOBS = 20000  # per 256 x 1024 x 1024


def gaussian_psf(sigma=1.2, ks=5):
    g = np.exp(-((np.arange(ks) - ks // 2) ** 2) / (2 * sigma * sigma)).astype(np.float32)
    p = (g[:, None, None] * g[None, :, None] * g[None, None, :]).astype(np.float32)
    return (p / p.sum()).astype(np.float32)


def bench_rl(A, L, _lib, torch, stream, sptr, args):
    """Plain APR Richardson-Lucy on the deconvolution workload: float ground
    truth (background 50, Gaussian blobs sigma U[1,4], amplitude U[500,5000]),
    blurred by the normalised 5x5x5 Gaussian PSF (sigma 1.2), Poisson noise,
    uint16; APR with lambda=3, E=0.1, Ip_th=0, sigma_th=50, grad_th=10.  FP32 RL
    time per iteration, and its relative L2 error after 20/100/500 iterations
    against the FP64 RL (the reference's double instantiation on the GPU, which
    the tests pin bit-exact to the FP64 oracle) after 500 iterations."""
    from libapr_b200 import learned as Lr
    shape = tuple(int(v) for v in args.rl_shape.split(","))
    n = shape[0] * shape[1] * shape[2]
    apr, parts, psf, n_blobs = Lr.deconvolution_workload(shape, seed=3000, stream=stream)
    P = apr.total_number_particles()
    T = apr.total_number_tree_particles()
    pp = C.c_void_p(parts.data_ptr())
    st = C.c_void_p(psf.ctypes.data)
    o32 = torch.empty(max(P, 1), dtype=torch.float32, device="cuda")
    o64 = torch.empty(max(P, 1), dtype=torch.float64, device="cuda")

    def rl32(iters, resume):
        _lib.check(L.aprb_richardson_lucy_device(apr._h, pp, C.c_void_p(o32.data_ptr()), st, 5, iters, 1, 1,
                                                 int(resume), sptr))

    def rl64(iters, resume):
        _lib.check(L.aprb_richardson_lucy_fp64_device(apr._h, pp, C.c_void_p(o64.data_ptr()), st, 5, iters, 1, 1,
                                                      int(resume), sptr))

    def timed(fn, *a):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn(*a)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    rl32(2, False)
    torch.cuda.synchronize()
    L.aprb_profile_reset()
    L.aprb_profile_enable(1)
    ms32 = timed(rl32, 20, False) / 20
    L.aprb_profile_enable(0)
    L.aprb_profile_reset()
    f64 = {}
    ms64 = 0.0
    done = 0
    for kk in (20, 100, 500):
        ms64 += timed(rl64, kk - done, done > 0)
        done = kk
        f64[kk] = o64[:P].clone()
    ref = f64[500]
    rnorm = float(torch.linalg.norm(ref))
    errs, errs_same, k_hit = {}, {}, None
    done = 0
    while done < 500:
        step = 10
        rl32(step, done > 0)
        done += step
        e = float(torch.linalg.norm(o32[:P].double() - ref)) / rnorm
        if k_hit is None and e < 1e-3:
            k_hit = done
        if done in (20, 100, 500):
            errs[done] = e
            errs_same[done] = float(torch.linalg.norm(o32[:P].double() - f64[done])) / float(
                torch.linalg.norm(f64[done]))
    learned = None
    if not args.no_learned and os.path.exists(Lr.WEIGHTS_FILE):
        learned = bench_learned(Lr, torch, apr, parts, psf, ref, rnorm, ms32, k_hit, stream)
    bytes_it = 2 * (10 * P + 10 * T) + 2 * P
    hbm, kind = peaks()
    res = {
        "workload": "deconvolution: %dx%dx%d (z,x,y) blob ground truth (bg 50, %d blobs sigma U[1,4], amp "
                    "U[500,5000]) * normalised 5^3 Gaussian PSF sigma 1.2, Poisson, uint16; APR lambda=3 E=0.1 "
                    "Ip_th=0 sigma_th=50 grad_th=10; PSF as APR stencil, downsampled + normalised"
                    % (shape + (n_blobs,)),
        "particles": P, "tree_nodes": T,
        "fp32_ms_per_iteration": ms32, "fp32_gpart_per_s": P / (ms32 / 1e3) / 1e9,
        "fp64_ms_per_iteration": ms64 / 500,
        "roofline": {"bound": "hbm", "algorithmic_bytes_per_iteration": bytes_it,
                     "achieved": bytes_it / (ms32 / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
                     "frac": bytes_it / (ms32 / 1e3) / 1e9 / hbm, "peak_source": kind},
        "rel_l2_vs_fp64_500": {str(kk): v for kk, v in errs.items()},
        "rel_l2_fp32_vs_fp64_same_iterations": {str(kk): v for kk, v in errs_same.items()},
        "iterations_to_1e-3_of_fp64_500": k_hit,
        "time_to_1e-3_ms": None if k_hit is None else k_hit * ms32,
    }
    if learned is not None:
        res["learned_proposal"] = learned
    del o32, o64, parts, f64, ref
    apr._free()
    return res


def bench_learned(Lr, torch, apr, raw, psf, ref, rnorm, ms_plain, k_plain, stream, budget=600):
    """Learned-proposal RL on the same workload (a seed the network was not
    trained on): device time until the estimate is within 1e-3 relative L2
    of the FP64 500-iteration solution, beside plain RL's."""
    net = Lr.ProposalCNN.load()
    P = raw.numel()
    u = torch.empty(P, dtype=torch.float32, device="cuda")
    # time of one proposal (features + 4 layers + apply): the first call
    # builds the per-particle row table and the bf16 weights, so it is
    # timed apart; the cost a proposal adds inside the run is the mean of
    # the next three calls
    Lr.rl_iterations(apr, raw, u, psf, 10, resume=False, stream=stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    scratch = u.clone()
    e0.record(stream)
    net.propose(apr, raw, scratch, psf, stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_first = e0.elapsed_time(e1)
    ts = []
    for _ in range(3):
        scratch.copy_(u)
        e0.record(stream)
        net.propose(apr, raw, scratch, psf, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    ms_prop = sum(ts) / len(ts)
    del scratch
    acc = Lr.AcceleratedRL(apr, raw, u, psf, net, every=10, warmup=10, stream=stream)
    total_ms, hit_ms, hit_it, best = 0.0, None, None, float("inf")
    while acc.iterations < budget:
        e0.record(stream)
        acc.step()
        e1.record(stream)
        torch.cuda.synchronize()
        total_ms += e0.elapsed_time(e1)
        err = float(torch.linalg.norm(u.double() - ref)) / rnorm
        best = min(best, err)
        if err < 1e-3:
            hit_ms, hit_it = total_ms, acc.iterations
            break
    plain_ms = None if k_plain is None else k_plain * ms_plain
    return {"weights": os.path.relpath(Lr.WEIGHTS_FILE, ROOT),
            "network": "4 layers of per-level 3x3x3 stencils, channels 3-16-16-16-1, bf16 tensor-core operands",
            "proposal_ms": ms_prop, "proposal_first_call_ms": ms_first,
            "plain_rl_ms_per_iteration": ms_plain, "proposals_tried": acc.tried, "proposals_kept": acc.kept,
            "time_to_1e-3_ms": hit_ms, "rl_iterations_to_1e-3": hit_it, "best_rel_l2": best,
            "plain_time_to_1e-3_ms": plain_ms,
            "time_ratio_learned_over_plain": (hit_ms / plain_ms) if (hit_ms and plain_ms) else None}


def run_split(args):
    """--split-volume: one 2048x2048x512 volume's blocked construction (z tiles
    of 128 planes, 16 ghost planes) split by tiles over the ranks
    (libapr_b200.distributed): each rank converts its tiles from its own slab
    of planes, one MAX all-reduce of the particle-cell pyramid over NCCL, and
    every rank builds the volume's structure.  Strong scaling: value = the
    volume's voxels / the slowest rank's device time per step."""
    import datetime

    import torch
    import torch.distributed as dist

    import libapr_b200 as A
    from libapr_b200 import distributed as D
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    shape = tuple(int(v) for v in args.shape.split(",")) if args.shape else SHAPE
    zb, ghost = 128, 16
    img = torch.empty(shape, dtype=torch.int16, device="cuda")
    A.synth_blobs_device(img, int(BLOBS * img.numel() / (SHAPE[0] * SHAPE[1] * SHAPE[2])), SIGMA, AMP, BG,
                         seed=volume_seed(0))
    lo, hi = D.rank_slab(shape[0], zb, ghost, rank, world)
    slab = img[lo:hi].contiguous() if hi > lo else img[:1].contiguous()
    del img
    torch.cuda.synchronize()
    be = D.TileBackend(args.image_type, lib_params())
    for _ in range(args.warmup):
        D.get_apr_by_block_distributed(be, shape, slab, lo, zb, ghost)._free()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    P = 0
    for _ in range(args.steps):
        apr = D.get_apr_by_block_distributed(be, shape, slab, lo, zb, ghost)
        P = apr.total_number_particles()
        apr._free()
    e1.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, "cuda")
    if rank == 0:
        z, x, y = shape
        print(json.dumps({"metric": METRIC, "value": z * x * y / (ms / 1e3) / 1e9, "unit": "GVox/s",
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                          "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                          "dtype": "f32" if args.image_type == "float" else "u16", "data": "synthetic",
                          "config": {"workload": "get_apr by block (z tiles 128, ghost 16) of one uint16 %dx%dx%d "
                                                 "(y,x,z) blob volume split by tiles over the GPUs" % (y, x, z),
                                     "image_type": args.image_type, **PARAMS, "particles": P,
                                     "parallelism": "z-tiles per rank, MAX all-reduce of the pyramid"}}))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--shape", default=None, help="z,x,y override (debugging only)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-conv", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-rl", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--rl-shape", default="256,1024,1024", help="z,x,y of the deconvolution workload")
    ap.add_argument("--split-volume", action="store_true",
                    help="one volume's blocked construction split by z-tiles over the GPUs (strong scaling)")
    ap.add_argument("--image-type", default="float", choices=["float", "uint16"],
                    help="APRConverter ImageType; uint16 throws the reference's overflow error on this volume")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.split_volume:
        return run_split(args)

    import torch
    import torch.distributed as dist
    import libapr_b200 as A
    from libapr_b200 import _lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    shape = tuple(int(v) for v in args.shape.split(",")) if args.shape else SHAPE
    z, x, y = shape
    N = z * x * y
    L = _lib.lib()
    stream = torch.cuda.current_stream()
    sptr = C.c_void_p(stream.cuda_stream)

    img = torch.empty(shape, dtype=torch.int16, device="cuda")
    A.synth_blobs_device(img, int(BLOBS * N / (SHAPE[0] * SHAPE[1] * SHAPE[2])), SIGMA, AMP, BG,
                         seed=volume_seed(rank), stream=stream)
    torch.cuda.synchronize()
    conv = A.APRConverter(args.image_type)
    par = lib_params().c()
    it_code = 1 if args.image_type == "uint16" else 0
    iptr = C.c_void_p(img.data_ptr())

    def get_apr_dev():
        h = C.c_void_p()
        _lib.check(L.aprb_get_apr_device(conv._h, C.byref(par), iptr, y, x, z, sptr, C.byref(h)))
        return h

    # learn P, allocate particle output
    h0 = get_apr_dev()
    info = _lib.aprb_apr_info()
    _lib.check(L.aprb_apr_get_info(h0, C.byref(info)))
    P = int(info.total_number_particles)
    parts = torch.empty(max(P, 1), dtype=torch.int16, device="cuda")
    pptr = C.c_void_p(parts.data_ptr())
    L.aprb_apr_free(h0)

    def step(keep):
        # one APR alive at a time, as a converter loop over a stream of volumes
        h = get_apr_dev()
        _lib.check(L.aprb_sample_image_device(h, iptr, pptr, sptr))
        while keep:
            L.aprb_apr_free(keep.pop())
        keep.append(h)

    hs = []
    for _ in range(args.warmup):
        step(hs)
    torch.cuda.synchronize()
    for h in hs:
        L.aprb_apr_free(h)
    hs = []

    clocks = Clocks(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    L.aprb_profile_reset()
    L.aprb_profile_enable(1)
    launches0 = L.aprb_kernel_launch_count()
    if rank == 0:
        clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step(hs)
    ev1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ck = clocks.stop() if rank == 0 else None
    launches = L.aprb_kernel_launch_count() - launches0
    L.aprb_profile_enable(0)
    ms = ev0.elapsed_time(ev1) / args.steps
    names = (C.c_char_p * 64)()
    tms = (C.c_double * 64)()
    cnts = (C.c_uint64 * 64)()
    ns = L.aprb_profile_read(names, tms, cnts, 64)
    stages = {names[i].decode(): (tms[i], int(cnts[i])) for i in range(ns)}
    L.aprb_profile_reset()
    ms_all = max_over_ranks(ms, world, "cuda")
    last = hs[-1]
    for h in hs[:-1]:
        L.aprb_apr_free(h)

    Nd = ((z + 1) // 2) * ((x + 1) // 2) * ((y + 1) // 2)
    hbm, peak_kind = peaks()
    out = {}
    if rank == 0:
        # dominant stage and its roofline (algorithmic bytes / mean launch time)
        # the dominant single-kernel stage (the local intensity scale stage is
        # seven kernels and the pulling scheme dozens; they are reported per stage)
        single = {k: v for k, v in stages.items() if k in SINGLE_KERNEL_STAGES}
        dom = max((single or stages).items(), key=lambda kv: kv[1][0])
        dname, (dms, dcnt) = dom
        per = dms / dcnt / 1e3
        ab = algorithmic_bytes(dname, N, Nd, P, 0, 2 if it_code == 1 else 4)
        achieved = ab / per / 1e9 if ab else None
        tr = TRAFFIC_PER_VOXEL.get(dname)
        out["roofline"] = {"bound": "hbm", "kernel": dname, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                           "frac": achieved / hbm if achieved else None,
                           "traffic": tr[0] * N if tr else None, "traffic_source": tr[1] if tr else None,
                           "peak_source": peak_kind, "algorithmic_bytes_per_launch": ab,
                           "launch_ms": per * 1e3}
        pipe_b = (10 if it_code == 1 else 14) * N + 4 * P
        out["pipeline_roofline"] = {"algorithmic_bytes": pipe_b, "achieved_gbs": pipe_b / (ms_all / 1e3) / 1e9,
                                    "frac": pipe_b / (ms_all / 1e3) / 1e9 / hbm}
        out["stages_ms_per_step"] = {k: v[0] / args.steps for k, v in stages.items()}

    # --- end to end through the host-buffer C ABI, on every rank (before the
    # other workloads, as a process that converts a stream of volumes runs it)
    e2e = None
    host = torch.empty(shape, dtype=torch.int16, pin_memory=True)
    host.copy_(img)
    hparts = torch.empty(max(P, 1), dtype=torch.int16, pin_memory=True)
    hp = C.c_void_p(host.data_ptr())
    hpp = C.c_void_p(hparts.data_ptr())

    def e2e_step():
        h = C.c_void_p()
        _lib.check(L.aprb_get_apr(conv._h, C.byref(par), hp, y, x, z, C.byref(h)))
        _lib.check(L.aprb_sample_image(h, hp, hpp))
        L.aprb_apr_free(h)

    # the image goes to the GPU once per step: get_apr hands its device copy
    # to the APR and sample_image of the same host buffer uses it
    _lib.check(L.aprb_converter_keep_input(conv._h, 1))
    e2e_step()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize()
    te1 = max_over_ranks((time.perf_counter() - t0) / args.steps, world, "cuda")
    _lib.check(L.aprb_converter_keep_input(conv._h, 0))

    # Two volumes in flight: a second converter on a second host thread, each
    # thread taking every other step (get_apr + sample_image of one volume).
    # The library lets one host-buffer upload at a time cross PCIe, so the
    # uploads run back to back while the other volume's construction,
    # sampling and particle download proceed (PCIe carries both directions at
    # once).  Every step still moves its own image up and its own particles
    # down inside the timed region.
    import threading
    conv2 = A.APRConverter(args.image_type)
    hparts2 = torch.empty(max(P, 1), dtype=torch.int16, pin_memory=True)
    outs = [hpp, C.c_void_p(hparts2.data_ptr())]
    convs = [conv, conv2]
    for cv in convs:
        _lib.check(L.aprb_converter_keep_input(cv._h, 1))

    def worker(i, count, errs):
        try:
            torch.cuda.set_device(local)
            for _ in range(count):
                h = C.c_void_p()
                _lib.check(L.aprb_get_apr(convs[i]._h, C.byref(par), hp, y, x, z, C.byref(h)))
                _lib.check(L.aprb_sample_image(h, hp, outs[i]))
                L.aprb_apr_free(h)
        except Exception as e:  # noqa: BLE001 -- reported after the join
            errs.append(e)

    def run_pair(counts):
        errs = []
        ths = [threading.Thread(target=worker, args=(i, counts[i], errs)) for i in range(2)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        if errs:
            raise errs[0]

    run_pair([1, 1])  # each thread's first call sets up its streams and scratch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    run_pair([(args.steps + 1) // 2, args.steps // 2])
    torch.cuda.synchronize()
    te = max_over_ranks((time.perf_counter() - t0) / args.steps, world, "cuda")
    for cv in convs:
        _lib.check(L.aprb_converter_keep_input(cv._h, 0))
    del conv2
    e2e = {"value": N * world / te / 1e9, "unit": "GVox/s", "h2d_bytes_per_step": 2 * N,
           "d2h_bytes_per_step": 2 * P, "ms_per_step": te * 1e3,
           "one_volume_in_flight": {"value": N * world / te1 / 1e9, "ms_per_step": te1 * 1e3},
           "note": "aprb_get_apr + aprb_sample_image on pinned host buffers, converter keep_input on (the "
                   "image crosses PCIe once per step, in z-chunks overlapped with smoothing; the particles "
                   "come back once); two converters on two host threads take alternate steps, the uploads "
                   "in turn, so one volume's construction and download overlap the next one's upload; "
                   "one_volume_in_flight: the same calls on one thread"}
    # --- convolution over the particles of the last step (float intensities)
    conv_res = {}
    if not args.no_conv:
        pf = parts[:P].to(torch.int32).bitwise_and(0xFFFF).to(torch.float32).contiguous()
        outp = torch.empty_like(pf)
        _lib.check(L.aprb_apr_init_tree(last))
        _lib.check(L.aprb_apr_get_info(last, C.byref(info)))
        T = int(info.tree_total_number_particles)
        rng = np.random.default_rng(7)
        # FP32 FMA peak of this GPU, measured (the measured-peaks file has none)
        fp32_peak = C.c_double(0.0)
        _lib.check(L.aprb_measure_fp32_fma_peak(sptr, C.byref(fp32_peak)))
        for ks in (3, 5):
            st = rng.uniform(-1, 1, ks ** 3).astype(np.float32)
            st = (st / st.sum()).astype(np.float32)
            stp = C.c_void_p(st.ctypes.data)

            def run_conv():
                _lib.check(L.aprb_convolve_device(last, stp, ks, C.c_void_p(pf.data_ptr()),
                                                  C.c_void_p(outp.data_ptr()), 1, 1, 0, sptr))

            for _ in range(2):
                run_conv()
            torch.cuda.synchronize()
            L.aprb_profile_reset()
            L.aprb_profile_enable(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            reps = max(2, args.steps)
            e0.record(stream)
            for _ in range(reps):
                run_conv()
            e1.record(stream)
            torch.cuda.synchronize()
            L.aprb_profile_enable(0)
            cn = (C.c_char_p * 64)()
            ct = (C.c_double * 64)()
            cc = (C.c_uint64 * 64)()
            nst = L.aprb_profile_read(cn, ct, cc, 64)
            cstages = {cn[i].decode(): ct[i] / reps for i in range(nst)}
            L.aprb_profile_reset()
            cms = e0.elapsed_time(e1) / reps
            ab = 10 * P + 10 * T
            flops = 2 * (ks ** 3) * P
            conv_res["conv%d%d%d" % (ks, ks, ks)] = {
                "value": P / (cms / 1e3) / 1e9, "unit": "Gpart/s", "ms": cms, "particles": P, "tree_nodes": T,
                "roofline": {"bound": "hbm", "achieved": ab / (cms / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
                             "frac": ab / (cms / 1e3) / 1e9 / hbm, "algorithmic_bytes": ab},
                "gflops": flops / (cms / 1e3) / 1e9, "stages_ms": cstages,
                "fp32": {"achieved_tflops": flops / (cms / 1e3) / 1e12, "peak_tflops": fp32_peak.value,
                         "frac": flops / (cms / 1e3) / 1e12 / fp32_peak.value if fp32_peak.value else None,
                         "peak_source": "measured here: independent FP32 FMA chains (aprb_measure_fp32_fma_peak)",
                         "note": "2 ks^3 flops per particle; the bit-exact taps are a separate multiply "
                                 "and add, so 0.5 is the ceiling of this fraction"}}
        # gradient magnitude on the particles (APRNumerics::gradient_magnitude_cfd
        # and _sobel): three directional 3x3x3 convolutions, squares and a root
        deltas = (C.c_float * 3)(1.0, 1.0, 1.0)
        for sobel in (0, 1):
            def run_grad():
                _lib.check(L.aprb_gradient_magnitude_device(last, C.c_void_p(pf.data_ptr()),
                                                            C.c_void_p(outp.data_ptr()), deltas, sobel, sptr))

            for _ in range(2):
                run_grad()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            reps = max(2, args.steps)
            e0.record(stream)
            for _ in range(reps):
                run_grad()
            e1.record(stream)
            torch.cuda.synchronize()
            gms = e0.elapsed_time(e1) / reps
            ab = 3 * (10 * P + 10 * T)
            conv_res["gradient_magnitude_sobel" if sobel else "gradient_magnitude_cfd"] = {
                "value": P / (gms / 1e3) / 1e9, "unit": "Gpart/s", "ms": gms,
                "roofline": {"bound": "hbm", "achieved": ab / (gms / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
                             "frac": ab / (gms / 1e3) / 1e9 / hbm, "algorithmic_bytes": ab,
                             "note": "three directional convolutions at 10P + 10T each"}}
        del pf, outp
        # piecewise-constant reconstruction of the volume from its particles
        # (reconstruct_constant): writes every pixel once
        rimg = torch.empty(N, dtype=torch.int16, device="cuda")

        def run_recon():
            _lib.check(L.aprb_reconstruct_constant_u16_device(last, C.c_void_p(parts.data_ptr()),
                                                              C.c_void_p(rimg.data_ptr()), sptr))

        for _ in range(2):
            run_recon()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = max(2, args.steps)
        e0.record(stream)
        for _ in range(reps):
            run_recon()
        e1.record(stream)
        torch.cuda.synchronize()
        rms = e0.elapsed_time(e1) / reps
        ab = 2 * N + 4 * P
        conv_res["reconstruct_constant"] = {
            "value": N / (rms / 1e3) / 1e9, "unit": "GVox/s", "ms": rms,
            "roofline": {"bound": "hbm", "achieved": ab / (rms / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
                         "frac": ab / (rms / 1e3) / 1e9 / hbm, "algorithmic_bytes": ab}}
        del rimg
    L.aprb_apr_free(last)

    # automatic parameters (autoParametersLiEntropy before applyParameters):
    # the same get_apr with par.auto_parameters on, the step's stage time
    auto_res = None
    if rank == 0 and not args.no_conv:
        par_auto = lib_params().c()
        par_auto.auto_parameters = 1

        def get_apr_auto():
            h = C.c_void_p()
            _lib.check(L.aprb_get_apr_device(conv._h, C.byref(par_auto), iptr, y, x, z, sptr, C.byref(h)))
            return h

        L.aprb_apr_free(get_apr_auto())
        torch.cuda.synchronize()
        L.aprb_profile_reset()
        L.aprb_profile_enable(1)
        reps = max(2, args.steps)
        for _ in range(reps):
            ha = get_apr_auto()
            used = _lib.aprb_params()
            _lib.check(L.aprb_apr_get_parameters(ha, C.byref(used)))
            L.aprb_apr_free(ha)
        torch.cuda.synchronize()
        L.aprb_profile_enable(0)
        an = (C.c_char_p * 64)()
        at = (C.c_double * 64)()
        ac = (C.c_uint64 * 64)()
        na = L.aprb_profile_read(an, at, ac, 64)
        astages = {an[i].decode(): at[i] / reps for i in range(na)}
        L.aprb_profile_reset()
        ams = astages.get("auto_parameters")
        auto_res = {"ms": ams, "ds_cells": Nd, "ds_cells_per_s": Nd / (ams / 1e3) if ams else None,
                    "grad_th": used.grad_th, "sigma_th": used.sigma_th,
                    "note": "foreground count + scan + subsample + Li steps (host round trip per step)"}

    # the batch and deconvolution workloads are single-GPU measurements
    batch_res = None
    if not args.no_batch and world == 1:
        batch_res = bench_batch(A, L, _lib, torch, stream, sptr, args)
    rl_res = None
    if not args.no_rl and world == 1:
        rl_res = bench_rl(A, L, _lib, torch, stream, sptr, args)

    cpu, parity = None, None
    if not args.no_cpu and world == 1 and shape == SHAPE:
        hv = host.numpy().view(np.uint16)
        parity = parity_full_volume(A, hv, img, args.image_type)
        cpu = cpu_baseline(hv, it_code)
    if rank == 0:
        line = {"metric": METRIC, "value": N * world / (ms_all / 1e3) / 1e9, "unit": "GVox/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_all, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32" if it_code == 0 else "u16",
                "data": "synthetic",
                "config": workload_config(args.image_type, P, world),
                "gpu_launches": int(launches), "e2e": e2e, "cpu_baseline": cpu, **out, **conv_res}
        line["smoothing_schedule"] = {"variants": A.smoothing_schedule(),
                                      "source": "libapr_b200/data/smoothing_schedule.json (libapr_b200.autotune)"}
        if parity:
            line["parity"] = parity
        if auto_res:
            line["auto_parameters"] = auto_res
        if batch_res:
            line["batch_by_block"] = batch_res
        if rl_res:
            line["rl_deconvolution"] = rl_res
        if ck:
            line["clocks"] = ck
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
