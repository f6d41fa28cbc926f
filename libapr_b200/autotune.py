"""Autotuner of the smoothing schedule: for every axis of the recursive
B-spline smoothing (bspline_filt_rec_y/x/z, ComputeGradient.hpp:249-779) and
every line-length bucket (n <= 128, 256, 512, 1024, 2048, longer), times each
kernel variant of the library on the current GPU -- the pass's own stage time
from the library's CUDA-event stage timer, median of a few get_apr calls on a
seeded synthetic volume of about 2^29 voxels whose lines along that axis have
the bucket's length -- and writes the fastest variant per (axis, bucket) with
all timings to a JSON file, which the package applies when it loads the
library.  Every variant computes the same bits, so the schedule changes only
the speed.

    python -m libapr_b200.autotune [--out libapr_b200/data/smoothing_schedule.json] [--reps 3]
"""
import argparse
import ctypes as C
import json
import os
import statistics
import time

from . import _lib

LENGTHS = (128, 256, 512, 1024, 2048, 4096)  # one line length per bucket
STAGE = {"y": "bspline_y", "x": "bspline_x", "z": "bspline_z"}
TARGET = 1 << 29  # voxels of a timing volume


def timing_shape(axis, n):
    """(z, x, y) with lines of length n along the axis and about TARGET voxels;
    y_num stays 1024 for the x / z axes (a multiple of 4, >= 256: TMA layouts)."""
    other = max(16, TARGET // (n * 1024))
    if axis == "y":
        return (other, 1024, n)
    if axis == "x":
        return (other, n, 1024)
    return (n, other, 1024)


def stage_ms(A, L, conv, par, img, stage, reps, stream):
    z, x, y = img.shape
    sp = C.c_void_p(stream.cuda_stream)
    h = C.c_void_p()
    _lib.check(L.aprb_get_apr_device(conv._h, C.byref(par), C.c_void_p(img.data_ptr()), y, x, z, sp, C.byref(h)))
    L.aprb_apr_free(h)
    ts = []
    for _ in range(reps):
        L.aprb_profile_reset()
        L.aprb_profile_enable(1)
        h = C.c_void_p()
        _lib.check(L.aprb_get_apr_device(conv._h, C.byref(par), C.c_void_p(img.data_ptr()), y, x, z, sp,
                                         C.byref(h)))
        L.aprb_apr_free(h)
        stream.synchronize()
        L.aprb_profile_enable(0)
        names = (C.c_char_p * 64)()
        tms = (C.c_double * 64)()
        cnts = (C.c_uint64 * 64)()
        ns = L.aprb_profile_read(names, tms, cnts, 64)
        got = {names[i].decode(): tms[i] for i in range(ns)}
        ts.append(got.get(stage, float("nan")))
    L.aprb_profile_reset()
    return statistics.median(ts)


def tune(reps=3, log=print):
    import torch

    import libapr_b200 as A
    L = _lib.lib()
    stream = torch.cuda.current_stream()
    conv = A.APRConverter("float")
    p = A.APRParameters()
    for k, v in dict(lambda_=3.0, rel_error=0.1, Ip_th=0.0, sigma_th=50.0, grad_th=10.0).items():
        setattr(p, k, v)
    par = p.c()
    variants = A.smoothing_variants()
    schedule = A.smoothing_schedule()
    timings = {}
    for axis in ("y", "x", "z"):
        for b, n in enumerate(LENGTHS):
            shape = timing_shape(axis, n)
            img = torch.empty(shape, dtype=torch.int16, device="cuda")
            A.synth_blobs_device(img, max(1, shape[0] * shape[1] * shape[2] // 35000), (2.0, 8.0), (500.0, 6000.0),
                                 100.0, seed=77 + b)
            res = {}
            for v in range(variants[axis]):
                row = list(schedule[axis])
                row[b] = v
                A.set_smoothing_schedule({axis: row})
                res[v] = stage_ms(A, L, conv, par, img, STAGE[axis], reps, stream)
            best = min(res, key=lambda k: res[k])
            schedule[axis][b] = best
            A.set_smoothing_schedule({axis: schedule[axis]})
            timings["%s/%d" % (axis, n)] = {"shape_zxy": list(shape), "ms": {str(k): v for k, v in res.items()},
                                            "best": best}
            log("%s n=%d %s -> variant %d" % (axis, n, {k: round(v, 3) for k, v in res.items()}, best))
            del img
    return schedule, timings


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=_lib.SCHEDULE_FILE)
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args()
    import torch
    t0 = time.time()
    schedule, timings = tune(args.reps)
    doc = {"device": torch.cuda.get_device_name(0), "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
           "seconds": round(time.time() - t0, 1),
           "buckets": "line length n <= 128, 256, 512, 1024, 2048, longer",
           "variants": {"y": "0 cp.async tiles, 1 TMA 2 stages, 2 TMA 3 stages",
                        "x/z": "0 register lines, 1 TMA (1 box, 2 lines, 4 stages), 2 (2, 4, 3), 3 (1, 1, 4), "
                               "4 (2, 2, 3)"},
           "schedule": schedule, "timings": timings}
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    with open(args.out, "w") as f:
        json.dump(doc, f, indent=1)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
