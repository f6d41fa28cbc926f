"""Builds tests/golden/*.npz from LibAPR's own test fixtures.

Run once in a container that has the LibAPR source tree (default
/root/reference); the .npz files are committed so that tests never read the
reference tree at run time.

Inputs (LibAPR test/files/Apr/<case>/): the original uint16 volume, the
reference pipeline's saved down-sampled gradient (gradient_saved.tif, uint16)
and local intensity scale (scale_saved.tif, float32) that test_pipeline_u16
compares against at tolerance 1 (test/APRTest.cpp:2771-2848), and the
per-pixel level / particle-coordinate / piecewise-constant intensity images
that the iterator tests sample at each particle's nearest pixel
(test/APRTest.cpp:2600-2665).  APR parameters and the particle count come
from the HDF5 attributes of the case's .apr file, read by byte scan (no HDF5
library here).  All TIFFs are uncompressed; width is y (fastest), height is
x, pages are z, as TiffUtils::getMesh maps them.
"""
import os
import re
import struct
import sys

import numpy as np

# the LibAPR source tree: first argument, else $LIBAPR_SRC/.. (LIBAPR_SRC names its src/ directory)
REF = sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.normpath(os.environ["LIBAPR_SRC"]))
OUT = os.path.dirname(os.path.abspath(__file__))

_TYPES = {1: 1, 2: 1, 3: 2, 4: 4, 5: 8, 6: 1, 7: 1, 8: 2, 9: 4, 10: 8, 11: 4, 12: 8, 16: 8}


def read_tiff(path):
    b = open(path, "rb").read()
    e = "<" if b[:2] == b"II" else ">"
    assert struct.unpack_from(e + "H", b, 2)[0] == 42, "not a classic TIFF"
    off = struct.unpack_from(e + "I", b, 4)[0]
    pages = []
    while off:
        n = struct.unpack_from(e + "H", b, off)[0]
        tags = {}
        for k in range(n):
            tag, typ, cnt = struct.unpack_from(e + "HHI", b, off + 2 + 12 * k)
            size = _TYPES[typ] * cnt
            voff = off + 2 + 12 * k + 8
            if size > 4:
                voff = struct.unpack_from(e + "I", b, voff)[0]
            fmt = {1: "B", 3: "H", 4: "I", 6: "b", 8: "h", 9: "i", 11: "f", 12: "d", 16: "Q"}.get(typ)
            tags[tag] = struct.unpack_from(e + fmt * cnt, b, voff) if fmt else None
        width, height = tags[256][0], tags[257][0]
        bits = tags.get(258, (1,))[0]
        assert tags.get(259, (1,))[0] == 1, "compressed TIFF"
        fmt = tags.get(339, (1,))[0]
        dt = {(8, 1): np.uint8, (16, 1): np.uint16, (32, 3): np.float32, (32, 1): np.uint32}[(bits, fmt)]
        raw = b"".join(b[o:o + c] for o, c in zip(tags[273], tags[279]))
        pages.append(np.frombuffer(raw, dtype=np.dtype(dt).newbyteorder(e))[: width * height]
                     .reshape(height, width).astype(dt))
        off = struct.unpack_from(e + "I", b, off + 2 + 12 * n)[0]
    return np.stack(pages)  # (z, x, y)


def apr_attr(b, name, kind):
    m = re.search(re.escape(name.encode()) + b"\x00", b)
    if m is None:
        return None
    pad = (len(name) + 1 + 7) // 8 * 8
    if kind == "f":  # float32 scalar attribute: name, datatype (24 B), dataspace (24 B), value
        return struct.unpack_from("<f", b, m.start() + pad + 48)[0]
    return struct.unpack_from("<Q", b, m.start() + pad + 40)[0]  # uint64 scalar attribute: datatype (16 B), dataspace (24 B), value


CASES = {
    "sphere_diff_dims": ("sphere_original.tif", "sphere.apr", "sphere_"),
    "sphere_120": ("sphere_original.tif", "sphere.apr", "sphere_"),
    "sphere_2D": ("original.tif", "sphere_2D.apr", "sphere_2D_"),
    "sphere_1D": ("original.tif", "sphere_1D.apr", "sphere_1D_"),
}


def main():
    for case, (orig, apr, pre) in CASES.items():
        d = os.path.join(REF, "test", "files", "Apr", case)
        b = open(os.path.join(d, apr), "rb").read()
        arrays = {
            "original": read_tiff(os.path.join(d, orig)),
            "gradient_saved": read_tiff(os.path.join(d, "gradient_saved.tif")),
            "scale_saved": read_tiff(os.path.join(d, "scale_saved.tif")),
        }
        for k in ("level", "x", "y", "z", "pc"):
            arrays["img_" + k] = read_tiff(os.path.join(d, pre + k + ".tif"))
        params = np.array([apr_attr(b, n, "f") or 0.0 for n in
                           ("lambda", "rel_error", "grad_th", "sigma_th", "sigma_th_max")], dtype=np.float32)
        arrays["params"] = params
        arrays["total_number_particles"] = np.array([apr_attr(b, "total_number_particles", "u")], dtype=np.uint64)
        np.savez_compressed(os.path.join(OUT, case + ".npz"), **arrays)
        print(case, {k: (v.shape, v.dtype) for k, v in arrays.items()}, params,
              arrays["total_number_particles"])


if __name__ == "__main__":
    main()
