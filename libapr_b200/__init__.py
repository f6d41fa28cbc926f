"""libapr_b200 -- B200-native APR construction and filtering.

Python mirror of LibAPR's interface for the hot path, over the C ABI of
libaprb200.so (include/aprb200.h):

* ``APRParameters``            -- src/algorithm/APRParameters.hpp:11-50
* ``APRConverter(image_type)`` -- src/algorithm/APRConverter.hpp:35-134;
  ``get_apr(apr, img)`` returns False on a failed dimension check and raises
  ``ValueError`` on uint16 smoothing overflow (the reference throws
  std::invalid_argument, ComputeGradient.hpp:409-412)
* ``APR``                      -- src/data_structures/APR/APR.hpp (linear access)
* ``ParticleData``             -- sample_image (ParticleData.hpp:123-127)
* ``APRTreeNumerics.fill_tree_mean`` (APRTreeNumerics.hpp:63-203)
* ``APRFilter.convolve_pencil`` (APRFilter.hpp:139-149) and
  ``isotropic_convolve_333/555`` (APRIsoConvGPU333/555.hpp)
* ``APRNumerics.richardson_lucy`` (APRNumerics.hpp:576-593); stencils other
  than 3^3 / 5^3 raise RuntimeError as in APRNumericsGPU.cu:201-203
* ``APRStencil.create_gaussian_filter`` (APRStencil.hpp:174-228)

Images are numpy arrays of shape (z, x, y) (C order, y fastest: the
reference's PixelData order) on the host, or CUDA tensors of the same layout
(torch) for the device entry points.  All computation runs on the GPU; there
is no CPU fallback.
"""
import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import APRBError, check, lib

__all__ = ["APRParameters", "APRConverter", "APR", "ParticleData", "APRFilter", "APRNumerics", "APRTreeNumerics",
           "APRStencil", "APRBError", "isotropic_convolve_333", "isotropic_convolve_555"]


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


def _dptr(t):
    """Device pointer of a CUDA tensor-like object (torch.Tensor)."""
    return C.c_void_p(int(t.data_ptr()))


def _stream(stream):
    if stream is None:
        return None
    return C.c_void_p(int(getattr(stream, "cuda_stream", stream)))


class APRParameters:
    """APRParameters (src/algorithm/APRParameters.hpp:11-50).  ``lambda`` is a
    Python keyword: use ``par.lambda_`` or ``setattr(par, 'lambda', v)``."""

    _FIELDS = ("dx", "dy", "dz", "psfx", "psfy", "psfz", "Ip_th", "lambda_", "rel_error", "sigma_th",
               "sigma_th_max", "grad_th", "reflect_bc_lis", "neighborhood_optimization", "constant_intensity_scale",
               "check_input", "swap_dimensions", "auto_parameters")
    _FLAGS = ("reflect_bc_lis", "neighborhood_optimization", "constant_intensity_scale", "check_input",
              "swap_dimensions", "auto_parameters")

    def __init__(self, **kw):
        p = _lib.aprb_params()
        lib().aprb_default_params(C.byref(p))
        for f in self._FIELDS:
            v = getattr(p, f)
            object.__setattr__(self, f, bool(v) if f in self._FLAGS else float(v))
        for k, v in kw.items():
            setattr(self, k, v)

    def __setattr__(self, k, v):
        if k == "lambda":
            k = "lambda_"
        if k not in self._FIELDS:
            raise AttributeError("APRParameters has no field %r" % k)
        object.__setattr__(self, k, v)

    def __getattr__(self, k):
        if k == "lambda":
            return self.lambda_
        raise AttributeError(k)

    def c(self):
        p = _lib.aprb_params()
        for f in self._FIELDS:
            setattr(p, f, getattr(self, f))
        return p

    @classmethod
    def _from_c(cls, p):
        par = cls()
        for f in cls._FIELDS:
            v = getattr(p, f)
            object.__setattr__(par, f, bool(v) if f in cls._FLAGS else float(v))
        return par


class APR:
    """An APR: the linear access structure, resident on the GPU."""

    def __init__(self):
        self._h = None
        self._info = None

    def _set(self, h):
        self._free()
        self._h = C.c_void_p(h) if not isinstance(h, C.c_void_p) else h
        self._info = None

    def _free(self):
        if self._h is not None and self._h.value:
            lib().aprb_apr_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self._free()
        except Exception:
            pass

    @classmethod
    def from_arrays(cls, shape_zxy, level_xz, xz_end, y_vec):
        z, x, y = shape_zxy
        lx = np.ascontiguousarray(level_xz, np.uint64)
        xe = np.ascontiguousarray(xz_end, np.uint64)
        yv = np.ascontiguousarray(y_vec, np.uint16)
        h = C.c_void_p()
        check(lib().aprb_apr_from_arrays(y, x, z, _ptr(lx), len(lx), _ptr(xe), len(xe),
                                         _ptr(yv) if len(yv) else None, int(xe[-1]), C.byref(h)))
        a = cls()
        a._set(h)
        return a

    def info(self):
        if self._info is None or not self._info.tree_n_xz:
            i = _lib.aprb_apr_info()
            check(lib().aprb_apr_get_info(self._h, C.byref(i)))
            self._info = i
        return self._info

    def level_min(self):
        return self.info().l_min

    def level_max(self):
        return self.info().l_max

    def total_number_particles(self):
        return int(self.info().total_number_particles)

    def org_dims(self, d):
        return self.info().org_dims[d]

    def y_num(self, l):
        return self.info().y_num[l]

    def x_num(self, l):
        return self.info().x_num[l]

    def z_num(self, l):
        return self.info().z_num[l]

    def bspline_offset(self):
        return float(self.info().bspline_offset)

    def get_apr_parameters(self):
        """APR::get_apr_parameters (APR.hpp:99-101): the parameters the APR was
        built with, grad_th / sigma_th as the automatic parameters chose them."""
        p = _lib.aprb_params()
        check(lib().aprb_apr_get_parameters(self._h, C.byref(p)))
        return APRParameters._from_c(p)

    def linear_access(self):
        """(level_xz, xz_end, y_vec) numpy copies of LinearAccess (LinearAccess.hpp:33-35)."""
        i = self.info()
        lx = np.zeros(i.n_level_xz, np.uint64)
        xe = np.zeros(i.n_xz, np.uint64)
        yv = np.zeros(max(i.total_number_particles, 1), np.uint16)
        check(lib().aprb_apr_export(self._h, _ptr(lx), _ptr(xe), _ptr(yv)))
        return lx, xe, yv[: i.total_number_particles]

    def init_tree(self):
        check(lib().aprb_apr_init_tree(self._h))
        self._info = None

    def tree_access(self):
        self.init_tree()
        i = self.info()
        lx = np.zeros(i.tree_n_level_xz, np.uint64)
        xe = np.zeros(i.tree_n_xz, np.uint64)
        yv = np.zeros(max(i.tree_total_number_particles, 1), np.uint16)
        check(lib().aprb_apr_export_tree(self._h, _ptr(lx), _ptr(xe), _ptr(yv)))
        return lx, xe, yv[: i.tree_total_number_particles]

    def total_number_tree_particles(self):
        self.init_tree()
        return int(self.info().tree_total_number_particles)


class APRConverter:
    """APRConverter<ImageType> (src/algorithm/APRConverter.hpp:35-134)."""

    def __init__(self, image_type="uint16"):
        it = {"uint16": 1, "uint16_t": 1, np.uint16: 1, "float": 0, "float32": 0, np.float32: 0}[image_type]
        self.image_type = it
        self.par = APRParameters()
        h = C.c_void_p()
        check(lib().aprb_converter_create(it, C.byref(h)))
        self._h = h
        self.bspline_offset = 0.0

    def __del__(self):
        try:
            if self._h is not None:
                lib().aprb_converter_destroy(self._h)
        except Exception:
            pass

    def keep_intermediates(self, keep=True):
        check(lib().aprb_converter_keep_intermediates(self._h, int(keep)))

    def _finish(self, st, h, apr):
        if st == 2:  # dimension check failed: the reference returns false
            return False
        if st == 3:
            raise ValueError(lib().aprb_last_error().decode())
        check(st)
        apr._set(h)
        self.bspline_offset = apr.bspline_offset()
        if self.par.auto_parameters:  # autoParametersLiEntropy writes the converter's par (APRConverter.hpp:558)
            used = apr.get_apr_parameters()
            self.par.grad_th, self.par.sigma_th = used.grad_th, used.sigma_th
        return True

    def get_apr(self, apr, img):
        """APRConverter::get_apr (APRConverter.hpp:591-600): img is a (z, x, y)
        uint16 numpy array, or a CUDA tensor for the device path."""
        p = self.par.c()
        h = C.c_void_p()
        if hasattr(img, "data_ptr"):
            z, x, y = img.shape
            st = lib().aprb_get_apr_device(self._h, C.byref(p), _dptr(img), y, x, z, None, C.byref(h))
        else:
            a = np.ascontiguousarray(img, np.uint16)
            z, x, y = a.shape
            st = lib().aprb_get_apr(self._h, C.byref(p), _ptr(a), y, x, z, C.byref(h))
        return self._finish(st, h, apr)

    def keep_input(self, keep=True):
        """Host-buffer get_apr hands its device copy of the image to the APR, and
        the next sample_image of that APR from the same numpy array samples it
        without a second upload (the array must not change in between)."""
        check(lib().aprb_converter_keep_input(self._h, int(keep)))

    def intermediate(self, stage, shape_zxy):
        """Copy of one APRB_STAGE_* buffer of the last get_apr (needs keep_intermediates)."""
        out = np.zeros(shape_zxy, np.float32)
        check(lib().aprb_converter_intermediate(self._h, int(stage), _ptr(out), out.size))
        return out

    def level_margins(self, rel_tol=1e-5):
        """(near_boundary, active) of the last get_apr (needs keep_intermediates):
        down-sampled cells whose level argument (grad / scale) * 2^l_max *
        min(dx, dy, dz) / E lies within rel_tol of a power of two (where a level
        decision of computeLevels, LocalParticleCellSet.hpp:129-171, can flip
        under a relative error rel_tol), and cells whose argument is >= 1."""
        n, a = C.c_uint64(), C.c_uint64()
        check(lib().aprb_converter_level_margins(self._h, float(rel_tol), C.byref(n), C.byref(a)))
        return int(n.value), int(a.value)


class APRConverterBatch(APRConverter):
    """APRConverterBatch<ImageType> (src/algorithm/APRConverterBatch.hpp:32-98):
    the pipeline per z-tile of ``z_block_size`` planes with ``ghost_z`` planes
    of overlap, then one pulling scheme for the volume.  The reference reads
    the tiles from ``par.input_dir + par.input_image_name`` (a TIFF file);
    here ``get_apr(apr, img)`` takes the volume (numpy (z, x, y) uint16 array or
    a CUDA tensor)."""

    def __init__(self, image_type="uint16", z_block_size=128, ghost_z=32):
        super().__init__(image_type)
        self.z_block_size = z_block_size
        self.ghost_z = ghost_z

    def get_apr(self, apr, img):
        p = self.par.c()
        h = C.c_void_p()
        if hasattr(img, "data_ptr"):
            z, x, y = img.shape
            st = lib().aprb_get_apr_by_block_device(self._h, C.byref(p), _dptr(img), y, x, z, self.z_block_size,
                                                    self.ghost_z, None, C.byref(h))
        else:
            a = np.ascontiguousarray(img, np.uint16)
            z, x, y = a.shape
            st = lib().aprb_get_apr_by_block(self._h, C.byref(p), _ptr(a), y, x, z, self.z_block_size, self.ghost_z,
                                             C.byref(h))
        return self._finish(st, h, apr)

    def get_apr_batch(self, imgs, stream=None):
        """Blocked get_apr of many device volumes (CUDA tensors (z, x, y)) in one
        call; returns the list of APRs."""
        p = self.par.c()
        n = len(imgs)
        vols = (_lib.aprb_volume * max(n, 1))()
        for i, t in enumerate(imgs):
            z, x, y = t.shape
            vols[i] = _lib.aprb_volume(_dptr(t), y, x, z)
        outs = (C.c_void_p * max(n, 1))()
        sp = None if stream is None else C.c_void_p(stream.cuda_stream)
        check(lib().aprb_get_apr_batch_device(self._h, C.byref(p), n, vols, self.z_block_size, self.ghost_z, sp,
                                              outs))
        res = []
        for i in range(n):
            a = APR()
            a._set(C.c_void_p(outs[i]))
            res.append(a)
        return res


class ParticleData:
    """ParticleData<T> (ParticleData.hpp:26-218): ``data`` is a numpy array."""

    def __init__(self, data=None):
        self.data = data

    def __len__(self):
        return 0 if self.data is None else len(self.data)

    def sample_parts_from_img_blocked(self, apr, img, z_block_size=256, ghost_z=32):
        """sample_parts_from_img_blocked (ParticleData.hpp:140-142): tiles of the
        in-memory volume instead of a TIFF file."""
        a = np.ascontiguousarray(img, np.uint16)
        out = np.zeros(max(apr.total_number_particles(), 1), np.uint16)
        check(lib().aprb_sample_image_by_block(apr._h, _ptr(a), z_block_size, ghost_z, _ptr(out)))
        self.data = out[: apr.total_number_particles()]
        return self

    def sample_image(self, apr, img):
        a = np.ascontiguousarray(img, np.uint16)
        out = np.zeros(max(apr.total_number_particles(), 1), np.uint16)
        check(lib().aprb_sample_image(apr._h, _ptr(a), _ptr(out)))
        self.data = out[: apr.total_number_particles()]
        return self


class APRReconstruction:
    """Piecewise-constant and level images of an APR at full resolution
    (APRReconstruction::reconstruct_constant / reconstruct_level,
    src/numerics/APRReconstruction.hpp:80, 132)."""

    @staticmethod
    def reconstruct_constant(apr, particle_data):
        """(z, x, y) image of the particles' values; uint16 or float32 like the
        particle data."""
        parts = getattr(particle_data, "data", particle_data)
        if hasattr(parts, "data_ptr"):
            raise TypeError("use the device entry points for CUDA tensors")
        kind = np.float32 if np.asarray(parts).dtype.kind == "f" else np.uint16
        p = np.ascontiguousarray(parts, kind)
        z, x, y = apr.org_dims(2), apr.org_dims(1), apr.org_dims(0)
        img = np.empty((z, x, y), kind)
        fn = lib().aprb_reconstruct_constant_f32 if kind is np.float32 else lib().aprb_reconstruct_constant_u16
        check(fn(apr._h, _ptr(p) if p.size else None, _ptr(img)))
        return img

    @staticmethod
    def reconstruct_level(apr):
        """(z, x, y) uint8 image of the particles' levels."""
        z, x, y = apr.org_dims(2), apr.org_dims(1), apr.org_dims(0)
        img = np.empty((z, x, y), np.uint8)
        check(lib().aprb_reconstruct_level(apr._h, _ptr(img)))
        return img


class APRTreeNumerics:
    @staticmethod
    def fill_tree_mean(apr, particle_data, tree_data=None):
        parts = np.ascontiguousarray(getattr(particle_data, "data", particle_data), np.float32)
        apr.init_tree()
        out = np.zeros(max(apr.total_number_tree_particles(), 1), np.float32)
        check(lib().aprb_fill_tree_mean(apr._h, _ptr(parts), _ptr(out)))
        res = out[: apr.total_number_tree_particles()]
        if tree_data is not None:
            tree_data.data = res
        return res


class APRFilter:
    @staticmethod
    def convolve_pencil(apr, stencil, particle_input, particle_output=None, reflect_boundary=True,
                        use_stencil_downsample=True, normalize=False):
        st = np.ascontiguousarray(stencil, np.float32).ravel()
        ks = int(round(st.size ** (1.0 / 3.0)))
        if ks ** 3 != st.size:
            raise ValueError("stencil must be cubic")
        parts = np.ascontiguousarray(getattr(particle_input, "data", particle_input), np.float32)
        out = np.zeros(max(len(parts), 1), np.float32)
        st_ = lib().aprb_convolve(apr._h, _ptr(st), ks, _ptr(parts), _ptr(out), int(reflect_boundary),
                                  int(use_stencil_downsample), int(normalize))
        check(st_)
        res = out[: len(parts)]
        if particle_output is not None:
            particle_output.data = res
        return res

    convolve = convolve_pencil


def isotropic_convolve_333(apr, particle_input, stencil, reflective_bc=True, use_stencil_downsample=True,
                           normalize_stencil=False):
    """isotropic_convolve_333 (APRIsoConvGPU333.hpp:37-51); unlike the reference
    GPU kernel the coarsest level l_min is filtered too (the CPU semantics)."""
    st = np.asarray(stencil, np.float32)
    if st.size != 27:
        raise ValueError("isotropic_convolve_333 needs a 3x3x3 stencil")
    return APRFilter.convolve_pencil(apr, st, particle_input, None, reflective_bc, use_stencil_downsample,
                                     normalize_stencil)


def isotropic_convolve_555(apr, particle_input, stencil, reflective_bc=True, use_stencil_downsample=True,
                           normalize_stencil=False):
    st = np.asarray(stencil, np.float32)
    if st.size != 125:
        raise ValueError("isotropic_convolve_555 needs a 5x5x5 stencil")
    return APRFilter.convolve_pencil(apr, st, particle_input, None, reflective_bc, use_stencil_downsample,
                                     normalize_stencil)


class APRNumerics:
    @staticmethod
    def gradient_cfd(apr, particle_input, dimension, delta=1.0):
        """APRNumerics::gradient_cfd (APRNumerics.hpp:165-184): central
        difference along dimension 0 (y), 1 (x) or 2 (z); float32 particles."""
        return APRNumerics._gradient(apr, particle_input, dimension, delta, 0)

    @staticmethod
    def gradient_sobel(apr, particle_input, dimension, delta=1.0):
        """APRNumerics::gradient_sobel (APRNumerics.hpp:187-215)."""
        return APRNumerics._gradient(apr, particle_input, dimension, delta, 1)

    @staticmethod
    def gradient_magnitude_cfd(apr, particle_input, deltas=(1.0, 1.0, 1.0)):
        """APRNumerics::gradient_magnitude_cfd (APRNumerics.hpp:218-251)."""
        return APRNumerics._magnitude(apr, particle_input, deltas, 0)

    @staticmethod
    def gradient_magnitude_sobel(apr, particle_input, deltas=(1.0, 1.0, 1.0)):
        """APRNumerics::gradient_magnitude_sobel (APRNumerics.hpp:254-287)."""
        return APRNumerics._magnitude(apr, particle_input, deltas, 1)

    @staticmethod
    def _gradient(apr, particle_input, dimension, delta, sobel):
        x = np.ascontiguousarray(getattr(particle_input, "data", particle_input), np.float32)
        out = np.zeros(max(x.size, 1), np.float32)
        check(lib().aprb_gradient(apr._h, _ptr(x) if x.size else None, _ptr(out), int(dimension), float(delta),
                                  int(sobel)))
        return out[: x.size]

    @staticmethod
    def _magnitude(apr, particle_input, deltas, sobel):
        x = np.ascontiguousarray(getattr(particle_input, "data", particle_input), np.float32)
        out = np.zeros(max(x.size, 1), np.float32)
        d = np.ascontiguousarray(deltas, np.float32)
        check(lib().aprb_gradient_magnitude(apr._h, _ptr(x) if x.size else None, _ptr(out), _ptr(d), int(sobel)))
        return out[: x.size]

    @staticmethod
    def richardson_lucy(apr, particle_input, particle_output, psf, number_iterations, use_stencil_downsample=True,
                        normalize=False, resume=False, dtype=np.float32):
        """APRNumerics::richardson_lucy (APRNumerics.hpp:132-134, 551-593).
        dtype float64 runs the reference's double instantiation (double
        stencils, tree and output), as a particle_output holding float64 data
        also selects."""
        st = np.ascontiguousarray(psf, np.float32).ravel()
        ks = int(round(st.size ** (1.0 / 3.0)))
        if ks ** 3 != st.size or ks not in (3, 5):
            raise RuntimeError("APR RL: stencil side must be 3 or 5")
        parts = np.ascontiguousarray(getattr(particle_input, "data", particle_input), np.uint16)
        n = len(parts)
        prev = getattr(particle_output, "data", None)
        if prev is not None and np.asarray(prev).dtype == np.float64:
            dtype = np.float64
        dtype = np.dtype(dtype)
        if resume and prev is not None:
            out = np.ascontiguousarray(prev, dtype).copy()
        else:
            out = np.zeros(max(n, 1), dtype)
        out = np.resize(out, max(n, 1)).astype(dtype)
        fn = lib().aprb_richardson_lucy_fp64 if dtype == np.float64 else lib().aprb_richardson_lucy
        check(fn(apr._h, _ptr(parts), _ptr(out), _ptr(st), ks, int(number_iterations), int(use_stencil_downsample),
                 int(normalize), int(resume)))
        res = out[:n]
        if particle_output is not None:
            particle_output.data = res
        return res


class APRStencil:
    @staticmethod
    def create_gaussian_filter(sigma=(1.0, 1.0, 1.0), size=(5, 5, 5), normalize=True):
        """APRStencil::create_gaussian_filter<float> (APRStencil.hpp:174-228),
        float arithmetic as the reference (expf, sqrtf of 2*pi)."""
        f32 = np.float32

        def g1(s, n):
            if n <= 1:
                return np.ones(1, f32)
            i = np.arange(-(n // 2), n // 2 + 1)
            num = np.exp((-(i * i) / (2 * f32(s) * f32(s))).astype(f32)).astype(f32)
            den = f32(s) * f32(math.sqrt(np.float32(2 * math.pi)))
            return (num / den).astype(f32)

        gy, gx, gz = g1(sigma[0], size[0]), g1(sigma[1], size[1]), g1(sigma[2], size[2])
        st = np.zeros((size[2], size[1], size[0]), f32)
        s = f32(0)
        for i in range(size[0]):
            for j in range(size[1]):
                for k in range(size[2]):
                    v = f32(f32(gy[i] * gx[j]) * gz[k])
                    st[k, j, i] = v
                    s = f32(s + v)
        if normalize:
            st = (st / s).astype(f32)
        return st


def threshold_li(values, integer_values=False):
    """threshold_li<T> (src/algorithm/AutoParameters.hpp:50-100): Li's minimum
    cross entropy threshold of the values (T = uint16 when integer_values,
    else float), computed on the GPU with FP64 sums."""
    v = np.ascontiguousarray(values, np.float32).ravel()
    out = C.c_float()
    check(lib().aprb_threshold_li(_ptr(v) if v.size else None, v.size, int(bool(integer_values)), C.byref(out)))
    return out.value


def auto_parameters_li_entropy(par, image, local_intensity_scale, grad, bspline_offset=0.0, grad_integer=True):
    """autoParametersLiEntropy (src/algorithm/AutoParameters.hpp:103-153) on
    down-sampled arrays of one shape: sets par.grad_th and par.sigma_th from the
    cells whose image value exceeds par.Ip_th + bspline_offset.  grad holds
    ImageType values (grad_integer for uint16)."""
    im, ls, g = (np.ascontiguousarray(a, np.float32).ravel() for a in (image, local_intensity_scale, grad))
    if not (im.size == ls.size == g.size):
        raise ValueError("image, local_intensity_scale and grad must have the same size")
    p = par.c()
    check(lib().aprb_auto_parameters(C.byref(p), _ptr(im), _ptr(ls), _ptr(g), im.size, int(bool(grad_integer)),
                                     float(bspline_offset)))
    par.grad_th = float(p.grad_th)
    par.sigma_th = float(p.sigma_th)
    return par


SCHEDULE_BUCKETS = (128, 256, 512, 1024, 2048, None)  # line-length bucket limits (None: longer)


def smoothing_variants():
    """Number of kernel variants of the smoothing passes per axis {"y", "x", "z"}."""
    out = {}
    for a, name in enumerate(_lib.AXES):
        n = C.c_int()
        check(lib().aprb_smoothing_variants(a, C.byref(n)))
        out[name] = n.value
    return out


def smoothing_schedule():
    """The process's smoothing schedule: {axis: [variant per line-length bucket]}."""
    out = {}
    for a, name in enumerate(_lib.AXES):
        row = []
        for b in range(len(SCHEDULE_BUCKETS)):
            v = C.c_int()
            check(lib().aprb_smoothing_schedule_get(a, b, C.byref(v)))
            row.append(v.value)
        out[name] = row
    return out


def set_smoothing_schedule(schedule):
    """Sets {axis: [variant per bucket]} (every variant computes the same bits)."""
    for a, name in enumerate(_lib.AXES):
        for b, v in enumerate(schedule.get(name, [])):
            check(lib().aprb_smoothing_schedule_set(a, b, int(v)))


def kernel_launch_count():
    return int(lib().aprb_kernel_launch_count())


def synth_blobs_device(out_tensor, n_blobs, sigma=(2.0, 6.0), amp=(800.0, 4000.0), background=100.0, seed=0,
                       stream=None):
    """Fills a (z, x, y) uint16 CUDA tensor with the seeded blob + Poisson model."""
    z, x, y = out_tensor.shape
    check(lib().aprb_synth_blobs_u16(_dptr(out_tensor), y, x, z, int(n_blobs), sigma[0], sigma[1], amp[0], amp[1],
                                     background, int(seed), _stream(stream)))


def synth_ground_truth_device(out_tensor, n_blobs, sigma=(1.0, 4.0), amp=(500.0, 5000.0), background=50.0, seed=0,
                              stream=None):
    """Fills a (z, x, y) float32 CUDA tensor with the noise-free blob intensities."""
    z, x, y = out_tensor.shape
    check(lib().aprb_synth_blobs_f32(_dptr(out_tensor), y, x, z, int(n_blobs), sigma[0], sigma[1], amp[0], amp[1],
                                     background, int(seed), _stream(stream)))

from . import learned  # noqa: E402,F401  (the learned RL proposal)
