/*
 * aprb200_libapr.hpp -- the B200 path inside LibAPR itself.
 *
 * What a LibAPR build includes (with LibAPR's src/ directory on the include
 * path and libaprb200.so linked) to run its hot path on the GPU while every
 * caller keeps LibAPR's own objects: the functions below take and fill the
 * reference's APR, PixelData, ParticleData and VectorData, with the
 * signatures and error behaviour of the functions they replace:
 *
 *   aprb200::libapr::get_apr(conv, apr, img)        APRConverter<IT>::get_apr (APRConverter.hpp:69, 591-600)
 *   aprb200::libapr::sample_image(parts, apr, img)  ParticleData<T>::sample_image (ParticleData.hpp:123-127)
 *   aprb200::libapr::get_apr_by_block(conv, apr, img)
 *                                                   APRConverterBatch<IT>::get_apr (APRConverterBatch.hpp:48-64,
 *                                                   114-175) with the volume in memory instead of a TIFF file
 *   aprb200::libapr::sample_parts_from_img_blocked(parts, apr, img, z_block, ghost)
 *                                                   ParticleData::sample_parts_from_img_blocked (ParticleData.hpp:140)
 *   aprb200::libapr::convolve_pencil(...)           APRFilter::convolve_pencil (APRFilter.hpp:139-149)
 *   aprb200::libapr::richardson_lucy(...)           APRNumerics::richardson_lucy (APRNumerics.hpp:132-134)
 *   aprb200::libapr::isotropic_convolve_333/555     isotropic_convolve_333/555 (APRIsoConvGPU333.hpp:37-51,
 *                                                   APRIsoConvGPU555.hpp:38-52)
 *   aprb200::libapr::richardson_lucy_gpu            APRNumericsGPU::richardson_lucy (APRNumericsGPU.hpp:105-108)
 *
 * get_apr returns false when the input dimension check fails and throws
 * std::invalid_argument on uint16 smoothing overflow (ComputeGradient.hpp:409-412);
 * a stencil whose side is not 3 or 5 throws std::runtime_error
 * (APRNumericsGPU.cu:201-203); other failures throw std::runtime_error with the
 * library's message.  The GPU-form functions read only the structure of the
 * access helpers (their linearAccess), so a LibAPR build passes its
 * GPUAccessHelper objects unchanged.  Unlike the reference's GPU convolution,
 * level l_min is filtered too (the CPU semantics).
 */
#ifndef APRB200_LIBAPR_HPP
#define APRB200_LIBAPR_HPP

#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "aprb200.h"
#include "algorithm/APRConverter.hpp"
#include "data_structures/APR/APR.hpp"
#include "data_structures/APR/particles/ParticleData.hpp"
#ifdef HAVE_LIBTIFF
#include "algorithm/APRConverterBatch.hpp"
#endif

namespace aprb200 {
namespace libapr {

inline void raise(aprb_status s) {
    if (s == APRB_OK) return;
    const std::string msg = std::string(aprb_status_string(s)) + ": " + aprb_last_error();
    if (s == APRB_ERR_INTEGER_OVERFLOW) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

// APRParameters (APRParameters.hpp:14-41) as the C ABI's parameter block
inline aprb_params params(const APRParameters &par) {
    aprb_params p;
    aprb_default_params(&p);
    p.dx = par.dx; p.dy = par.dy; p.dz = par.dz;
    p.psfx = par.psfx; p.psfy = par.psfy; p.psfz = par.psfz;
    p.Ip_th = par.Ip_th; p.lambda = par.lambda; p.rel_error = par.rel_error;
    p.sigma_th = par.sigma_th; p.sigma_th_max = par.sigma_th_max; p.grad_th = par.grad_th;
    p.reflect_bc_lis = par.reflect_bc_lis; p.neighborhood_optimization = par.neighborhood_optimization;
    p.constant_intensity_scale = par.constant_intensity_scale; p.check_input = par.check_input;
    p.swap_dimensions = par.swap_dimensions; p.auto_parameters = par.auto_parameters;
    return p;
}

// An APR handle of the library, freed on scope exit.
struct Handle {
    aprb_apr *a = nullptr;
    Handle() = default;
    Handle(const Handle &) = delete;
    Handle &operator=(const Handle &) = delete;
    ~Handle() {
        if (a) aprb_apr_free(a);
    }
};

// A handle on the structure of LibAPR's linear access (its three arrays are
// copied to the GPU).
inline void handle_of(LinearAccess &la, Handle &h) {
    GenInfo &g = *la.genInfo;
    raise(aprb_apr_from_arrays(g.org_dims[0], g.org_dims[1], g.org_dims[2], la.level_xz_vec.begin(),
                               la.level_xz_vec.size(), la.xz_end_vec.begin(), la.xz_end_vec.size(),
                               la.y_vec.begin(), la.y_vec.size(), &h.a));
}

// Fills LibAPR's APR (aprInfo and linearAccess, APR.hpp:40-59) from a handle.
inline void fill_apr(APR &apr, aprb_apr *a, const APRParameters &par) {
    aprb_apr_info info;
    raise(aprb_apr_get_info(a, &info));
    apr.parameters = par;
    apr.aprInfo.init(info.org_dims[0], info.org_dims[1], info.org_dims[2]);
    apr.linearAccess.genInfo = &apr.aprInfo;
    apr.linearAccess.level_xz_vec.resize(info.n_level_xz);
    apr.linearAccess.xz_end_vec.resize(info.n_xz);
    apr.linearAccess.y_vec.resize(info.total_number_particles);
    raise(aprb_apr_export(a, apr.linearAccess.level_xz_vec.begin(), apr.linearAccess.xz_end_vec.begin(),
                          apr.linearAccess.y_vec.begin()));
    apr.aprInfo.total_number_particles = info.total_number_particles;
    apr.apr_initialized = true;
    apr.tree_initialized = false;
}

/* APRConverter<ImageType>::get_apr(APR&, PixelData<T>&) on the GPU: the
 * converter's par (and, with par.auto_parameters, the thresholds it chooses)
 * and bspline_offset are set as the reference sets them. */
template <typename ImageType, typename T>
bool get_apr(APRConverter<ImageType> &conv, APR &apr, PixelData<T> &img) {
    static_assert(std::is_same<T, uint16_t>::value, "the B200 path takes uint16 input images");
    aprb_params p = params(conv.par);
    aprb_converter *c = nullptr;
    raise(aprb_converter_create(std::is_floating_point<ImageType>::value ? APRB_IMAGE_FLOAT : APRB_IMAGE_U16, &c));
    Handle h;
    const aprb_status s = aprb_get_apr(c, &p, img.mesh.begin(), img.y_num, img.x_num, img.z_num, &h.a);
    aprb_converter_destroy(c);
    if (s == APRB_ERR_DIMENSIONS) return false;
    raise(s);
    aprb_params used;
    raise(aprb_apr_get_parameters(h.a, &used));
    conv.par.grad_th = used.grad_th;
    conv.par.sigma_th = used.sigma_th;
    aprb_apr_info info;
    raise(aprb_apr_get_info(h.a, &info));
    conv.bspline_offset = info.bspline_offset;
    fill_apr(apr, h.a, conv.par);
    return true;
}

/* ParticleData<T>::sample_image(APR&, PixelData<uint16_t>&): uint16
 * intensities as the reference computes them, converted to T. */
template <typename T>
void sample_image(ParticleData<T> &parts, APR &apr, PixelData<uint16_t> &img) {
    Handle h;
    handle_of(apr.linearAccess, h);
    std::vector<uint16_t> v(apr.total_number_particles());
    raise(aprb_sample_image(h.a, img.mesh.begin(), v.data()));
    parts.data.resize(v.size());
    for (size_t i = 0; i < v.size(); ++i) parts.data[i] = (T)v[i];
}

/* ParticleData<T>::sample_parts_from_img_blocked (ParticleData.hpp:140-142,
 * 288-372): every z-tile of z_block_size planes (ghost_z planes of overlap)
 * samples its rows from its own pyramid; the volume comes from memory where
 * the reference reads the tiles from a TIFF file. */
template <typename T>
void sample_parts_from_img_blocked(ParticleData<T> &parts, APR &apr, PixelData<uint16_t> &img,
                                   int z_block_size = 256, int ghost_z = 32) {
    Handle h;
    handle_of(apr.linearAccess, h);
    std::vector<uint16_t> v(apr.total_number_particles());
    raise(aprb_sample_image_by_block(h.a, img.mesh.begin(), z_block_size, ghost_z, v.data()));
    parts.data.resize(v.size());
    for (size_t i = 0; i < v.size(); ++i) parts.data[i] = (T)v[i];
}

#ifdef HAVE_LIBTIFF
/* APRConverterBatch<ImageType>::get_apr(APR&) (APRConverterBatch.hpp:48-64,
 * 114-175): the pixel pipeline per z-tile of conv.z_block_size planes with
 * conv.ghost_z planes of overlap (get_apr_method_patch :190-271), one global
 * particle-cell tree, one pulling scheme; the volume comes from memory where
 * the reference reads it tile by tile from par.input_dir +
 * par.input_image_name.  The per-tile form (get_apr_method_patch on one
 * ImagePatch) is aprb_pyramid_fill_tiles_device of the C ABI. */
template <typename ImageType>
bool get_apr_by_block(APRConverterBatch<ImageType> &conv, APR &apr, PixelData<uint16_t> &img) {
    aprb_params p = params(conv.par);
    aprb_converter *c = nullptr;
    raise(aprb_converter_create(std::is_floating_point<ImageType>::value ? APRB_IMAGE_FLOAT : APRB_IMAGE_U16, &c));
    Handle h;
    const aprb_status s = aprb_get_apr_by_block(c, &p, img.mesh.begin(), img.y_num, img.x_num, img.z_num,
                                                conv.z_block_size, conv.ghost_z, &h.a);
    aprb_converter_destroy(c);
    if (s == APRB_ERR_DIMENSIONS) return false;
    raise(s);
    aprb_params used;
    raise(aprb_apr_get_parameters(h.a, &used));
    conv.par.grad_th = used.grad_th;
    conv.par.sigma_th = used.sigma_th;
    fill_apr(apr, h.a, conv.par);
    return true;
}
#endif

namespace detail {
template <typename S>
std::vector<float> stencil_floats(const PixelData<S> &st, int &ksize) {
    if (!(st.y_num == st.x_num && st.x_num == st.z_num && (st.y_num == 3 || st.y_num == 5)))
        throw std::runtime_error("stencil must be 3x3x3 or 5x5x5");
    ksize = st.y_num;
    std::vector<float> f(st.mesh.size());
    for (size_t i = 0; i < f.size(); ++i) f[i] = (float)st.mesh[i];
    return f;
}
template <typename V>
std::vector<float> floats(const V &v, size_t n) {
    std::vector<float> f(n);
    for (size_t i = 0; i < n; ++i) f[i] = (float)v[i];
    return f;
}
}  // namespace detail

/* APRFilter::convolve_pencil(APR&, const PixelData<S>&, in, out, reflect, ds, normalize) */
template <typename S, typename In, typename Out>
void convolve_pencil(APR &apr, const PixelData<S> &stencil, const ParticleData<In> &in, ParticleData<Out> &out,
                     bool reflect_boundary = true, bool use_stencil_downsample = true, bool normalize = false) {
    int ks = 0;
    std::vector<float> st = detail::stencil_floats(stencil, ks);
    Handle h;
    handle_of(apr.linearAccess, h);
    const size_t P = apr.total_number_particles();
    std::vector<float> fin = detail::floats(in.data, P), fout(P);
    raise(aprb_convolve(h.a, st.data(), ks, fin.data(), fout.data(), reflect_boundary, use_stencil_downsample,
                        normalize));
    out.data.resize(P);
    for (size_t i = 0; i < P; ++i) out.data[i] = (Out)fout[i];
}

/* APRNumerics::richardson_lucy(APR&, ParticleData<In>&, ParticleData<Out>&,
 * PixelData<S>& psf, niter, ds, normalize, resume); Out = double runs the FP64
 * instantiation. */
template <typename In, typename Out, typename S>
void richardson_lucy(APR &apr, ParticleData<In> &in, ParticleData<Out> &out, PixelData<S> &psf, int niter,
                     bool use_stencil_downsample = true, bool normalize = false, bool resume = false) {
    static_assert(std::is_floating_point<Out>::value, "richardson_lucy writes floating-point particles");
    int ks = 0;
    std::vector<float> st = detail::stencil_floats(psf, ks);
    Handle h;
    handle_of(apr.linearAccess, h);
    const size_t P = apr.total_number_particles();
    std::vector<uint16_t> raw(P);
    for (size_t i = 0; i < P; ++i) raw[i] = (uint16_t)in.data[i];
    if (!resume || out.data.size() != P) out.data.resize(P);
    if (std::is_same<Out, double>::value) {
        raise(aprb_richardson_lucy_fp64(h.a, raw.data(), (double *)out.data.begin(), st.data(), ks, niter,
                                        use_stencil_downsample, normalize, resume));
    } else {
        std::vector<float> f = resume ? detail::floats(out.data, P) : std::vector<float>(P);
        raise(aprb_richardson_lucy(h.a, raw.data(), f.data(), st.data(), ks, niter, use_stencil_downsample, normalize,
                                   resume));
        for (size_t i = 0; i < P; ++i) out.data[i] = (Out)f[i];
    }
}

namespace detail {
template <class Access, typename In, typename Out, typename S, typename Tree>
void isotropic_convolve(int side, Access &access, VectorData<In> &input, VectorData<Out> &output,
                        PixelData<S> &stencil, VectorData<Tree> &tree_data, bool reflective_bc,
                        bool use_stencil_downsample, bool normalize) {
    int ks = 0;
    std::vector<float> st = stencil_floats(stencil, ks);
    if (ks != side) throw std::runtime_error("stencil side does not match the convolution");
    Handle h;
    handle_of(*access.linearAccess, h);
    aprb_apr_info info;
    raise(aprb_apr_get_info(h.a, &info));
    const size_t P = info.total_number_particles;
    std::vector<float> fin = floats(input, P), fout(P);
    raise(aprb_convolve(h.a, st.data(), ks, fin.data(), fout.data(), reflective_bc, use_stencil_downsample,
                        normalize));
    output.resize(P);
    for (size_t i = 0; i < P; ++i) output[i] = (Out)fout[i];
    // the reference leaves the tree means it filtered with in tree_data
    raise(aprb_apr_init_tree(h.a));
    raise(aprb_apr_get_info(h.a, &info));
    std::vector<float> tm(info.tree_total_number_particles ? info.tree_total_number_particles : 1);
    raise(aprb_fill_tree_mean(h.a, fin.data(), tm.data()));
    tree_data.resize(info.tree_total_number_particles);
    for (size_t i = 0; i < info.tree_total_number_particles; ++i) tree_data[i] = (Tree)tm[i];
}
}  // namespace detail

/* isotropic_convolve_333(GPUAccessHelper&, GPUAccessHelper&, VectorData<in>&,
 * VectorData<out>&, PixelData<S>& stencil, VectorData<tree>&, reflective_bc,
 * use_stencil_downsample, normalize) */
template <class Access, typename In, typename Out, typename S, typename Tree>
void isotropic_convolve_333(Access &access, Access & /*tree_access*/, VectorData<In> &input, VectorData<Out> &output,
                            PixelData<S> &stencil, VectorData<Tree> &tree_data, bool reflective_bc = false,
                            bool use_stencil_downsample = false, bool normalize_stencil = false) {
    detail::isotropic_convolve(3, access, input, output, stencil, tree_data, reflective_bc, use_stencil_downsample,
                               normalize_stencil);
}

/* isotropic_convolve_555, the same with a 5x5x5 stencil */
template <class Access, typename In, typename Out, typename S, typename Tree>
void isotropic_convolve_555(Access &access, Access & /*tree_access*/, VectorData<In> &input, VectorData<Out> &output,
                            PixelData<S> &stencil, VectorData<Tree> &tree_data, bool reflective_bc = false,
                            bool use_stencil_downsample = false, bool normalize_stencil = false) {
    detail::isotropic_convolve(5, access, input, output, stencil, tree_data, reflective_bc, use_stencil_downsample,
                               normalize_stencil);
}

/* APRNumericsGPU::richardson_lucy(GPUAccessHelper&, GPUAccessHelper&,
 * VectorData<In>&, VectorData<S>& output, PixelData<S>& psf, niter, ds,
 * normalize, resume) */
template <class Access, typename In, typename S>
void richardson_lucy_gpu(Access &access, Access & /*tree_access*/, VectorData<In> &input, VectorData<S> &output,
                         PixelData<S> &psf, int niter, bool use_stencil_downsample = true,
                         bool normalize_stencil = false, bool resume = false) {
    int ks = 0;
    std::vector<float> st = detail::stencil_floats(psf, ks);
    Handle h;
    handle_of(*access.linearAccess, h);
    const size_t P = input.size();
    std::vector<uint16_t> raw(P);
    for (size_t i = 0; i < P; ++i) raw[i] = (uint16_t)input[i];
    if (!resume || output.size() != P) output.resize(P);
    if (std::is_same<S, double>::value) {
        raise(aprb_richardson_lucy_fp64(h.a, raw.data(), (double *)output.begin(), st.data(), ks, niter,
                                        use_stencil_downsample, normalize_stencil, resume));
    } else {
        std::vector<float> f = resume ? detail::floats(output, P) : std::vector<float>(P);
        raise(aprb_richardson_lucy(h.a, raw.data(), f.data(), st.data(), ks, niter, use_stencil_downsample,
                                   normalize_stencil, resume));
        for (size_t i = 0; i < P; ++i) output[i] = (S)f[i];
    }
}

}  // namespace libapr
}  // namespace aprb200

#endif
