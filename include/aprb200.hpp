/*
 * aprb200.hpp -- header-only C++ host layer over the C ABI of libaprb200.so.
 *
 * aprb200::compat re-creates the call signatures of LibAPR's hot path so that
 * code written against LibAPR keeps its shape:
 *
 *   PixelData<uint16_t> img(y, x, z);            // PixelData.hpp (y fastest)
 *   APRConverter<float> conv;                     // APRConverter.hpp:35-134
 *   conv.par.lambda = 3; ...                      // APRParameters.hpp:11-50
 *   APR apr;  conv.get_apr(apr, img);             // APRConverter.hpp:591-600
 *   ParticleData<uint16_t> parts;
 *   parts.sample_image(apr, img);                 // ParticleData.hpp:123-127
 *   APRFilter::convolve_pencil(apr, stencil, in, out, true, true, false);   // APRFilter.hpp:139-149
 *   APRNumerics::richardson_lucy(apr, parts, out, psf, 20, true, false, false); // APRNumerics.hpp:132-134
 *
 * Errors follow the reference: get_apr returns false when the dimension check
 * fails and throws std::invalid_argument on uint16 smoothing overflow;
 * unsupported stencil sizes throw std::runtime_error; other failures throw
 * aprb200::Error carrying the aprb_status.
 */
#ifndef APRB200_HPP
#define APRB200_HPP

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "aprb200.h"

namespace aprb200 {

struct Error : std::runtime_error {
    aprb_status status;
    Error(aprb_status s, const std::string &m) : std::runtime_error(m), status(s) {}
};

inline void check(aprb_status s) {
    if (s == APRB_OK) return;
    std::string msg = std::string(aprb_status_string(s)) + ": " + aprb_last_error();
    if (s == APRB_ERR_INTEGER_OVERFLOW) throw std::invalid_argument(msg);
    if (s == APRB_ERR_UNSUPPORTED) throw std::runtime_error(msg);
    throw Error(s, msg);
}

namespace compat {

struct APRParameters {
    float dx = 1, dy = 1, dz = 1;
    float psfx = 2, psfy = 2, psfz = 2;
    float Ip_th = 0, lambda = 3.0f, rel_error = 0.1f, sigma_th = 0, sigma_th_max = 0, grad_th = 0;
    bool auto_parameters = false;
    bool reflect_bc_lis = true, check_input = false, swap_dimensions = false, neighborhood_optimization = true,
         constant_intensity_scale = false, output_steps = false;

    aprb_params c() const {
        aprb_params p;
        aprb_default_params(&p);
        p.dx = dx; p.dy = dy; p.dz = dz; p.psfx = psfx; p.psfy = psfy; p.psfz = psfz;
        p.Ip_th = Ip_th; p.lambda = lambda; p.rel_error = rel_error; p.sigma_th = sigma_th;
        p.sigma_th_max = sigma_th_max; p.grad_th = grad_th;
        p.reflect_bc_lis = reflect_bc_lis; p.neighborhood_optimization = neighborhood_optimization;
        p.constant_intensity_scale = constant_intensity_scale; p.check_input = check_input;
        p.swap_dimensions = swap_dimensions;
        p.auto_parameters = auto_parameters;
        return p;
    }
    static APRParameters from_c(const aprb_params &p) {
        APRParameters r;
        r.dx = p.dx; r.dy = p.dy; r.dz = p.dz; r.psfx = p.psfx; r.psfy = p.psfy; r.psfz = p.psfz;
        r.Ip_th = p.Ip_th; r.lambda = p.lambda; r.rel_error = p.rel_error; r.sigma_th = p.sigma_th;
        r.sigma_th_max = p.sigma_th_max; r.grad_th = p.grad_th;
        r.reflect_bc_lis = p.reflect_bc_lis != 0; r.neighborhood_optimization = p.neighborhood_optimization != 0;
        r.constant_intensity_scale = p.constant_intensity_scale != 0; r.check_input = p.check_input != 0;
        r.swap_dimensions = p.swap_dimensions != 0; r.auto_parameters = p.auto_parameters != 0;
        return r;
    }
};

template <typename T>
struct PixelData {
    int y_num = 0, x_num = 0, z_num = 0;
    std::vector<T> mesh;
    PixelData() = default;
    PixelData(int y, int x, int z) { init(y, x, z); }
    void init(int y, int x, int z) {
        y_num = y; x_num = x; z_num = z;
        mesh.assign((size_t)y * x * z, T(0));
    }
    T &at(int y, int x, int z) { return mesh[((size_t)z * x_num + x) * y_num + y]; }
    const T &at(int y, int x, int z) const { return mesh[((size_t)z * x_num + x) * y_num + y]; }
};

class APR {
  public:
    APR() = default;
    APR(const APR &) = delete;
    APR &operator=(const APR &) = delete;
    APR(APR &&o) noexcept : h_(o.h_) { o.h_ = nullptr; }
    ~APR() { reset(nullptr); }
    void reset(aprb_apr *h) {
        if (h_) aprb_apr_free(h_);
        h_ = h;
    }
    aprb_apr *handle() const { return h_; }
    aprb_apr_info info() const {
        aprb_apr_info i;
        check(aprb_apr_get_info(h_, &i));
        return i;
    }
    int level_max() const { return info().l_max; }
    int level_min() const { return info().l_min; }
    uint64_t total_number_particles() const { return info().total_number_particles; }
    uint64_t org_dims(int d) const { return (uint64_t)info().org_dims[d]; }
    /* APR::get_apr_parameters (APR.hpp:99-101) */
    APRParameters get_apr_parameters() const {
        aprb_params p;
        check(aprb_apr_get_parameters(h_, &p));
        return APRParameters::from_c(p);
    }
    /* LinearAccess arrays (LinearAccess.hpp:33-35) */
    void linear_access(std::vector<uint64_t> &level_xz, std::vector<uint64_t> &xz_end, std::vector<uint16_t> &y_vec) const {
        aprb_apr_info i = info();
        level_xz.resize(i.n_level_xz);
        xz_end.resize(i.n_xz);
        y_vec.resize(i.total_number_particles);
        check(aprb_apr_export(h_, level_xz.data(), xz_end.data(), y_vec.data()));
    }

  private:
    aprb_apr *h_ = nullptr;
};

template <typename ImageType>
class APRConverter {
  public:
    APRParameters par;
    float bspline_offset = 0;
    bool verbose = false;

    APRConverter() {
        check(aprb_converter_create(std::is_floating_point<ImageType>::value ? APRB_IMAGE_FLOAT : APRB_IMAGE_U16, &c_));
    }
    APRConverter(const APRConverter &) = delete;
    APRConverter &operator=(const APRConverter &) = delete;
    ~APRConverter() { aprb_converter_destroy(c_); }

    /* APRConverter::get_apr (APRConverter.hpp:591-600) */
    bool get_apr(APR &apr, PixelData<uint16_t> &img) {
        aprb_params p = par.c();
        aprb_apr *h = nullptr;
        aprb_status s = aprb_get_apr(c_, &p, img.mesh.data(), img.y_num, img.x_num, img.z_num, &h);
        if (s == APRB_ERR_DIMENSIONS) return false;
        check(s);
        apr.reset(h);
        bspline_offset = apr.info().bspline_offset;
        if (par.auto_parameters) {  // autoParametersLiEntropy writes the converter's par (APRConverter.hpp:558)
            const APRParameters used = apr.get_apr_parameters();
            par.grad_th = used.grad_th;
            par.sigma_th = used.sigma_th;
        }
        return true;
    }

  private:
    aprb_converter *c_ = nullptr;
};

template <typename T>
struct ParticleData {
    std::vector<T> data;
    size_t size() const { return data.size(); }
    T &operator[](size_t i) { return data[i]; }
    const T &operator[](size_t i) const { return data[i]; }
    void init(uint64_t n) { data.assign(n, T(0)); }
    void fill(T v) { std::fill(data.begin(), data.end(), v); }

    /* ParticleData::sample_image (ParticleData.hpp:123-127) */
    template <typename IT>
    void sample_image(APR &apr, PixelData<IT> &img) {
        static_assert(std::is_same<IT, uint16_t>::value, "sample_image: uint16 images");
        std::vector<uint16_t> tmp(apr.total_number_particles());
        check(aprb_sample_image(apr.handle(), img.mesh.data(), tmp.data()));
        data.assign(tmp.begin(), tmp.end());
    }
};

namespace APRTreeNumerics {
/* fill_tree_mean (APRTreeNumerics.hpp:63-203) */
template <typename S>
inline void fill_tree_mean(APR &apr, const ParticleData<S> &parts, ParticleData<float> &tree) {
    std::vector<float> in(parts.data.begin(), parts.data.end());
    check(aprb_apr_init_tree(apr.handle()));
    tree.init(apr.info().tree_total_number_particles);
    check(aprb_fill_tree_mean(apr.handle(), in.data(), tree.data.data()));
}
}  // namespace APRTreeNumerics

namespace APRFilter {
/* convolve_pencil (APRFilter.hpp:139-149) */
template <typename S, typename TI, typename TO>
inline void convolve_pencil(APR &apr, const PixelData<S> &stencil, const ParticleData<TI> &in, ParticleData<TO> &out,
                            bool reflect_boundary = true, bool use_stencil_downsample = true, bool normalize = false) {
    std::vector<float> st(stencil.mesh.begin(), stencil.mesh.end());
    std::vector<float> fin(in.data.begin(), in.data.end());
    std::vector<float> fout(fin.size());
    const int ks = stencil.y_num;
    if (stencil.x_num != ks || stencil.z_num != ks) throw std::invalid_argument("stencil must be cubic");
    check(aprb_convolve(apr.handle(), st.data(), ks, fin.data(), fout.data(), reflect_boundary, use_stencil_downsample,
                        normalize));
    out.data.assign(fout.begin(), fout.end());
}
}  // namespace APRFilter

namespace APRNumerics {
/* richardson_lucy (APRNumerics.hpp:132-134) */
template <typename S>
inline void richardson_lucy(APR &apr, ParticleData<uint16_t> &in, ParticleData<float> &out, PixelData<S> &psf,
                            int number_iterations, bool use_stencil_downsample = true, bool normalize = false,
                            bool resume = false) {
    std::vector<float> st(psf.mesh.begin(), psf.mesh.end());
    if (!resume) out.init(in.size());
    check(aprb_richardson_lucy(apr.handle(), in.data.data(), out.data.data(), st.data(), psf.y_num, number_iterations,
                               use_stencil_downsample, normalize, resume));
}
/* gradient_cfd / gradient_sobel (APRNumerics.hpp:165-215), float particles */
template <typename In>
inline void gradient_cfd(APR &apr, const ParticleData<In> &in, ParticleData<float> &out, int dimension,
                         float delta = 1.0f) {
    std::vector<float> x(in.data.begin(), in.data.end());
    out.init(x.size());
    check(aprb_gradient(apr.handle(), x.data(), out.data.data(), dimension, delta, 0));
}
template <typename In>
inline void gradient_sobel(APR &apr, const ParticleData<In> &in, ParticleData<float> &out, int dimension,
                           float delta = 1.0f) {
    std::vector<float> x(in.data.begin(), in.data.end());
    out.init(x.size());
    check(aprb_gradient(apr.handle(), x.data(), out.data.data(), dimension, delta, 1));
}
/* gradient_magnitude_cfd / _sobel (APRNumerics.hpp:218-287) */
template <typename In>
inline void gradient_magnitude_cfd(APR &apr, const ParticleData<In> &in, ParticleData<float> &out,
                                   const std::vector<float> &deltas = {1.0f, 1.0f, 1.0f}) {
    std::vector<float> x(in.data.begin(), in.data.end());
    out.init(x.size());
    check(aprb_gradient_magnitude(apr.handle(), x.data(), out.data.data(), deltas.data(), 0));
}
template <typename In>
inline void gradient_magnitude_sobel(APR &apr, const ParticleData<In> &in, ParticleData<float> &out,
                                     const std::vector<float> &deltas = {1.0f, 1.0f, 1.0f}) {
    std::vector<float> x(in.data.begin(), in.data.end());
    out.init(x.size());
    check(aprb_gradient_magnitude(apr.handle(), x.data(), out.data.data(), deltas.data(), 1));
}
}  // namespace APRNumerics

namespace APRReconstruction {
/* reconstruct_constant (APRReconstruction.hpp:80-123): uint16 or float values */
template <typename U, typename S>
inline void reconstruct_constant(APR &apr, PixelData<U> &img, const ParticleData<S> &parts) {
    img.init((int)apr.org_dims(0), (int)apr.org_dims(1), (int)apr.org_dims(2));
    if (std::is_floating_point<U>::value) {
        std::vector<float> p(parts.data.begin(), parts.data.end());
        std::vector<float> out(img.mesh.size());
        check(aprb_reconstruct_constant_f32(apr.handle(), p.data(), out.data()));
        img.mesh.assign(out.begin(), out.end());
    } else {
        std::vector<uint16_t> p(parts.data.begin(), parts.data.end());
        std::vector<uint16_t> out(img.mesh.size());
        check(aprb_reconstruct_constant_u16(apr.handle(), p.data(), out.data()));
        img.mesh.assign(out.begin(), out.end());
    }
}
/* reconstruct_level (APRReconstruction.hpp:132-170) */
template <typename U>
inline void reconstruct_level(APR &apr, PixelData<U> &img) {
    img.init((int)apr.org_dims(0), (int)apr.org_dims(1), (int)apr.org_dims(2));
    std::vector<uint8_t> out(img.mesh.size());
    check(aprb_reconstruct_level(apr.handle(), out.data()));
    img.mesh.assign(out.begin(), out.end());
}
}  // namespace APRReconstruction

}  // namespace compat
}  // namespace aprb200

#endif
