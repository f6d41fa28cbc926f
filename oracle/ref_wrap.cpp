/*
 * TEST INFRASTRUCTURE ONLY -- not part of the product.
 *
 * extern "C" wrapper around the LibAPR reference CPU code itself, compiled
 * from the unmodified reference headers (include path -I<LibAPR>/src) by
 * oracle/Makefile into oracle/_ref/libaprref.so.  It pins the plain-C
 * restatement in oracle/apr_oracle.c and serves as the timed CPU baseline
 * ("kind": "reference").  Nothing here is copied from the reference: every
 * call goes through the reference's own classes.
 */
#include "algorithm/APRConverter.hpp"
#include "algorithm/APRConverterBatch.hpp"
#include "algorithm/AutoParameters.hpp"
#include "numerics/APRFilter.hpp"
#include "numerics/APRNumerics.hpp"
#include "numerics/APRStencil.hpp"
#include "numerics/APRTreeNumerics.hpp"

#include "apr_oracle.h"

#include <omp.h>

#include <cstring>
#include <stdexcept>
#include <type_traits>

namespace {

void set_params(APRParameters &par, const orc_params *p) {
    par.dx = p->dx; par.dy = p->dy; par.dz = p->dz;
    par.psfx = p->psfx; par.psfy = p->psfy; par.psfz = p->psfz;
    par.Ip_th = p->Ip_th; par.lambda = p->lambda; par.rel_error = p->rel_error;
    par.sigma_th = p->sigma_th; par.sigma_th_max = p->sigma_th_max; par.grad_th = p->grad_th;
    par.reflect_bc_lis = p->reflect_bc_lis != 0;
    par.neighborhood_optimization = p->neighborhood_optimization != 0;
    par.constant_intensity_scale = p->constant_intensity_scale != 0;
    par.auto_parameters = false;
    par.output_steps = false;
}

template <typename T>
void to_float(const PixelData<T> &m, float *dst) {
    for (size_t i = 0; i < m.mesh.size(); ++i) dst[i] = (float)m.mesh[i];
}

/* Runs APRConverter<IT>::get_apr_cpu stage by stage (the same calls, in the
 * same order, src/algorithm/APRConverter.hpp:535-582) so the down-sampled
 * intermediates can be captured for stage-level parity. */
template <typename IT>
struct StagedConverter : public APRConverter<IT> {
    std::vector<float> grad_raw, ids, lis_raw, grad_app, lis_app, levels;

    bool run(APR &apr, PixelData<uint16_t> &img) {
        this->verbose = false;
        if (!this->initPipelineAPR(apr, img)) return false;
        this->initPipelineMemory(img.y_num, img.x_num, img.z_num);
        this->computeL(apr, img);
        size_t nd = this->grad_temp.mesh.size();
        grad_raw.resize(nd); ids.resize(nd); lis_raw.resize(nd);
        to_float(this->grad_temp, grad_raw.data());
        to_float(this->local_scale_temp2, ids.data());
        to_float(this->local_scale_temp, lis_raw.data());
        this->applyParameters(apr, this->par);
        grad_app.resize(nd); lis_app.resize(nd);
        to_float(this->grad_temp, grad_app.data());
        to_float(this->local_scale_temp, lis_app.data());
        /* solveForAPR (APRConverter.hpp:301-336), split to expose the levels */
        this->iLocalParticleSet.computeLevels(this->grad_temp, this->local_scale_temp, apr.level_max(),
                                              this->par.rel_error, this->par.dx, this->par.dy, this->par.dz);
        levels.resize(nd);
        to_float(this->local_scale_temp, levels.data());
        this->iPullingScheme.initialize_particle_cell_tree(apr.aprInfo);
        this->iLocalParticleSet.get_local_particle_cell_set(this->iPullingScheme, this->local_scale_temp,
                                                            this->local_scale_temp2, this->par);
        this->iPullingScheme.pulling_scheme_main();
        this->generateDatastructures(apr);
        return true;
    }
};

/* APRConverterBatch<IT> driven from memory: the steps of
 * get_apr_batch_method_from_file (src/algorithm/APRConverterBatch.hpp:114-175)
 * with each z-tile cut from the in-memory volume where the reference reads it
 * from a TIFF file (TiffUtils::getMesh); the per-tile work is the reference's
 * own public get_apr_method_patch. */
template <typename IT>
struct BlockConverter : public APRConverterBatch<IT> {
    bool run(APR &apr, const PixelData<uint16_t> &img, int zblock, int ghost) {
        this->z_block_size = zblock;
        this->ghost_z = ghost;
        apr.parameters = this->par;
        apr.aprInfo.init(img.y_num, img.x_num, img.z_num);
        apr.linearAccess.genInfo = &apr.aprInfo;
        apr.apr_access.genInfo = &apr.aprInfo;
        const int y_num = img.y_num, x_num = img.x_num, z_num = img.z_num;
        const int nb = std::max(z_num / zblock, 1);
        std::vector<ImagePatch> patches(nb);
        this->iPullingScheme.initialize_particle_cell_tree(apr.aprInfo);
        for (int b = 0; b < nb; ++b) {
            const int z0 = b * zblock, zf = (b == nb - 1) ? z_num : (b + 1) * zblock;
            const int gl = std::min(z0, ghost), gr = std::min(z_num - zf, ghost);
            initPatchGlobal(patches[b], z0 - gl, zf + gr, 0, x_num, 0, y_num);
            patches[b].z_ghost_l = gl;
            patches[b].z_ghost_r = gr;
            patches[b].z_offset = z0 - gl;
            PixelData<uint16_t> tile(y_num, x_num, zf + gr - (z0 - gl));
            std::memcpy(tile.mesh.begin(), img.mesh.begin() + (size_t)(z0 - gl) * x_num * y_num,
                        tile.mesh.size() * sizeof(uint16_t));
            this->get_apr_method_patch(apr, tile, patches[b]);
        }
        this->iPullingScheme.pulling_scheme_main();
        this->generateDatastructures(apr);
        return true;
    }
};

struct RefHandle {
    APR apr;
    float offset = 0;
    std::vector<float> inter[7];
};

void copy_access(const LinearAccess &la, uint64_t *level_xz, uint64_t *xz_end, uint16_t *y_vec) {
    if (level_xz) std::memcpy(level_xz, la.level_xz_vec.begin(), la.level_xz_vec.size() * sizeof(uint64_t));
    if (xz_end) std::memcpy(xz_end, la.xz_end_vec.begin(), la.xz_end_vec.size() * sizeof(uint64_t));
    if (y_vec) std::memcpy(y_vec, la.y_vec.begin(), la.y_vec.size() * sizeof(uint16_t));
}

}  // namespace

extern "C" {

/* 0 ok, 1 dimension check failed, 2 uint16 IIR overflow (std::invalid_argument) */
int ref_get_apr(const uint16_t *img, int y, int x, int z, const orc_params *p, int image_type, void **out) {
    *out = nullptr;
    PixelData<uint16_t> in(y, x, z);
    std::memcpy(in.mesh.begin(), img, sizeof(uint16_t) * (size_t)y * x * z);
    RefHandle *h = new RefHandle();
    try {
        bool ok;
        if (image_type == 1) {
            StagedConverter<uint16_t> c;
            set_params(c.par, p);
            ok = c.run(h->apr, in);
            h->offset = c.bspline_offset;
            h->inter[1] = c.grad_raw; h->inter[2] = c.ids; h->inter[3] = c.lis_raw;
            h->inter[4] = c.grad_app; h->inter[5] = c.lis_app; h->inter[6] = c.levels;
        } else {
            StagedConverter<float> c;
            set_params(c.par, p);
            ok = c.run(h->apr, in);
            h->offset = c.bspline_offset;
            h->inter[1] = c.grad_raw; h->inter[2] = c.ids; h->inter[3] = c.lis_raw;
            h->inter[4] = c.grad_app; h->inter[5] = c.lis_app; h->inter[6] = c.levels;
        }
        if (!ok) { delete h; return 1; }
    } catch (std::invalid_argument &) {
        delete h;
        return 2;
    }
    *out = h;
    return 0;
}

/* Blocked get_apr (APRConverterBatch) on an in-memory volume. */
int ref_get_apr_by_block(const uint16_t *img, int y, int x, int z, const orc_params *p, int image_type, int zblock,
                         int ghost, void **out) {
    *out = nullptr;
    PixelData<uint16_t> in(y, x, z);
    std::memcpy(in.mesh.begin(), img, sizeof(uint16_t) * (size_t)y * x * z);
    RefHandle *h = new RefHandle();
    try {
        if (image_type == 1) {
            BlockConverter<uint16_t> c;
            set_params(c.par, p);
            c.run(h->apr, in, zblock, ghost);
        } else {
            BlockConverter<float> c;
            set_params(c.par, p);
            c.run(h->apr, in, zblock, ghost);
        }
    } catch (std::invalid_argument &) {
        delete h;
        return 2;
    }
    *out = h;
    return 0;
}

/* sample_parts_from_img_downsampled_patch (ParticleData.hpp:330-372) over the
 * z-tiles of sample_parts_from_img_blocked_gen (:288-322), tiles from memory. */
int ref_sample_image_by_block(void *hv, const uint16_t *img, int zblock, int ghost, uint16_t *parts) {
    RefHandle *h = (RefHandle *)hv;
    APR &apr = h->apr;
    const int y_num = apr.org_dims(0), x_num = apr.org_dims(1), z_num = apr.org_dims(2);
    ParticleData<uint16_t> pd;
    pd.init(apr);
    const int nb = std::max(z_num / zblock, 1);
    for (int b = 0; b < nb; ++b) {
        const int z0 = b * zblock, zf = (b == nb - 1) ? z_num : (b + 1) * zblock;
        const int gl = std::min(z0, ghost), gr = std::min(z_num - zf, ghost);
        ImagePatch patch;
        initPatchGlobal(patch, z0 - gl, zf + gr, 0, x_num, 0, y_num);
        patch.z_ghost_l = gl;
        patch.z_ghost_r = gr;
        patch.z_offset = z0 - gl;
        PixelData<uint16_t> tile(y_num, x_num, zf + gr - (z0 - gl));
        std::memcpy(tile.mesh.begin(), img + (size_t)(z0 - gl) * x_num * y_num, tile.mesh.size() * sizeof(uint16_t));
        sample_parts_from_img_downsampled_patch(apr, pd, tile, patch);
    }
    std::memcpy(parts, pd.data.begin(), pd.size() * sizeof(uint16_t));
    return 0;
}

/* APRConverter::get_apr (the public entry point, no staging) for timing. */
int ref_get_apr_plain(const uint16_t *img, int y, int x, int z, const orc_params *p, int image_type, void **out) {
    *out = nullptr;
    PixelData<uint16_t> in(y, x, z);
    std::memcpy(in.mesh.begin(), img, sizeof(uint16_t) * (size_t)y * x * z);
    RefHandle *h = new RefHandle();
    try {
        bool ok;
        if (image_type == 1) {
            APRConverter<uint16_t> c;
            c.verbose = false;
            set_params(c.par, p);
            ok = c.get_apr(h->apr, in);
        } else {
            APRConverter<float> c;
            c.verbose = false;
            set_params(c.par, p);
            ok = c.get_apr(h->apr, in);
        }
        if (!ok) { delete h; return 1; }
    } catch (std::invalid_argument &) {
        delete h;
        return 2;
    }
    *out = h;
    return 0;
}

/* APRConverter::get_apr_custom_grad_scale after initPipelineAPR, with
 * bspline_offset = 0, as test_pipeline_u16 does (test/APRTest.cpp:2815-2817). */
int ref_get_apr_custom(const float *grad, const float *lis, int y, int x, int z, const orc_params *p, void **out) {
    RefHandle *h = new RefHandle();
    PixelData<uint16_t> in(y, x, z);
    APRConverter<uint16_t> c;
    c.verbose = false;
    set_params(c.par, p);
    int yd = (y + 1) / 2, xd = (x + 1) / 2, zd = (z + 1) / 2;
    PixelData<uint16_t> g(yd, xd, zd);
    PixelData<float> s(yd, xd, zd);
    for (size_t i = 0; i < g.mesh.size(); ++i) { g.mesh[i] = (uint16_t)grad[i]; s.mesh[i] = lis[i]; }
    c.bspline_offset = 0;
    c.initPipelineAPR(h->apr, in);
    c.get_apr_custom_grad_scale(h->apr, g, s);
    *out = h;
    return 0;
}

/* ------------------------------------------------------------------ automatic parameters
 * The reference's OpenMP reductions sum in an order that depends on the
 * thread count; nthreads (> 0) fixes it for the call. */
struct OmpThreads {
    int saved;
    explicit OmpThreads(int n) : saved(omp_get_max_threads()) { if (n > 0) omp_set_num_threads(n); }
    ~OmpThreads() { omp_set_num_threads(saved); }
};

/* threshold_li<T> (src/algorithm/AutoParameters.hpp:50-100), T = uint16_t
 * when is_u16, else float; v holds the values as float. */
float ref_threshold_li(const float *v, size_t n, int is_u16, int nthreads) {
    OmpThreads th(nthreads);
    if (is_u16) {
        std::vector<uint16_t> in(n);
        for (size_t i = 0; i < n; ++i) in[i] = (uint16_t)v[i];
        return threshold_li(in);
    }
    std::vector<float> in(v, v + n);
    return threshold_li(in);
}

/* autoParametersLiEntropy (src/algorithm/AutoParameters.hpp:103-153) on ds
 * arrays of shape (y, x, z): image = local_scale_temp2, lis =
 * local_scale_temp, grad = grad_temp holding ImageType values (uint16_t when
 * grad_u16). */
int ref_auto_parameters(const float *image, const float *lis, const float *grad, int y, int x, int z, int grad_u16,
                        float Ip_th, float bspline_offset, int nthreads, float *grad_th, float *sigma_th) {
    OmpThreads th(nthreads);
    PixelData<float> im(y, x, z), ls(y, x, z);
    std::memcpy(im.mesh.begin(), image, im.mesh.size() * sizeof(float));
    std::memcpy(ls.mesh.begin(), lis, ls.mesh.size() * sizeof(float));
    APRParameters par;
    par.Ip_th = Ip_th;
    if (grad_u16) {
        PixelData<uint16_t> g(y, x, z);
        for (size_t i = 0; i < g.mesh.size(); ++i) g.mesh[i] = (uint16_t)grad[i];
        autoParametersLiEntropy(par, im, ls, g, bspline_offset, false);
    } else {
        PixelData<float> g(y, x, z);
        std::memcpy(g.mesh.begin(), grad, g.mesh.size() * sizeof(float));
        autoParametersLiEntropy(par, im, ls, g, bspline_offset, false);
    }
    *grad_th = par.grad_th;
    *sigma_th = par.sigma_th;
    return 0;
}

/* APRConverter::get_apr with par.auto_parameters = true (the public entry
 * point, APRConverter.hpp:556-561); the thresholds it chose are read back
 * from APR::get_apr_parameters. */
int ref_get_apr_auto(const uint16_t *img, int y, int x, int z, const orc_params *p, int image_type, int nthreads,
                     void **out, float *grad_th, float *sigma_th) {
    OmpThreads th(nthreads);
    *out = nullptr;
    PixelData<uint16_t> in(y, x, z);
    std::memcpy(in.mesh.begin(), img, sizeof(uint16_t) * (size_t)y * x * z);
    RefHandle *h = new RefHandle();
    try {
        bool ok;
        if (image_type == 1) {
            APRConverter<uint16_t> c;
            c.verbose = false;
            set_params(c.par, p);
            c.par.auto_parameters = true;
            ok = c.get_apr(h->apr, in);
            h->offset = c.bspline_offset;
        } else {
            APRConverter<float> c;
            c.verbose = false;
            set_params(c.par, p);
            c.par.auto_parameters = true;
            ok = c.get_apr(h->apr, in);
            h->offset = c.bspline_offset;
        }
        if (!ok) { delete h; return 1; }
    } catch (std::invalid_argument &) {
        delete h;
        return 2;
    }
    const APRParameters par = h->apr.get_apr_parameters();
    *grad_th = par.grad_th;
    *sigma_th = par.sigma_th;
    *out = h;
    return 0;
}

/* The blocked converter with par.auto_parameters = true: every tile chooses
 * its thresholds (APRConverterBatch.hpp:243-247) and the APR keeps the last
 * tile's, read back from APR::get_apr_parameters. */
int ref_get_apr_by_block_auto(const uint16_t *img, int y, int x, int z, const orc_params *p, int image_type,
                              int zblock, int ghost, int nthreads, void **out, float *grad_th, float *sigma_th) {
    OmpThreads th(nthreads);
    *out = nullptr;
    PixelData<uint16_t> in(y, x, z);
    std::memcpy(in.mesh.begin(), img, sizeof(uint16_t) * (size_t)y * x * z);
    RefHandle *h = new RefHandle();
    try {
        if (image_type == 1) {
            BlockConverter<uint16_t> c;
            set_params(c.par, p);
            c.par.auto_parameters = true;
            c.run(h->apr, in, zblock, ghost);
        } else {
            BlockConverter<float> c;
            set_params(c.par, p);
            c.par.auto_parameters = true;
            c.run(h->apr, in, zblock, ghost);
        }
    } catch (std::invalid_argument &) {
        delete h;
        return 2;
    }
    const APRParameters par = h->apr.get_apr_parameters();
    *grad_th = par.grad_th;
    *sigma_th = par.sigma_th;
    *out = h;
    return 0;
}

void ref_free(void *hv) { delete (RefHandle *)hv; }

void ref_apr_info(void *hv, int *l_min, int *l_max, uint64_t *n_level_xz, uint64_t *n_xz, uint64_t *P, float *offset) {
    RefHandle *h = (RefHandle *)hv;
    *l_min = h->apr.level_min();
    *l_max = h->apr.level_max();
    *n_level_xz = h->apr.linearAccess.level_xz_vec.size();
    *n_xz = h->apr.linearAccess.xz_end_vec.size();
    *P = h->apr.total_number_particles();
    *offset = h->offset;
}

void ref_apr_copy(void *hv, uint64_t *level_xz, uint64_t *xz_end, uint16_t *y_vec) {
    copy_access(((RefHandle *)hv)->apr.linearAccess, level_xz, xz_end, y_vec);
}

int ref_copy_intermediate(void *hv, int which, float *dst, size_t n) {
    RefHandle *h = (RefHandle *)hv;
    if (which < 1 || which > 6 || h->inter[which].size() != n) return 4;
    std::memcpy(dst, h->inter[which].data(), n * sizeof(float));
    return 0;
}

/* Builds an APR handle from externally supplied linear-access arrays. */
void *ref_apr_from_arrays(int y, int x, int z, const uint64_t *level_xz, uint64_t n_level_xz,
                          const uint64_t *xz_end, uint64_t n_xz, const uint16_t *y_vec, uint64_t P) {
    RefHandle *h = new RefHandle();
    h->apr.aprInfo.init(y, x, z);
    h->apr.linearAccess.genInfo = &h->apr.aprInfo;
    h->apr.linearAccess.level_xz_vec.resize(n_level_xz);
    std::memcpy(h->apr.linearAccess.level_xz_vec.begin(), level_xz, n_level_xz * sizeof(uint64_t));
    h->apr.linearAccess.xz_end_vec.resize(n_xz);
    std::memcpy(h->apr.linearAccess.xz_end_vec.begin(), xz_end, n_xz * sizeof(uint64_t));
    h->apr.linearAccess.y_vec.resize(P);
    std::memcpy(h->apr.linearAccess.y_vec.begin(), y_vec, P * sizeof(uint16_t));
    h->apr.aprInfo.total_number_particles = P;
    h->apr.apr_initialized = true;
    return h;
}

/* ParticleData<uint16_t>::sample_image (ParticleData.hpp:123-127) */
int ref_sample_image(void *hv, const uint16_t *img, uint16_t *parts) {
    RefHandle *h = (RefHandle *)hv;
    PixelData<uint16_t> in(h->apr.org_dims(0), h->apr.org_dims(1), h->apr.org_dims(2));
    std::memcpy(in.mesh.begin(), img, sizeof(uint16_t) * in.mesh.size());
    ParticleData<uint16_t> pd;
    pd.sample_image(h->apr, in);
    std::memcpy(parts, pd.data.begin(), sizeof(uint16_t) * pd.size());
    return 0;
}

/* APR::initialize_tree_dense, exported as arrays. */
void ref_tree_info(void *hv, uint64_t *n_level_xz, uint64_t *n_xz, uint64_t *P) {
    RefHandle *h = (RefHandle *)hv;
    h->apr.initialize_tree_linear();
    *n_level_xz = h->apr.linearAccessTree.level_xz_vec.size();
    *n_xz = h->apr.linearAccessTree.xz_end_vec.size();
    *P = h->apr.treeInfo.total_number_particles;
}

void ref_tree_copy(void *hv, uint64_t *level_xz, uint64_t *xz_end, uint16_t *y_vec) {
    RefHandle *h = (RefHandle *)hv;
    h->apr.initialize_tree_linear();
    copy_access(h->apr.linearAccessTree, level_xz, xz_end, y_vec);
}

/* APRTreeNumerics::fill_tree_mean (APRTreeNumerics.hpp:63-203) */
int ref_fill_tree_mean(void *hv, const float *parts, float *tree) {
    RefHandle *h = (RefHandle *)hv;
    ParticleData<float> in(h->apr.total_number_particles());
    std::memcpy(in.data.begin(), parts, sizeof(float) * in.size());
    ParticleData<float> td;
    APRTreeNumerics::fill_tree_mean(h->apr, in, td);
    std::memcpy(tree, td.data.begin(), sizeof(float) * td.size());
    return 0;
}

/* APRFilter::convolve_pencil (APRFilter.hpp:139-149) */
int ref_convolve_pencil(void *hv, const float *stencil, int ks, const float *in, float *out, int reflect,
                        int use_stencil_ds, int normalize) {
    RefHandle *h = (RefHandle *)hv;
    PixelData<float> st(ks, ks, ks);
    std::memcpy(st.mesh.begin(), stencil, sizeof(float) * ks * ks * ks);
    ParticleData<float> pin(h->apr.total_number_particles());
    std::memcpy(pin.data.begin(), in, sizeof(float) * pin.size());
    ParticleData<float> pout;
    APRFilter::convolve_pencil(h->apr, st, pin, pout, reflect != 0, use_stencil_ds != 0, normalize != 0);
    std::memcpy(out, pout.data.begin(), sizeof(float) * pout.size());
    return 0;
}

/* APRNumerics::gradient_cfd / gradient_sobel (APRNumerics.hpp:165-215) of
 * dimension dim, and gradient_magnitude_cfd / _sobel (:218-287) when dim < 0. */
int ref_gradient(void *hv, const float *in, float *out, int dim, int sobel, const float *deltas) {
    RefHandle *h = (RefHandle *)hv;
    ParticleData<float> pin(h->apr.total_number_particles());
    std::memcpy(pin.data.begin(), in, sizeof(float) * pin.size());
    ParticleData<float> pout;
    if (dim < 0) {
        const std::vector<float> d = {deltas[0], deltas[1], deltas[2]};
        if (sobel)
            APRNumerics::gradient_magnitude_sobel(h->apr, pin, pout, d);
        else
            APRNumerics::gradient_magnitude_cfd(h->apr, pin, pout, d);
    } else {
        if (sobel)
            APRNumerics::gradient_sobel(h->apr, pin, pout, dim, deltas[dim]);
        else
            APRNumerics::gradient_cfd(h->apr, pin, pout, dim, deltas[dim]);
    }
    std::memcpy(out, pout.data.begin(), sizeof(float) * pout.size());
    return 0;
}

/* APRNumerics::richardson_lucy (APRNumerics.hpp:576-593), FP32 or FP64. */
int ref_richardson_lucy(void *hv, const uint16_t *in, void *out, const float *psf, int ks, int niter,
                        int use_stencil_ds, int normalize, int resume, int use_double) {
    RefHandle *h = (RefHandle *)hv;
    ParticleData<uint16_t> pin(h->apr.total_number_particles());
    std::memcpy(pin.data.begin(), in, sizeof(uint16_t) * pin.size());
    if (!use_double) {
        PixelData<float> st(ks, ks, ks);
        std::memcpy(st.mesh.begin(), psf, sizeof(float) * ks * ks * ks);
        ParticleData<float> pout(h->apr.total_number_particles());
        if (resume) std::memcpy(pout.data.begin(), out, sizeof(float) * pout.size());
        APRNumerics::richardson_lucy(h->apr, pin, pout, st, niter, use_stencil_ds != 0, normalize != 0, resume != 0);
        std::memcpy(out, pout.data.begin(), sizeof(float) * pout.size());
    } else {
        PixelData<double> st(ks, ks, ks);
        for (int i = 0; i < ks * ks * ks; ++i) st.mesh[i] = (double)psf[i];
        ParticleData<double> pout(h->apr.total_number_particles());
        if (resume) std::memcpy(pout.data.begin(), out, sizeof(double) * pout.size());
        APRNumerics::richardson_lucy(h->apr, pin, pout, st, niter, use_stencil_ds != 0, normalize != 0, resume != 0);
        std::memcpy(out, pout.data.begin(), sizeof(double) * pout.size());
    }
    return 0;
}

/* ComputeGradient::get_smooth_bspline_3D on the offset image (the stage the
 * pipeline runs inside computeL, APRConverter.hpp:216-229). */
int ref_smooth(const uint16_t *img, int y, int x, int z, float lambda, int image_type, float offset, float *dst) {
    ComputeGradient cg;
    try {
        if (image_type == 1) {
            PixelData<uint16_t> im(y, x, z);
            for (size_t i = 0; i < im.mesh.size(); ++i) im.mesh[i] = (uint16_t)(img[i] + offset);
            cg.get_smooth_bspline_3D(im, lambda);
            to_float(im, dst);
        } else {
            PixelData<float> im(y, x, z);
            for (size_t i = 0; i < im.mesh.size(); ++i) im.mesh[i] = (float)img[i];
            cg.get_smooth_bspline_3D(im, lambda);
            to_float(im, dst);
        }
    } catch (std::invalid_argument &) {
        return 2;
    }
    return 0;
}

}  // extern "C"
