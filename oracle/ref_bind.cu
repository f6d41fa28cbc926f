/* TEST INFRASTRUCTURE ONLY.
 *
 * Drives include/aprb200_libapr.hpp -- the B200 path as a LibAPR build
 * includes it -- with LibAPR's own objects: compiled against the reference's
 * headers (and its GPUAccess.cu, for the GPUAccessHelper objects its GPU-form
 * functions take) into _ref/libaprbind.so by oracle/Makefile.  Each entry
 * point fills the reference's APR / ParticleData / VectorData through the
 * binding and reads them back with LibAPR's own accessors (LinearIterator),
 * so the tests compare what a LibAPR caller would see with the oracle.  No
 * reference GPU kernel runs: the helpers only carry the structure.
 */
#include <cstring>
#include <memory>

#include "apr_oracle.h"
#include "aprb200_libapr.hpp"

namespace {

struct BindAPR {
    APR apr;
    float offset = 0;
};

void set_par(APRParameters &par, const orc_params *p) {
    par.dx = p->dx; par.dy = p->dy; par.dz = p->dz;
    par.psfx = p->psfx; par.psfy = p->psfy; par.psfz = p->psfz;
    par.Ip_th = p->Ip_th; par.lambda = p->lambda; par.rel_error = p->rel_error;
    par.sigma_th = p->sigma_th; par.sigma_th_max = p->sigma_th_max; par.grad_th = p->grad_th;
    par.reflect_bc_lis = p->reflect_bc_lis != 0;
    par.neighborhood_optimization = p->neighborhood_optimization != 0;
    par.constant_intensity_scale = p->constant_intensity_scale != 0;
}

template <typename IT>
int run_get_apr(const uint16_t *img, int y, int x, int z, const orc_params *p, BindAPR &b) {
    APRConverter<IT> conv;
    set_par(conv.par, p);
    PixelData<uint16_t> in(y, x, z);
    std::memcpy(in.mesh.begin(), img, sizeof(uint16_t) * (size_t)y * x * z);
    if (!aprb200::libapr::get_apr(conv, b.apr, in)) return 1;
    b.offset = conv.bspline_offset;
    return 0;
}

template <typename T>
PixelData<float> stencil_pd(const float *st, int ks) {
    PixelData<float> s(ks, ks, ks);
    for (int i = 0; i < ks * ks * ks; ++i) s.mesh[i] = st[i];
    return s;
}

}  // namespace

extern "C" {

/* get_apr through the binding (0 ok, 1 dimension check, 2 overflow, 3 other) */
int bind_get_apr(const uint16_t *img, int y, int x, int z, const orc_params *p, int image_type, void **out,
                 uint64_t *P, float *offset) {
    std::unique_ptr<BindAPR> b(new BindAPR());
    int e;
    try {
        e = image_type == 1 ? run_get_apr<uint16_t>(img, y, x, z, p, *b) : run_get_apr<float>(img, y, x, z, p, *b);
    } catch (std::invalid_argument &) {
        return 2;
    } catch (std::exception &) {
        return 3;
    }
    if (e) return e;
    *P = b->apr.total_number_particles();
    *offset = b->offset;
    *out = b.release();
    return 0;
}

void bind_free(void *h) { delete (BindAPR *)h; }

/* APRConverterBatch<IT>::get_apr through the binding, the volume from memory */
int bind_get_apr_by_block(const uint16_t *img, int y, int x, int z, const orc_params *p, int image_type, int zblock,
                          int ghost, void **out, uint64_t *P) {
    std::unique_ptr<BindAPR> b(new BindAPR());
    PixelData<uint16_t> in(y, x, z);
    std::memcpy(in.mesh.begin(), img, sizeof(uint16_t) * (size_t)y * x * z);
    try {
        bool ok;
        if (image_type == 1) {
            APRConverterBatch<uint16_t> conv;
            set_par(conv.par, p);
            conv.z_block_size = zblock;
            conv.ghost_z = ghost;
            ok = aprb200::libapr::get_apr_by_block(conv, b->apr, in);
        } else {
            APRConverterBatch<float> conv;
            set_par(conv.par, p);
            conv.z_block_size = zblock;
            conv.ghost_z = ghost;
            ok = aprb200::libapr::get_apr_by_block(conv, b->apr, in);
        }
        if (!ok) return 1;
    } catch (std::invalid_argument &) {
        return 2;
    } catch (std::exception &) {
        return 3;
    }
    *P = b->apr.total_number_particles();
    *out = b.release();
    return 0;
}

int bind_sample_blocked(void *h, const uint16_t *img, int zblock, int ghost, uint16_t *parts) {
    APR &apr = ((BindAPR *)h)->apr;
    PixelData<uint16_t> in(apr.org_dims(0), apr.org_dims(1), apr.org_dims(2));
    std::memcpy(in.mesh.begin(), img, sizeof(uint16_t) * in.mesh.size());
    ParticleData<uint16_t> pd;
    aprb200::libapr::sample_parts_from_img_blocked(pd, apr, in, zblock, ghost);
    std::memcpy(parts, pd.data.begin(), sizeof(uint16_t) * pd.size());
    return 0;
}

/* every particle's (level, z, x, y), walked with LibAPR's LinearIterator in
 * its storage order */
int bind_particles(void *h, uint16_t *level, uint16_t *zz, uint16_t *xx, uint16_t *yy) {
    APR &apr = ((BindAPR *)h)->apr;
    auto it = apr.iterator();
    uint64_t n = 0;
    for (int l = it.level_min(); l <= it.level_max(); ++l)
        for (int z = 0; z < it.z_num(l); ++z)
            for (int x = 0; x < it.x_num(l); ++x)
                for (it.begin(l, z, x); it < it.end(); it++) {
                    if ((uint64_t)it != n) return 1;  // the iterator's global index is the storage order
                    level[n] = (uint16_t)l;
                    zz[n] = (uint16_t)z;
                    xx[n] = (uint16_t)x;
                    yy[n] = it.y();
                    ++n;
                }
    return n == apr.total_number_particles() ? 0 : 2;
}

int bind_sample(void *h, const uint16_t *img, uint16_t *parts) {
    APR &apr = ((BindAPR *)h)->apr;
    PixelData<uint16_t> in(apr.org_dims(0), apr.org_dims(1), apr.org_dims(2));
    std::memcpy(in.mesh.begin(), img, sizeof(uint16_t) * in.mesh.size());
    ParticleData<uint16_t> pd;
    aprb200::libapr::sample_image(pd, apr, in);
    std::memcpy(parts, pd.data.begin(), sizeof(uint16_t) * pd.size());
    return 0;
}

/* convolve_pencil (gpu_form 0) or isotropic_convolve_333/555 with the APR's
 * own GPUAccessHelper objects (gpu_form 1) */
int bind_convolve(void *h, const float *stencil, int ks, const float *in, float *out, int reflect, int ds,
                  int normalize, int gpu_form) {
    APR &apr = ((BindAPR *)h)->apr;
    const size_t P = apr.total_number_particles();
    PixelData<float> st = stencil_pd<float>(stencil, ks);
    try {
        if (gpu_form) {
            auto access = apr.gpuAPRHelper();
            auto tree_access = apr.gpuTreeHelper();
            VectorData<float> vin, vout, tree;
            vin.resize(P);
            std::memcpy(vin.begin(), in, P * sizeof(float));
            if (ks == 3)
                aprb200::libapr::isotropic_convolve_333(access, tree_access, vin, vout, st, tree, reflect != 0,
                                                        ds != 0, normalize != 0);
            else
                aprb200::libapr::isotropic_convolve_555(access, tree_access, vin, vout, st, tree, reflect != 0,
                                                        ds != 0, normalize != 0);
            std::memcpy(out, vout.begin(), P * sizeof(float));
        } else {
            ParticleData<float> pin, pout;
            pin.data.resize(P);
            std::memcpy(pin.data.begin(), in, P * sizeof(float));
            aprb200::libapr::convolve_pencil(apr, st, pin, pout, reflect != 0, ds != 0, normalize != 0);
            std::memcpy(out, pout.data.begin(), P * sizeof(float));
        }
    } catch (std::runtime_error &) {
        return 4;
    }
    return 0;
}

/* APRNumerics::richardson_lucy (gpu_form 0) or APRNumericsGPU::richardson_lucy
 * (gpu_form 1) through the binding, FP32 */
int bind_rl(void *h, const uint16_t *in, float *out, const float *psf, int ks, int niter, int gpu_form) {
    APR &apr = ((BindAPR *)h)->apr;
    const size_t P = apr.total_number_particles();
    PixelData<float> st = stencil_pd<float>(psf, ks);
    if (gpu_form) {
        auto access = apr.gpuAPRHelper();
        auto tree_access = apr.gpuTreeHelper();
        VectorData<uint16_t> vin;
        VectorData<float> vout;
        vin.resize(P);
        std::memcpy(vin.begin(), in, P * sizeof(uint16_t));
        aprb200::libapr::richardson_lucy_gpu(access, tree_access, vin, vout, st, niter, true, false, false);
        std::memcpy(out, vout.begin(), P * sizeof(float));
    } else {
        ParticleData<uint16_t> pin;
        ParticleData<float> pout;
        pin.data.resize(P);
        std::memcpy(pin.data.begin(), in, P * sizeof(uint16_t));
        aprb200::libapr::richardson_lucy(apr, pin, pout, st, niter, true, false, false);
        std::memcpy(out, pout.data.begin(), P * sizeof(float));
    }
    return 0;
}

}  // extern "C"
