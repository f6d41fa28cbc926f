// C ABI of libaprb200 (include/aprb200.h): handle management, host<->device
// staging and the stage order of APRConverter::get_apr_cpu
// (APRConverter.hpp:535-582).  No exception crosses the ABI: every entry
// point returns an aprb_status.
#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "kernels.cuh"

namespace aprb {

static thread_local std::string g_last_error;
static thread_local uint64_t g_launches = 0;

void set_error(const std::string &msg) { g_last_error = msg; }
void count_launch(uint64_t n) { g_launches += n; }

struct ProfRec {
    const char *name;
    cudaEvent_t a, b;
};
static thread_local bool g_prof_on = false;
static thread_local std::vector<ProfRec> g_prof;
static thread_local std::vector<size_t> g_prof_open;

void prof_record(const char *name, cudaStream_t s, bool begin) {
    if (!g_prof_on) return;
    if (begin) {
        ProfRec r{name, nullptr, nullptr};
        cudaEventCreate(&r.a);
        cudaEventCreate(&r.b);
        cudaEventRecord(r.a, s);
        g_prof.push_back(r);
        g_prof_open.push_back(g_prof.size() - 1);
    } else {
        if (g_prof_open.empty()) return;
        const size_t i = g_prof_open.back();
        g_prof_open.pop_back();
        cudaEventRecord(g_prof[i].b, s);
    }
}

void *pool_alloc(size_t bytes, cudaStream_t s) {
    int dev = 0;
    APRB_CUDA(cudaGetDevice(&dev));
    static std::mutex mu;
    static uint64_t configured = 0;  // bit per device
    {
        std::lock_guard<std::mutex> lk(mu);
        if (dev < 64 && !(configured >> dev & 1)) {
            cudaMemPool_t pool;
            APRB_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
            uint64_t keep_all = UINT64_MAX;
            APRB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep_all));
            configured |= uint64_t(1) << dev;
        }
    }
    void *p = nullptr;
    APRB_CUDA(cudaMallocAsync(&p, bytes, s));
    return p;
}

// Work buffers of the filter and sampling calls, shared by every APR that the
// calling thread uses on one device (they only live for the duration of one
// call).  Calls issued by one thread on different streams that overlap on the
// GPU share these buffers; use one thread per concurrent stream.
constexpr int kBatchWorkers = 6;  // host threads of the batch entry point
constexpr int kSampleChunk = 16;  // fewest planes per transfer chunk of host-buffer sampling (even)

// Copy streams of the calling thread and device: uploads and downloads run
// beside the compute stream.
struct Streams3 {
    cudaStream_t up = nullptr, down = nullptr;
    ~Streams3() {
        if (up) cudaStreamDestroy(up);
        if (down) cudaStreamDestroy(down);
    }
};
static Streams3 &transfer_streams() {
    thread_local std::map<int, std::unique_ptr<Streams3>> per_device;
    int dev = 0;
    APRB_CUDA(cudaGetDevice(&dev));
    auto &p = per_device[dev];
    if (!p) {
        p.reset(new Streams3());
        APRB_CUDA(cudaStreamCreateWithFlags(&p->up, cudaStreamNonBlocking));
        APRB_CUDA(cudaStreamCreateWithFlags(&p->down, cudaStreamNonBlocking));
    }
    return *p;
}

struct ThreadScratch {
    DevBuf scan_tmp, tree_vals, pyr, parts_f, parts_u16, out_f, rb, stencils, stencils_f, io_in, t_flags, obj;
    FilterBuffers fb;
    CnnScratch cnn;
};

static ThreadScratch &scratch() {
    thread_local std::map<int, std::unique_ptr<ThreadScratch>> per_device;
    int dev = 0;
    APRB_CUDA(cudaGetDevice(&dev));
    auto &p = per_device[dev];
    if (!p) p.reset(new ThreadScratch());
    return *p;
}

static void require_device() {
    static int ok = -1;
    if (ok < 0) {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
            cudaGetLastError();
            ok = 0;
        } else {
            int dev = 0, major = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
            ok = major == 10 ? 1 : 0;
        }
    }
    if (!ok) {
        set_error("no sm_100 CUDA device available");
        throw Error{APRB_ERR_NO_DEVICE};
    }
}

#define ARG_CHECK(cond, msg)                         \
    do {                                             \
        if (!(cond)) {                               \
            set_error(msg);                          \
            throw Error{APRB_ERR_INVALID_ARGUMENT};  \
        }                                            \
    } while (0)

template <typename F>
static aprb_status guarded(F &&f) {
    try {
        f();
        return APRB_OK;
    } catch (const Error &e) {
        return e.status;
    } catch (const std::bad_alloc &) {
        set_error("host allocation failed");
        return APRB_ERR_OUT_OF_MEMORY;
    } catch (...) {
        set_error("unexpected exception");
        return APRB_ERR_CUDA;
    }
}

}  // namespace aprb

using namespace aprb;

struct aprb_apr {
    Geom g{};
    int org[3] = {0, 0, 0};
    uint64_t n_xz = 0, P = 0;
    float offset = 0;
    aprb_params par{};  // the parameters it was built with (APR.hpp:61)
    DevBuf xz_end, y_vec;  // pooled
    // tree
    bool tree_built = false;
    Geom tg{};
    uint64_t t_n_xz = 0, T = 0;
    DevBuf t_xz_end, t_y_vec;  // pooled
    FilterIndex fi;
    uint64_t last_stale = 0;
    // learned proposal: level row of every particle (pooled), built on first use
    DevBuf cnn_rows;
    bool cnn_ready = false;
    // device copy of the host image it was built from (converter keep_input),
    // used and released by the first sample_image from the same host buffer
    mutable DevBuf kept_img;
    mutable const uint16_t *kept_host = nullptr;
    // No work on the APR can be pending on any stream: set at the end of the
    // host-buffer get_apr / sample_image (each synchronises before it
    // returns), cleared by every other call that touches the APR (device
    // calls on the caller's streams, exported device pointers).  A quiet APR
    // gives its pooled memory back in stream order without a device-wide
    // synchronisation, so host threads converting other volumes at the same
    // time are not stalled; otherwise freeing waits for the device, as
    // cudaFree would.
    mutable bool quiet = false;
    ~aprb_apr() {
        if (!quiet) return;
        cudaStream_t s = cudaStreamPerThread;
        for (DevBuf *b : {&xz_end, &y_vec, &t_xz_end, &t_y_vec, &cnn_rows, &kept_img}) b->release_idle(s);
    }
};

struct aprb_converter {
    int image_type = APRB_IMAGE_U16;
    int keep = 0;
    int keep_input = 0;  // hand the host call's device copy of the input to its APR
    int dims[3] = {0, 0, 0};  // y, x, z of the last call
    DevBuf img, work, grad, grad_keep, ids_raw, ids, lis, lis_keep, pyr_status, pyr_level, mm, offset, err;
    DevBuf scan_tmp, tile_pyr, iir_ckpt;
    LisBuffers lisb;
    AutoParBuffers autop;
    bool have = false;
    aprb_params last_par{};  // parameters of the last get_apr after the automatic ones
    int last_l_max = 0;
    DevBuf margins;
    // host-buffer get_apr: the device's upload lock while this call's image
    // is still crossing PCIe, and the event that marks its last chunk landed
    std::unique_lock<std::mutex> *upload_lock = nullptr;
    cudaEvent_t up_done = nullptr;
    ~aprb_converter() {
        if (up_done) cudaEventDestroy(up_done);
    }
};

// One host-buffer upload at a time per device: concurrent host get_apr calls
// (other converters on other host threads) would share the link anyway; in
// turn, each call's smoothing, construction and the other calls' particle
// downloads overlap the next call's upload.
static std::mutex &upload_mutex() {
    static std::mutex mu[64];
    int dev = 0;
    APRB_CUDA(cudaGetDevice(&dev));
    return mu[dev & 63];
}

// Called once a host-buffer get_apr has enqueued all its upload chunks and
// before its first blocking wait: waits for the last chunk and lets the next
// caller's upload start.
static void release_upload(aprb_converter *c) {
    if (!c->upload_lock) return;
    APRB_CUDA(cudaEventSynchronize(c->up_done));
    c->upload_lock->unlock();
    c->upload_lock = nullptr;
}

// reconstruct_constant / reconstruct_level on device buffers
template <typename V>
static void reconstruct_device(const aprb_apr *a, const V *parts_dev, V *img_dev, bool level, cudaStream_t s) {
    launch_reconstruct<V>(a->g, (const uint64_t *)a->xz_end.p, (const uint16_t *)a->y_vec.p, parts_dev, img_dev, level,
                          s);
}

// the same from and to host buffers (the volume's worth of pixels is copied
// back in one piece)
template <typename V>
static void reconstruct_host(const aprb_apr *a, const V *parts, V *img, bool level) {
    cudaStream_t s = cudaStreamPerThread;
    const uint64_t n = (uint64_t)a->org[0] * a->org[1] * a->org[2];
    V *dimg = (V *)scratch().out_f.get(n * sizeof(V) ? n * sizeof(V) : 16);
    const V *dparts = nullptr;
    if (!level) {
        V *dp = (V *)scratch().parts_f.get(a->P ? a->P * sizeof(V) : 16);
        if (a->P) APRB_CUDA(cudaMemcpyAsync(dp, parts, a->P * sizeof(V), cudaMemcpyHostToDevice, s));
        dparts = dp;
    }
    reconstruct_device<V>(a, dparts, dimg, level, s);
    APRB_CUDA(cudaMemcpyAsync(img, dimg, n * sizeof(V), cudaMemcpyDeviceToHost, s));
    APRB_CUDA(cudaStreamSynchronize(s));
}

extern "C" {

const char *aprb_status_string(aprb_status s) {
    switch (s) {
        case APRB_OK: return "ok";
        case APRB_ERR_INVALID_ARGUMENT: return "invalid argument";
        case APRB_ERR_DIMENSIONS: return "input dimension check failed";
        case APRB_ERR_INTEGER_OVERFLOW: return "integer under-/overflow in the B-spline smoothing";
        case APRB_ERR_UNSUPPORTED: return "unsupported configuration";
        case APRB_ERR_OUT_OF_MEMORY: return "out of memory";
        case APRB_ERR_CUDA: return "CUDA error";
        case APRB_ERR_NO_DEVICE: return "no sm_100 CUDA device";
        case APRB_ERR_INCOMPLETE_NEIGHBOURHOOD: return "filter neighbourhood not covered by particles";
    }
    return "unknown status";
}

const char *aprb_last_error(void) { return g_last_error.c_str(); }
uint64_t aprb_kernel_launch_count(void) { return g_launches; }

aprb_status aprb_measure_fp32_fma_peak(void *stream, double *tflops) {
    return guarded([&] {
        require_device();
        ARG_CHECK(tflops, "null argument");
        *tflops = measure_fp32_fma_tflops((cudaStream_t)stream);
    });
}

aprb_status aprb_check_division_by_constant(float d, uint64_t *mismatches, uint32_t *first_bits) {
    return guarded([&] {
        require_device();
        ARG_CHECK(mismatches && first_bits, "null argument");
        cudaStream_t s = cudaStreamPerThread;
        unsigned long long *dev = (unsigned long long *)scratch().obj.get(2 * sizeof(unsigned long long));
        const unsigned long long init[2] = {0ull, ~0ull};
        APRB_CUDA(cudaMemcpyAsync(dev, init, sizeof(init), cudaMemcpyHostToDevice, s));
        launch_check_div_const(d, dev, s);
        unsigned long long h[2];
        APRB_CUDA(cudaMemcpyAsync(h, dev, sizeof(h), cudaMemcpyDeviceToHost, s));
        APRB_CUDA(cudaStreamSynchronize(s));
        *mismatches = h[0];
        *first_bits = h[1] == ~0ull ? 0u : (uint32_t)h[1];
    });
}

aprb_status aprb_profile_enable(int on) {
    g_prof_on = on != 0;
    return APRB_OK;
}

aprb_status aprb_profile_reset(void) {
    for (auto &r : g_prof) {
        cudaEventSynchronize(r.b);
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    g_prof.clear();
    g_prof_open.clear();
    return APRB_OK;
}

int aprb_profile_read(const char **names, double *ms, uint64_t *count, int max) {
    std::vector<const char *> order;
    std::vector<double> tot;
    std::vector<uint64_t> cnt;
    for (auto &r : g_prof) {
        cudaEventSynchronize(r.b);
        float t = 0;
        if (cudaEventElapsedTime(&t, r.a, r.b) != cudaSuccess) {
            cudaGetLastError();
            t = 0;
        }
        size_t j = 0;
        while (j < order.size() && std::strcmp(order[j], r.name) != 0) ++j;
        if (j == order.size()) {
            order.push_back(r.name);
            tot.push_back(0);
            cnt.push_back(0);
        }
        tot[j] += t;
        cnt[j] += 1;
    }
    int n = (int)order.size() < max ? (int)order.size() : max;
    for (int i = 0; i < n; ++i) {
        if (names) names[i] = order[i];
        if (ms) ms[i] = tot[i];
        if (count) count[i] = cnt[i];
    }
    return n;
}

void aprb_default_params(aprb_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->dx = p->dy = p->dz = 1;
    p->psfx = p->psfy = p->psfz = 2;
    p->Ip_th = 0;
    p->lambda = 3.0f;
    p->rel_error = 0.1f;
    p->sigma_th = 0;
    p->sigma_th_max = 0;
    p->grad_th = 0;
    p->reflect_bc_lis = 1;
    p->neighborhood_optimization = 1;
    p->constant_intensity_scale = 0;
    p->check_input = 0;
    p->swap_dimensions = 0;
    p->auto_parameters = 0;
}

aprb_status aprb_converter_create(int image_type, aprb_converter **out) {
    return guarded([&] {
        ARG_CHECK(out, "null output pointer");
        ARG_CHECK(image_type == APRB_IMAGE_U16 || image_type == APRB_IMAGE_FLOAT, "image_type must be 0 or 1");
        auto *c = new aprb_converter();
        c->image_type = image_type;
        *out = c;
    });
}

aprb_status aprb_converter_destroy(aprb_converter *c) {
    delete c;
    return APRB_OK;
}

aprb_status aprb_converter_keep_intermediates(aprb_converter *c, int keep) {
    return guarded([&] {
        ARG_CHECK(c, "null converter");
        c->keep = keep != 0;
    });
}

}  // extern "C"

namespace {

// APRConverter::check_input_dimensions (APRConverter.hpp:606-640)
bool check_dims(const aprb_params &p, int &y, int &x, int &z) {
    const int nd = (x > 1) + (y > 1) + (z > 1);
    if (nd == 0) return false;
    if (nd == 3) return true;
    if (y > 1) return true;
    if (p.swap_dimensions) {
        if (x > 1)
            std::swap(x, y);
        else
            std::swap(z, y);
        return true;
    }
    return false;
}

// Pixel stages of one image -- the whole volume, or one z-tile of the blocked
// converter (APRConverterBatch.hpp:190-271): offset, smoothing, gradient +
// ds image, inverse B-spline, local intensity scale.  Overflow is accumulated
// in the converter's error flag, which the caller clears and reads.
template <typename IT>
struct PixelOut {
    IT *grad;
    float *lis, *ids;
    const float *d_off;
    uint64_t nd;
};

// With `host` set, img is the device buffer that the volume is copied into
// from host memory, chunk by chunk on stream `up`, overlapped with smoothing.
template <typename IT>
PixelOut<IT> pixel_stages(aprb_converter *c, const aprb_params &p, const uint16_t *img, int yn, int xn, int zn,
                          cudaStream_t s, const uint16_t *host = nullptr, cudaStream_t up = nullptr) {
    const int yd = (yn + 1) / 2, xd = (xn + 1) / 2, zd = (zn + 1) / 2;
    const uint64_t n = (uint64_t)yn * xn * zn, nd = (uint64_t)yd * xd * zd;
    const bool is_u16 = sizeof(IT) == 2;
    unsigned *mm = c->mm.as_on<unsigned>(2, s);
    float *d_off = c->offset.as_on<float>(1, s);
    unsigned *d_err = c->err.as_on<unsigned>(2, s);  // [0] overflow count, [1] TMA wait timeout
    IT *work = c->work.as_on<IT>(n, s);
    if (host) {
        launch_upload_smooth<IT>(host, const_cast<uint16_t *>(img), work, yn, xn, zn, p.lambda, mm, d_off,
                                 is_u16 && p.lambda > 0, d_err, c->iir_ckpt, s, up);
        if (c->upload_lock) {
            if (!c->up_done) APRB_CUDA(cudaEventCreateWithFlags(&c->up_done, cudaEventDisableTiming));
            APRB_CUDA(cudaEventRecord(c->up_done, up));  // after the last chunk's copy
        }
    } else {
        launch_minmax_offset(img, n, mm, d_off, is_u16 && p.lambda > 0, s);
        launch_smooth<IT>(img, work, yn, xn, zn, p.lambda, d_off, d_err, c->iir_ckpt, s);
    }
    IT *grad = c->grad.as_on<IT>(nd, s);
    float *ids_raw = c->ids_raw.as_on<float>(nd, s);
    float *ids = c->ids.as_on<float>(nd, s);
    launch_gradient<IT>(work, yn, xn, zn, grad, ids_raw, ids, yd, xd, zd, p, d_err + 1, s);
    float *lis = c->lis.as_on<float>(nd, s);
    launch_local_intensity_scale(ids, lis, yd, xd, zd, p, c->lisb, s);
    return PixelOut<IT>{grad, lis, ids, d_off, nd};
}

void throw_if_overflow(aprb_converter *c, cudaStream_t s) {
    unsigned h[2] = {0, 0};
    APRB_CUDA(cudaMemcpyAsync(h, c->err.p, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    APRB_CUDA(cudaStreamSynchronize(s));
    if (h[1]) {
        set_error("a bounded wait for a TMA copy in the B-spline smoothing ran out");
        throw Error{APRB_ERR_CUDA};
    }
    const unsigned h_err = h[0];
    if (h_err) {
        set_error("integer under-/overflow encountered in the B-spline smoothing");
        throw Error{APRB_ERR_INTEGER_OVERFLOW};
    }
}

// Linear access structure from the solved particle-cell pyramid
// (generateDatastructures, APRConverter.hpp:339-363); reads the overflow
// flag before the particle count is trusted.
void build_structure(aprb_converter *c, const aprb_params &p, Pyramid &pm, aprb_apr *a, cudaStream_t s) {
    release_upload(c);
    const Geom &g = a->g;
    const int L = g.l_max;
    uint64_t *xz_end = a->xz_end.as_pooled<uint64_t>(a->n_xz, s);
    const int min_type = p.neighborhood_optimization ? 1 : 2;
    if (L <= 2) {
        APRB_CUDA(cudaMemsetAsync(xz_end, 0, a->n_xz * sizeof(uint64_t), s));
        launch_full_resolution_structure(g, xz_end, nullptr, s);
        a->P = (uint64_t)g.y_num[L] * g.x_num[L] * g.z_num[L];
        throw_if_overflow(c, s);
        uint16_t *yv = a->y_vec.as_pooled<uint16_t>(a->P, s);
        launch_full_resolution_structure(g, xz_end, yv, s);
    } else {
        a->P = launch_linear_counts(g, pm, xz_end, a->n_xz, min_type, c->scan_tmp, s);
        throw_if_overflow(c, s);
        uint16_t *yv = a->y_vec.as_pooled<uint16_t>(a->P ? a->P : 1, s);
        launch_linear_fill(g, pm, xz_end, yv, min_type, s);
    }
    APRB_CUDA(cudaMemcpyAsync(&a->offset, c->offset.p, sizeof(float), cudaMemcpyDeviceToHost, s));
    APRB_CUDA(cudaStreamSynchronize(s));
}

// autoParametersLiEntropy before applyParameters (APRConverter.hpp:556-561,
// APRConverterBatch.hpp:243-247): image = local_scale_temp2 (ids).
template <typename IT>
void apply_auto_parameters(aprb_converter *c, aprb_params &p, const PixelOut<IT> &po, cudaStream_t s) {
    if (!p.auto_parameters) return;
    auto_parameters<IT>(po.ids, po.grad, po.lis, po.nd, po.d_off, p.Ip_th, sizeof(IT) == 2, c->autop, s,
                        &p.grad_th, &p.sigma_th, nullptr);
}

template <typename IT>
void run_get_apr(aprb_converter *c, aprb_params p, const uint16_t *img, int yn, int xn, int zn,
                 cudaStream_t s, aprb_apr *a, const uint16_t *host = nullptr, cudaStream_t up = nullptr) {
    Geom &g = a->g;
    a->n_xz = apr_geometry(yn, xn, zn, g);
    a->org[0] = yn;
    a->org[1] = xn;
    a->org[2] = zn;
    const int L = g.l_max;
    const uint64_t nd = (uint64_t)((yn + 1) / 2) * ((xn + 1) / 2) * ((zn + 1) / 2);
    APRB_CUDA(cudaMemsetAsync(c->err.as_on<unsigned>(2, s), 0, 2 * sizeof(unsigned), s));
    PixelOut<IT> po = pixel_stages<IT>(c, p, img, yn, xn, zn, s, host, up);
    IT *grad = po.grad;
    float *lis = po.lis, *ids = po.ids;
    const float *d_off = po.d_off;
    if (c->keep) {
        APRB_CUDA(cudaMemcpyAsync(c->grad_keep.as_on<IT>(nd, s), grad, nd * sizeof(IT), cudaMemcpyDeviceToDevice, s));
        APRB_CUDA(cudaMemcpyAsync(c->lis_keep.as_on<float>(nd, s), lis, nd * sizeof(float), cudaMemcpyDeviceToDevice, s));
    }
    apply_auto_parameters<IT>(c, p, po, s);
    a->par = p;

    // particle-cell pyramid: pct levels l_min..L-1 (PullingScheme.hpp:92-104)
    Pyramid pm;
    const int top = L - 1;
    uint64_t tot = 0, off[32] = {};
    for (int l = g.l_min; l <= top; ++l) {
        off[l] = tot;
        tot += ((uint64_t)g.y_num[l] * g.x_num[l] * g.z_num[l] + 15) & ~uint64_t(15);
    }
    uint8_t *st = c->pyr_status.as_on<uint8_t>(tot ? tot : 16, s);
    uint8_t *lv = c->pyr_level.as_on<uint8_t>(tot ? tot : 16, s);
    for (int l = g.l_min; l <= top; ++l) {
        pm.status[l] = st + off[l];
        pm.level[l] = lv + off[l];
    }
    if (top >= g.l_min) {
        launch_levels<IT>(grad, lis, ids, nd, d_off, p, L, top, pm.level[top], pm.status[top], c->keep, s);
    } else {
        uint8_t *lvl = c->pyr_level.as_on<uint8_t>(nd, s), *sts = c->pyr_status.as_on<uint8_t>(nd, s);
        launch_levels<IT>(grad, lis, ids, nd, d_off, p, L, top, lvl, sts, c->keep, s);
    }
    if (L > 2) launch_pulling_scheme(g, pm, s);
    build_structure(c, p, pm, a, s);
    c->last_par = p;
    c->last_l_max = L;
    c->dims[0] = yn;
    c->dims[1] = xn;
    c->dims[2] = zn;
    c->have = true;
}

// APRConverterBatch<IT> (APRConverterBatch.hpp:114-175): the pixel stages and
// levels per z-tile with ghost planes, each tile filling the global
// particle-cell pyramid (fill_global_particle_cell_tree, :282-314), then one
// pulling scheme and one linear structure for the volume.
// Particle-cell pyramid of the blocked converter: pct levels l_min .. l_max - 1
// in one buffer, each level padded to 16 bytes.
uint64_t pyramid_layout(const Geom &g, uint8_t *base, Pyramid *pm) {
    uint64_t tot = 0;
    for (int l = g.l_min; l <= g.l_max - 1; ++l) {
        if (pm) pm->status[l] = base + tot;
        tot += ((uint64_t)g.y_num[l] * g.x_num[l] * g.z_num[l] + 15) & ~uint64_t(15);
    }
    return tot;
}

// get_apr_method_patch for z-tiles [first, first + count) of the volume's
// blocked tiling, each filling the global particle-cell pyramid
// (fill_global_particle_cell_tree); the tiles' planes, ghosts included, are
// read from slab, which holds planes [slab_z0, ...) of the volume.
template <typename IT>
void fill_tiles(aprb_converter *c, aprb_params &p, const Geom &g, Pyramid &pm, const uint16_t *slab, int slab_z0,
                int yn, int xn, int zn, int zblock, int ghost, int first, int count, cudaStream_t s) {
    const int L = g.l_max, top = L - 1;
    const int nb = std::max(zn / zblock, 1);
    for (int b = first; b < first + count && b < nb; ++b) {
        const ZTile t = z_tile(b, nb, zn, zblock, ghost);
        PixelOut<IT> po =
            pixel_stages<IT>(c, p, slab + (uint64_t)(t.z0 - t.gl - slab_z0) * xn * yn, yn, xn, t.pz, s);
        apply_auto_parameters<IT>(c, p, po, s);
        uint8_t *lev = c->pyr_level.as_on<uint8_t>(po.nd, s);
        launch_levels<IT>(po.grad, po.lis, po.ids, po.nd, po.d_off, p, L, top, lev, nullptr, 0, s);
        launch_fill_patch(g, pm, lev, t, c->tile_pyr, s);
    }
}

// pulling scheme and linear structure of a filled pyramid (consumed)
void apr_from_pyramid(aprb_converter *c, const aprb_params &p, Pyramid &pm, aprb_apr *a, cudaStream_t s) {
    if (a->g.l_max > 2) launch_pulling_scheme(a->g, pm, s, false);
    build_structure(c, p, pm, a, s);
    a->par = p;  // the last tile's thresholds, as the reference's par keeps them
    c->have = false;  // intermediates are per tile
}

void init_apr_geometry(aprb_apr *a, int yn, int xn, int zn) {
    a->n_xz = apr_geometry(yn, xn, zn, a->g);
    a->org[0] = yn;
    a->org[1] = xn;
    a->org[2] = zn;
}

// APRConverterBatch<IT> (APRConverterBatch.hpp:114-175): the pixel stages and
// levels per z-tile with ghost planes, each tile filling the global
// particle-cell pyramid (fill_global_particle_cell_tree, :282-314), then one
// pulling scheme and one linear structure for the volume.
template <typename IT>
void run_get_apr_by_block(aprb_converter *c, aprb_params p, const uint16_t *img, int yn, int xn, int zn,
                          int zblock, int ghost, cudaStream_t s, aprb_apr *a) {
    init_apr_geometry(a, yn, xn, zn);
    APRB_CUDA(cudaMemsetAsync(c->err.as_on<unsigned>(2, s), 0, 2 * sizeof(unsigned), s));
    Pyramid pm;
    const uint64_t tot = pyramid_layout(a->g, nullptr, nullptr);
    uint8_t *st = c->pyr_status.as_on<uint8_t>(tot ? tot : 16, s);
    APRB_CUDA(cudaMemsetAsync(st, 0, tot ? tot : 16, s));
    pyramid_layout(a->g, st, &pm);
    fill_tiles<IT>(c, p, a->g, pm, img, 0, yn, xn, zn, zblock, ghost, 0, std::max(zn / zblock, 1), s);
    apr_from_pyramid(c, p, pm, a, s);
}

void get_apr_impl(aprb_converter *c, const aprb_params *p, const uint16_t *img_dev, int y, int x, int z,
                  cudaStream_t s, aprb_apr **out, const uint16_t *host = nullptr, cudaStream_t up = nullptr) {
    require_device();
    ARG_CHECK(c && p && img_dev && out, "null argument");
    ARG_CHECK(y >= 1 && x >= 1 && z >= 1, "dimensions must be positive");
    ARG_CHECK(y <= 65535 && x <= 65535 && z <= 65535, "each dimension must fit the uint16 coordinates");
    aprb_params par = *p;
    if (par.check_input && !check_dims(par, y, x, z)) {
        set_error("Input dimension check failed");
        throw Error{APRB_ERR_DIMENSIONS};
    }
    ARG_CHECK(par.rel_error > 0, "rel_error must be positive");
    std::unique_ptr<aprb_apr> a(new aprb_apr());
    if (c->image_type == APRB_IMAGE_U16)
        run_get_apr<uint16_t>(c, par, img_dev, y, x, z, s, a.get(), host, up);
    else
        run_get_apr<float>(c, par, img_dev, y, x, z, s, a.get(), host, up);
    *out = a.release();
}

void get_apr_by_block_impl(aprb_converter *c, const aprb_params *p, const uint16_t *img_dev, int y, int x, int z,
                           int zblock, int ghost, cudaStream_t s, aprb_apr **out) {
    require_device();
    ARG_CHECK(c && p && img_dev && out, "null argument");
    ARG_CHECK(y >= 1 && x >= 1 && z >= 1, "dimensions must be positive");
    ARG_CHECK(y <= 65535 && x <= 65535 && z <= 65535, "each dimension must fit the uint16 coordinates");
    ARG_CHECK(zblock >= 1 && ghost >= 0, "z_block_size must be positive and ghost_z non-negative");
    ARG_CHECK(p->rel_error > 0, "rel_error must be positive");
    std::unique_ptr<aprb_apr> a(new aprb_apr());
    if (c->image_type == APRB_IMAGE_U16)
        run_get_apr_by_block<uint16_t>(c, *p, img_dev, y, x, z, zblock, ghost, s, a.get());
    else
        run_get_apr_by_block<float>(c, *p, img_dev, y, x, z, zblock, ghost, s, a.get());
    *out = a.release();
}

}  // namespace

extern "C" {

aprb_status aprb_get_apr_by_block_device(aprb_converter *c, const aprb_params *p, const uint16_t *img_dev, int y_num,
                                         int x_num, int z_num, int z_block_size, int ghost_z, void *stream,
                                         aprb_apr **out) {
    return guarded([&] {
        get_apr_by_block_impl(c, p, img_dev, y_num, x_num, z_num, z_block_size, ghost_z, (cudaStream_t)stream, out);
    });
}

aprb_status aprb_get_apr_by_block(aprb_converter *c, const aprb_params *p, const uint16_t *img, int y_num, int x_num,
                                  int z_num, int z_block_size, int ghost_z, aprb_apr **out) {
    return guarded([&] {
        require_device();
        ARG_CHECK(c && img, "null argument");
        const uint64_t n = (uint64_t)y_num * x_num * z_num;
        cudaStream_t s = cudaStreamPerThread;
        uint16_t *d = c->img.as_on<uint16_t>(n, s);
        APRB_CUDA(cudaMemcpyAsync(d, img, n * sizeof(uint16_t), cudaMemcpyHostToDevice, s));
        get_apr_by_block_impl(c, p, d, y_num, x_num, z_num, z_block_size, ghost_z, s, out);
    });
}

aprb_status aprb_pyramid_bytes(int y_num, int x_num, int z_num, uint64_t *bytes) {
    return guarded([&] {
        ARG_CHECK(bytes && y_num >= 1 && x_num >= 1 && z_num >= 1, "invalid argument");
        Geom g;
        apr_geometry(y_num, x_num, z_num, g);
        const uint64_t tot = pyramid_layout(g, nullptr, nullptr);
        *bytes = tot ? tot : 16;
    });
}

aprb_status aprb_pyramid_fill_tiles_device(aprb_converter *c, const aprb_params *p, uint8_t *pyramid_dev, int y_num,
                                           int x_num, int z_num, int z_block_size, int ghost_z, int first_tile,
                                           int n_tiles, const uint16_t *slab_dev, int slab_z0, int slab_z_num,
                                           void *stream) {
    return guarded([&] {
        require_device();
        ARG_CHECK(c && p && pyramid_dev && slab_dev, "null argument");
        ARG_CHECK(y_num >= 1 && x_num >= 1 && z_num >= 1 && y_num <= 65535 && x_num <= 65535 && z_num <= 65535,
                  "invalid dimensions");
        ARG_CHECK(z_block_size >= 1 && ghost_z >= 0 && p->rel_error > 0, "invalid tiling or parameters");
        const int nb = std::max(z_num / z_block_size, 1);
        ARG_CHECK(first_tile >= 0 && n_tiles >= 0 && first_tile + n_tiles <= nb, "tile range outside the tiling");
        if (n_tiles == 0) return;
        const ZTile t0 = z_tile(first_tile, nb, z_num, z_block_size, ghost_z);
        const ZTile t1 = z_tile(first_tile + n_tiles - 1, nb, z_num, z_block_size, ghost_z);
        ARG_CHECK(slab_z0 <= t0.z0 - t0.gl && t1.zf + t1.gr <= slab_z0 + slab_z_num,
                  "the slab does not hold the tiles' planes and ghosts");
        cudaStream_t s = (cudaStream_t)stream;
        Geom g;
        apr_geometry(y_num, x_num, z_num, g);
        Pyramid pm;
        pyramid_layout(g, pyramid_dev, &pm);
        APRB_CUDA(cudaMemsetAsync(c->err.as_on<unsigned>(2, s), 0, 2 * sizeof(unsigned), s));
        aprb_params par = *p;
        if (c->image_type == APRB_IMAGE_U16)
            fill_tiles<uint16_t>(c, par, g, pm, slab_dev, slab_z0, y_num, x_num, z_num, z_block_size, ghost_z,
                                 first_tile, n_tiles, s);
        else
            fill_tiles<float>(c, par, g, pm, slab_dev, slab_z0, y_num, x_num, z_num, z_block_size, ghost_z,
                              first_tile, n_tiles, s);
        throw_if_overflow(c, s);
    });
}

aprb_status aprb_get_apr_from_pyramid_device(aprb_converter *c, const aprb_params *p, uint8_t *pyramid_dev, int y_num,
                                             int x_num, int z_num, void *stream, aprb_apr **out) {
    return guarded([&] {
        require_device();
        ARG_CHECK(c && p && pyramid_dev && out, "null argument");
        ARG_CHECK(y_num >= 1 && x_num >= 1 && z_num >= 1 && y_num <= 65535 && x_num <= 65535 && z_num <= 65535,
                  "invalid dimensions");
        cudaStream_t s = (cudaStream_t)stream;
        std::unique_ptr<aprb_apr> a(new aprb_apr());
        init_apr_geometry(a.get(), y_num, x_num, z_num);
        APRB_CUDA(cudaMemsetAsync(c->err.as_on<unsigned>(2, s), 0, 2 * sizeof(unsigned), s));
        Pyramid pm;
        pyramid_layout(a->g, pyramid_dev, &pm);
        apr_from_pyramid(c, *p, pm, a.get(), s);
        *out = a.release();
    });
}

aprb_status aprb_get_apr_batch_device(aprb_converter *c, const aprb_params *p, int n_volumes,
                                      const aprb_volume *volumes, int z_block_size, int ghost_z, void *stream,
                                      aprb_apr **outs) {
    return guarded([&] {
        require_device();
        ARG_CHECK(c && p && n_volumes >= 0 && (n_volumes == 0 || (volumes && outs)), "invalid volume list");
        for (int i = 0; i < n_volumes; ++i) outs[i] = nullptr;
        if (n_volumes == 0) return;
        // the inputs are ready once the caller's stream is
        APRB_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
        int dev = 0;
        APRB_CUDA(cudaGetDevice(&dev));
        // Volumes are independent: kBatchWorkers host threads, each with its
        // own converter (same ImageType) and stream, take volumes in turn, so
        // the small volumes' launches and particle-count reads overlap.
        const int nw = std::min(n_volumes, kBatchWorkers);
        std::vector<aprb_status> st(nw, APRB_OK);
        std::vector<std::string> msg(nw);
        std::atomic<int> next(0);
        auto work = [&](int w) {
            cudaSetDevice(dev);
            aprb_converter wc;
            wc.image_type = c->image_type;
            cudaStream_t ws = nullptr;
            st[w] = guarded([&] {
                APRB_CUDA(cudaStreamCreateWithFlags(&ws, cudaStreamNonBlocking));
                for (int i = next.fetch_add(1); i < n_volumes; i = next.fetch_add(1))
                    get_apr_by_block_impl(&wc, p, volumes[i].img_dev, volumes[i].y_num, volumes[i].x_num,
                                          volumes[i].z_num, z_block_size, ghost_z, ws, &outs[i]);
            });
            if (st[w] != APRB_OK) msg[w] = aprb_last_error();
            if (ws) {
                cudaStreamSynchronize(ws);
                cudaStreamDestroy(ws);
            }
        };
        std::vector<std::thread> threads;
        for (int w = 1; w < nw; ++w) threads.emplace_back(work, w);
        work(0);
        for (auto &t : threads) t.join();
        for (int w = 0; w < nw; ++w)
            if (st[w] != APRB_OK) {
                for (int i = 0; i < n_volumes; ++i) {
                    delete outs[i];
                    outs[i] = nullptr;
                }
                set_error(msg[w]);
                throw Error{st[w]};
            }
    });
}

aprb_status aprb_get_apr_device(aprb_converter *c, const aprb_params *p, const uint16_t *img_dev, int y_num,
                                int x_num, int z_num, void *stream, aprb_apr **out) {
    return guarded([&] { get_apr_impl(c, p, img_dev, y_num, x_num, z_num, (cudaStream_t)stream, out); });
}

aprb_status aprb_get_apr(aprb_converter *c, const aprb_params *p, const uint16_t *img, int y_num, int x_num,
                         int z_num, aprb_apr **out) {
    return guarded([&] {
        require_device();
        ARG_CHECK(c && img, "null argument");
        const uint64_t n = (uint64_t)y_num * x_num * z_num;
        cudaStream_t s = cudaStreamPerThread;
        uint16_t *d = c->img.as_on<uint16_t>(n, s);
        // the copy goes in z-chunks on the transfer stream, overlapped with
        // the smoothing of the chunks already on the device
        cudaStream_t up = transfer_streams().up;
        std::unique_lock<std::mutex> lk(upload_mutex());  // released once this call's upload has landed
        c->upload_lock = &lk;
        try {
            get_apr_impl(c, p, d, y_num, x_num, z_num, s, out, img, up);
        } catch (...) {
            c->upload_lock = nullptr;
            cudaStreamSynchronize(up);  // no copy from the caller's buffer outlives the call
            throw;
        }
        c->upload_lock = nullptr;
        if (c->keep_input) {
            (*out)->kept_img.swap(c->img);
            (*out)->kept_host = img;
        }
        (*out)->quiet = true;  // get_apr_impl synchronised its streams
    });
}

aprb_status aprb_converter_keep_input(aprb_converter *c, int keep) {
    return guarded([&] {
        ARG_CHECK(c, "null argument");
        c->keep_input = keep != 0;
    });
}

aprb_status aprb_converter_intermediate(const aprb_converter *c, int stage, float *dst, size_t n) {
    return guarded([&] {
        ARG_CHECK(c && dst, "null argument");
        ARG_CHECK(c->have && c->keep, "no intermediates kept (enable aprb_converter_keep_intermediates first)");
        const int y = c->dims[0], x = c->dims[1], z = c->dims[2];
        const uint64_t full = (uint64_t)y * x * z;
        const uint64_t nd = (uint64_t)((y + 1) / 2) * ((x + 1) / 2) * ((z + 1) / 2);
        const bool u16 = c->image_type == APRB_IMAGE_U16;
        const void *src = nullptr;
        int kind = 0;  // 0 IT, 1 float, 2 uint8
        uint64_t cnt = nd;
        switch (stage) {
            case APRB_STAGE_SMOOTHED: src = c->work.p; cnt = full; kind = 0; break;
            case APRB_STAGE_GRADIENT: src = c->grad_keep.p; kind = 0; break;
            case APRB_STAGE_DS_IMAGE: src = c->ids.p; kind = 1; break;
            case APRB_STAGE_LOCAL_SCALE: src = c->lis_keep.p; kind = 1; break;
            case APRB_STAGE_GRADIENT_APPLIED: src = c->grad.p; kind = 0; break;
            case APRB_STAGE_SCALE_APPLIED: src = c->lis.p; kind = 1; break;
            case APRB_STAGE_LEVELS: {
                Geom g;
                apr_geometry(y, x, z, g);
                const int top = g.l_max - 1;
                uint64_t o = 0;
                for (int l = g.l_min; l < top; ++l) o += ((uint64_t)g.y_num[l] * g.x_num[l] * g.z_num[l] + 15) & ~uint64_t(15);
                src = (const uint8_t *)c->pyr_level.p + (top >= g.l_min ? o : 0);
                kind = 2;
                break;
            }
            default: ARG_CHECK(false, "unknown stage");
        }
        ARG_CHECK(n == cnt, "element count does not match the stage size");
        if (kind == 1) {
            APRB_CUDA(cudaMemcpy(dst, src, cnt * sizeof(float), cudaMemcpyDeviceToHost));
        } else if (kind == 2) {
            std::vector<uint8_t> h(cnt);
            APRB_CUDA(cudaMemcpy(h.data(), src, cnt, cudaMemcpyDeviceToHost));
            for (uint64_t i = 0; i < cnt; ++i) dst[i] = (float)h[i];
        } else if (u16) {
            std::vector<uint16_t> h(cnt);
            APRB_CUDA(cudaMemcpy(h.data(), src, cnt * sizeof(uint16_t), cudaMemcpyDeviceToHost));
            for (uint64_t i = 0; i < cnt; ++i) dst[i] = (float)h[i];
        } else {
            APRB_CUDA(cudaMemcpy(dst, src, cnt * sizeof(float), cudaMemcpyDeviceToHost));
        }
    });
}

aprb_status aprb_smoothing_variants(int axis, int *count) {
    return guarded([&] {
        ARG_CHECK(count && axis >= 0 && axis <= 2, "axis must be 0 (y), 1 (x) or 2 (z)");
        *count = smoothing_variants(axis);
    });
}

aprb_status aprb_smoothing_schedule_set(int axis, int bucket, int variant) {
    return guarded([&] {
        ARG_CHECK(set_smoothing_variant(axis, bucket, variant), "axis, bucket or variant out of range");
    });
}

aprb_status aprb_smoothing_schedule_get(int axis, int bucket, int *variant) {
    return guarded([&] {
        ARG_CHECK(variant && axis >= 0 && axis <= 2 && bucket >= 0 && bucket < kSchedBuckets,
                  "axis or bucket out of range");
        *variant = smoothing_variant(axis, bucket == 0 ? 1 : (64 << bucket) + 1);
    });
}

aprb_status aprb_converter_level_margins(aprb_converter *c, double rel_tol, uint64_t *near_boundary,
                                         uint64_t *active) {
    return guarded([&] {
        ARG_CHECK(c && near_boundary && active, "null argument");
        ARG_CHECK(rel_tol >= 0.0, "rel_tol must be >= 0");
        ARG_CHECK(c->have && c->keep, "no intermediates kept (enable aprb_converter_keep_intermediates first)");
        require_device();
        const int y = c->dims[0], x = c->dims[1], z = c->dims[2];
        const uint64_t nd = (uint64_t)((y + 1) / 2) * ((x + 1) / 2) * ((z + 1) / 2);
        cudaStream_t s = cudaStreamPerThread;
        unsigned long long *cnt = c->margins.as_on<unsigned long long>(2, s);
        if (c->image_type == APRB_IMAGE_U16)
            launch_level_margins<uint16_t>((const uint16_t *)c->grad.p, (const float *)c->lis.p, nd, c->last_par,
                                           c->last_l_max, rel_tol, cnt, s);
        else
            launch_level_margins<float>((const float *)c->grad.p, (const float *)c->lis.p, nd, c->last_par,
                                        c->last_l_max, rel_tol, cnt, s);
        unsigned long long h[2];
        APRB_CUDA(cudaMemcpyAsync(h, cnt, sizeof(h), cudaMemcpyDeviceToHost, s));
        APRB_CUDA(cudaStreamSynchronize(s));
        *near_boundary = h[0];
        *active = h[1];
    });
}

aprb_status aprb_apr_free(aprb_apr *a) {
    delete a;
    return APRB_OK;
}

aprb_status aprb_apr_get_parameters(const aprb_apr *a, aprb_params *par) {
    return guarded([&] {
        ARG_CHECK(a && par, "null argument");
        *par = a->par;
    });
}

aprb_status aprb_threshold_li(const float *values, uint64_t n, int integer_values, float *threshold) {
    return guarded([&] {
        require_device();
        ARG_CHECK(threshold && (values || n == 0), "null argument");
        cudaStream_t s = cudaStreamPerThread;
        AutoParBuffers b;
        float *v = n ? b.sub_g.as_on<float>(n, s) : nullptr;
        if (n) APRB_CUDA(cudaMemcpyAsync(v, values, n * sizeof(float), cudaMemcpyHostToDevice, s));
        const float *vv[2] = {v, v};
        const int integer[2] = {integer_values != 0, 0}, active[2] = {1, 0};
        float out[2];
        threshold_li_pair(vv, n, integer, active, b, s, out);
        *threshold = out[0];
    });
}

aprb_status aprb_auto_parameters(aprb_params *par, const float *image, const float *lis, const float *grad,
                                 uint64_t n, int grad_integer, float bspline_offset) {
    return guarded([&] {
        require_device();
        ARG_CHECK(par && ((image && lis && grad) || n == 0), "null argument");
        cudaStream_t s = cudaStreamPerThread;
        AutoParBuffers b;
        DevBuf d_img, d_lis, d_grad, d_off;
        float *di = d_img.as_on<float>(n ? n : 1, s), *dl = d_lis.as_on<float>(n ? n : 1, s);
        float *dg = d_grad.as_on<float>(n ? n : 1, s), *doff = d_off.as_on<float>(1, s);
        if (n) {
            APRB_CUDA(cudaMemcpyAsync(di, image, n * sizeof(float), cudaMemcpyHostToDevice, s));
            APRB_CUDA(cudaMemcpyAsync(dl, lis, n * sizeof(float), cudaMemcpyHostToDevice, s));
            APRB_CUDA(cudaMemcpyAsync(dg, grad, n * sizeof(float), cudaMemcpyHostToDevice, s));
        }
        APRB_CUDA(cudaMemcpyAsync(doff, &bspline_offset, sizeof(float), cudaMemcpyHostToDevice, s));
        auto_parameters<float>(di, dg, dl, n, doff, par->Ip_th, grad_integer, b, s, &par->grad_th, &par->sigma_th,
                               nullptr);
    });
}

aprb_status aprb_apr_get_info(const aprb_apr *a, aprb_apr_info *info) {
    return guarded([&] {
        ARG_CHECK(a && info, "null argument");
        std::memset(info, 0, sizeof(*info));
        info->l_min = a->g.l_min;
        info->l_max = a->g.l_max;
        for (int i = 0; i < 3; ++i) info->org_dims[i] = a->org[i];
        for (int l = 0; l < 32; ++l) {
            info->y_num[l] = a->g.y_num[l];
            info->x_num[l] = a->g.x_num[l];
            info->z_num[l] = a->g.z_num[l];
        }
        info->total_number_particles = a->P;
        info->n_level_xz = (uint64_t)a->g.l_max + 2;
        info->n_xz = a->n_xz;
        info->bspline_offset = a->offset;
        if (a->tree_built) {
            info->tree_l_min = a->tg.l_min;
            info->tree_l_max = a->tg.l_max;
            info->tree_total_number_particles = a->T;
            info->tree_n_level_xz = (uint64_t)a->tg.l_max + 2;
            info->tree_n_xz = a->t_n_xz;
        }
    });
}

aprb_status aprb_apr_export(const aprb_apr *a, uint64_t *level_xz, uint64_t *xz_end, uint16_t *y_vec) {
    return guarded([&] {
        if (a) a->quiet = false;
        ARG_CHECK(a, "null apr");
        if (level_xz) std::memcpy(level_xz, a->g.level_xz, sizeof(uint64_t) * (a->g.l_max + 2));
        if (xz_end) APRB_CUDA(cudaMemcpy(xz_end, a->xz_end.p, a->n_xz * sizeof(uint64_t), cudaMemcpyDeviceToHost));
        if (y_vec && a->P) APRB_CUDA(cudaMemcpy(y_vec, a->y_vec.p, a->P * sizeof(uint16_t), cudaMemcpyDeviceToHost));
    });
}

aprb_status aprb_apr_device_arrays(const aprb_apr *a, const uint64_t **level_xz, const uint64_t **xz_end,
                                   const uint16_t **y_vec) {
    return guarded([&] {
        if (a) a->quiet = false;
        ARG_CHECK(a, "null apr");
        if (level_xz) *level_xz = nullptr;  // level offsets are host-side geometry (aprb_apr_export)
        if (xz_end) *xz_end = (const uint64_t *)a->xz_end.p;
        if (y_vec) *y_vec = (const uint16_t *)a->y_vec.p;
    });
}

aprb_status aprb_apr_from_arrays(int y_num, int x_num, int z_num, const uint64_t *level_xz, uint64_t n_level_xz,
                                 const uint64_t *xz_end, uint64_t n_xz, const uint16_t *y_vec, uint64_t n_particles,
                                 aprb_apr **out) {
    return guarded([&] {
        require_device();
        ARG_CHECK(level_xz && xz_end && out, "null argument");
        std::unique_ptr<aprb_apr> a(new aprb_apr());
        a->n_xz = apr_geometry(y_num, x_num, z_num, a->g);
        ARG_CHECK(n_level_xz == (uint64_t)a->g.l_max + 2, "level_xz length does not match the dimensions");
        ARG_CHECK(n_xz == a->n_xz, "xz_end length does not match the dimensions");
        for (uint64_t i = 0; i < n_level_xz; ++i)
            ARG_CHECK(level_xz[i] == a->g.level_xz[i], "level_xz does not match the dimensions");
        ARG_CHECK(xz_end[n_xz - 1] == n_particles, "xz_end total does not match the particle count");
        a->org[0] = y_num;
        a->org[1] = x_num;
        a->org[2] = z_num;
        a->P = n_particles;
        APRB_CUDA(cudaMemcpy(a->xz_end.as_pooled<uint64_t>(n_xz, 0), xz_end, n_xz * sizeof(uint64_t), cudaMemcpyHostToDevice));
        uint16_t *yv = a->y_vec.as_pooled<uint16_t>(n_particles ? n_particles : 1, 0);
        if (n_particles) {
            ARG_CHECK(y_vec, "null y_vec");
            APRB_CUDA(cudaMemcpy(yv, y_vec, n_particles * sizeof(uint16_t), cudaMemcpyHostToDevice));
        }
        *out = a.release();
    });
}

aprb_status aprb_reconstruct_constant_u16(const aprb_apr *a, const uint16_t *parts, uint16_t *img) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && img && (parts || a->P == 0), "null argument");
        reconstruct_host<uint16_t>(a, parts, img, false);
    });
}
aprb_status aprb_reconstruct_constant_f32(const aprb_apr *a, const float *parts, float *img) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && img && (parts || a->P == 0), "null argument");
        reconstruct_host<float>(a, parts, img, false);
    });
}
aprb_status aprb_reconstruct_level(const aprb_apr *a, uint8_t *img) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && img, "null argument");
        reconstruct_host<uint8_t>(a, nullptr, img, true);
    });
}
aprb_status aprb_reconstruct_constant_u16_device(const aprb_apr *a, const uint16_t *parts_dev, uint16_t *img_dev,
                                                 void *stream) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && img_dev && (parts_dev || a->P == 0), "null argument");
        reconstruct_device<uint16_t>(a, parts_dev, img_dev, false, (cudaStream_t)stream);
    });
}
aprb_status aprb_reconstruct_constant_f32_device(const aprb_apr *a, const float *parts_dev, float *img_dev,
                                                 void *stream) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && img_dev && (parts_dev || a->P == 0), "null argument");
        reconstruct_device<float>(a, parts_dev, img_dev, false, (cudaStream_t)stream);
    });
}
aprb_status aprb_reconstruct_level_device(const aprb_apr *a, uint8_t *img_dev, void *stream) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && img_dev, "null argument");
        reconstruct_device<uint8_t>(a, nullptr, img_dev, true, (cudaStream_t)stream);
    });
}

aprb_status aprb_sample_image_device(const aprb_apr *a, const uint16_t *img_dev, uint16_t *parts_dev, void *stream) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && img_dev && parts_dev, "null argument");
        launch_sample(a->g, (const uint64_t *)a->xz_end.p, (const uint16_t *)a->y_vec.p, img_dev, parts_dev, scratch().pyr,
                      (cudaStream_t)stream);
    });
}

aprb_status aprb_sample_image_by_block_device(const aprb_apr *a, const uint16_t *img_dev, int z_block_size,
                                              int ghost_z, uint16_t *parts_dev, void *stream) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && img_dev && parts_dev, "null argument");
        ARG_CHECK(z_block_size >= 1 && ghost_z >= 0, "z_block_size must be positive and ghost_z non-negative");
        launch_sample_by_block(a->g, (const uint64_t *)a->xz_end.p, (const uint16_t *)a->y_vec.p, img_dev, parts_dev,
                               z_block_size, ghost_z, scratch().pyr, (cudaStream_t)stream);
    });
}

aprb_status aprb_sample_image_by_block(const aprb_apr *a, const uint16_t *img, int z_block_size, int ghost_z,
                                       uint16_t *parts) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && img && parts, "null argument");
        ARG_CHECK(z_block_size >= 1 && ghost_z >= 0, "z_block_size must be positive and ghost_z non-negative");
        cudaStream_t s = cudaStreamPerThread;
        const uint64_t n = (uint64_t)a->org[0] * a->org[1] * a->org[2];
        uint16_t *di = scratch().io_in.as<uint16_t>(n);
        uint16_t *dp = scratch().parts_u16.as<uint16_t>(a->P ? a->P : 1);
        APRB_CUDA(cudaMemcpyAsync(di, img, n * sizeof(uint16_t), cudaMemcpyHostToDevice, s));
        launch_sample_by_block(a->g, (const uint64_t *)a->xz_end.p, (const uint16_t *)a->y_vec.p, di, dp,
                               z_block_size, ghost_z, scratch().pyr, s);
        if (a->P) APRB_CUDA(cudaMemcpyAsync(parts, dp, a->P * sizeof(uint16_t), cudaMemcpyDeviceToHost, s));
        APRB_CUDA(cudaStreamSynchronize(s));
    });
}

aprb_status aprb_sample_image(const aprb_apr *a, const uint16_t *img, uint16_t *parts) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && img && parts, "null argument");
        cudaStream_t s = cudaStreamPerThread;
        const Geom &g = a->g;
        const int L = g.l_max, zn = a->org[2];
        const uint64_t n = (uint64_t)a->org[0] * a->org[1] * zn;
        const uint64_t plane = (uint64_t)a->org[0] * a->org[1];
        uint16_t *dp = scratch().parts_u16.as<uint16_t>(a->P ? a->P : 1);
        const uint64_t *xz = (const uint64_t *)a->xz_end.p;
        const uint16_t *yv = (const uint16_t *)a->y_vec.p;
        if (a->kept_img.p && a->kept_host == img) {
            // the APR still holds the device copy its converter made of this
            // host buffer (keep_input): no second upload
            launch_sample(g, xz, yv, (const uint16_t *)a->kept_img.p, dp, scratch().pyr, s);
            if (a->P) APRB_CUDA(cudaMemcpyAsync(parts, dp, a->P * sizeof(uint16_t), cudaMemcpyDeviceToHost, s));
            APRB_CUDA(cudaStreamSynchronize(s));
            // the copy's upload finished before get_apr returned and this
            // stream is drained: nothing can still read it
            a->kept_img.release_idle(s);
            a->kept_host = nullptr;
            a->quiet = true;
            return;
        }
        uint16_t *di = scratch().io_in.as<uint16_t>(n);
        // about 2^26 voxels (128 MiB) per chunk, an even number of planes
        const uint64_t want = ((uint64_t(1) << 26) / std::max<uint64_t>(plane, 1)) & ~uint64_t(1);
        const int chunk = (int)std::max<uint64_t>(kSampleChunk, want);
        if (zn < 2 * chunk || L <= g.l_min || a->P == 0) {
            APRB_CUDA(cudaMemcpyAsync(di, img, n * sizeof(uint16_t), cudaMemcpyHostToDevice, s));
            launch_sample(g, xz, yv, di, dp, scratch().pyr, s);
            if (a->P) APRB_CUDA(cudaMemcpyAsync(parts, dp, a->P * sizeof(uint16_t), cudaMemcpyDeviceToHost, s));
            APRB_CUDA(cudaStreamSynchronize(s));
            return;
        }
        // Pipelined over z-chunks: chunk k's upload
        // (stream up), its level l_max gather and means (stream s) and the
        // download of its particles (stream down) overlap the neighbouring
        // chunks'.  The level l_max particles of planes [z0, z1) are one
        // contiguous range of the output; the coarser levels come last.
        Streams3 &st3 = transfer_streams();
        const int nch = (zn + chunk - 1) / chunk;
        std::vector<uint64_t> bnd(nch + 1);
        for (int k = 0; k <= nch; ++k) {
            const uint64_t row = (uint64_t)std::min(k * chunk, zn) * g.x_num[L];
            APRB_CUDA(cudaMemcpyAsync(&bnd[k], xz + g.level_xz[L] + row - 1, sizeof(uint64_t), cudaMemcpyDeviceToHost,
                                      s));
        }
        APRB_CUDA(cudaStreamSynchronize(s));
        uint64_t off[32] = {};
        uint16_t *base = sample_pyramid(g, scratch().pyr, off);
        std::vector<cudaEvent_t> ev(2 * nch + 2, nullptr);
        try {
            for (auto &e : ev) APRB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            APRB_CUDA(cudaEventRecord(ev[2 * nch + 1], s));
            APRB_CUDA(cudaStreamWaitEvent(st3.up, ev[2 * nch + 1], 0));
            for (int k = 0; k < nch; ++k) {
                const int z0 = k * chunk, z1 = std::min(zn, z0 + chunk);
                APRB_CUDA(cudaMemcpyAsync(di + (uint64_t)z0 * plane, img + (uint64_t)z0 * plane,
                                          (uint64_t)(z1 - z0) * plane * sizeof(uint16_t), cudaMemcpyHostToDevice,
                                          st3.up));
                APRB_CUDA(cudaEventRecord(ev[2 * k], st3.up));
                APRB_CUDA(cudaStreamWaitEvent(s, ev[2 * k], 0));
                launch_sample_slab(g, xz, yv, di, z0, z1, base + off[L - 1], dp, s);
                APRB_CUDA(cudaEventRecord(ev[2 * k + 1], s));
            }
            launch_sample_coarse(g, xz, yv, base, off, dp, s);
            APRB_CUDA(cudaEventRecord(ev[2 * nch], s));
            // downloads are queued after all uploads: a copy to pageable
            // memory returns only once done, which would hold back the
            // next chunk's upload
            for (int k = 0; k < nch; ++k) {
                APRB_CUDA(cudaStreamWaitEvent(st3.down, ev[2 * k + 1], 0));
                if (bnd[k + 1] > bnd[k])
                    APRB_CUDA(cudaMemcpyAsync(parts + bnd[k], dp + bnd[k], (bnd[k + 1] - bnd[k]) * sizeof(uint16_t),
                                              cudaMemcpyDeviceToHost, st3.down));
            }
            APRB_CUDA(cudaStreamWaitEvent(st3.down, ev[2 * nch], 0));
            if (bnd[0] > 0)
                APRB_CUDA(cudaMemcpyAsync(parts, dp, bnd[0] * sizeof(uint16_t), cudaMemcpyDeviceToHost, st3.down));
            APRB_CUDA(cudaStreamSynchronize(st3.down));
            APRB_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            cudaStreamSynchronize(st3.up);
            cudaStreamSynchronize(st3.down);
            cudaStreamSynchronize(s);
            for (auto &e : ev)
                if (e) cudaEventDestroy(e);
            throw;
        }
        for (auto &e : ev) cudaEventDestroy(e);
    });
}

}  // extern "C"

namespace {

void ensure_tree(aprb_apr *a, cudaStream_t s) {
    if (a->tree_built) return;
    a->t_n_xz = tree_geometry(a->org[0], a->org[1], a->org[2], a->tg);
    uint64_t *txz = a->t_xz_end.as_pooled<uint64_t>(a->t_n_xz, s);
    a->T = launch_tree_build(a->g, (const uint64_t *)a->xz_end.p, (const uint16_t *)a->y_vec.p, a->tg, txz,
                             a->t_n_xz, scratch().t_flags, scratch().scan_tmp, s);
    uint16_t *ty = a->t_y_vec.as_pooled<uint16_t>(a->T ? a->T : 1, s);
    launch_tree_fill(a->tg, scratch().t_flags, txz, ty, s);
    APRB_CUDA(cudaStreamSynchronize(s));
    build_filter_index(a->g, (const uint64_t *)a->xz_end.p, (const uint16_t *)a->y_vec.p, a->tg, txz, ty, a->fi, s);
    a->tree_built = true;
}

// stencil set of APRFilter::convolve_pencil(apr, stencil, ..., use_stencil_downsample, normalize)
// (APRFilter.hpp:139-149): one stencil per level below l_max when downsampling
template <typename T>
ConvPlan make_plan(const aprb_apr *a, const T *stencil, int ks, int ds, int normalize, int reflect,
                   std::vector<T> &host) {
    if (ks != 3 && ks != 5) {
        set_error("stencil side must be 3 or 5");
        throw Error{APRB_ERR_UNSUPPORTED};
    }
    ConvPlan plan;
    const int nlev = ds ? std::max(a->g.l_max - a->g.l_min, 1) : 1;
    host = downsampled_stencils<T>(stencil, ks, nlev, normalize != 0, plan.sides);
    plan.nstencils = (int)plan.sides.size();
    int o = 0;
    for (int sd : plan.sides) {
        plan.offsets.push_back(o);
        o += sd * sd * sd;
    }
    plan.reflect = reflect != 0;
    plan.values.assign(host.begin(), host.end());
    return plan;
}

void convolve_impl(aprb_apr *a, const float *stencil, int ks, const float *in, float *out, int reflect, int ds,
                   int normalize, cudaStream_t s) {
    ensure_tree(a, s);
    std::vector<float> host;
    ConvPlan plan = make_plan(a, stencil, ks, ds, normalize, reflect, host);
    float *dst = scratch().stencils.as<float>(host.size());
    APRB_CUDA(cudaMemcpyAsync(dst, host.data(), host.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    float *tree = scratch().tree_vals.as<float>(a->T ? a->T : 1);
    filter_apply<float>(a->g, (const uint64_t *)a->xz_end.p, (const uint16_t *)a->y_vec.p, a->tg,
                 (const uint64_t *)a->t_xz_end.p, (const uint16_t *)a->t_y_vec.p, a->fi, in, tree, &plan, dst, out, 0,
                 nullptr, scratch().fb, s);
    a->last_stale = filter_stale_count(scratch().fb, s);
}

// ---------------------------------------------------------------------------
// APRNumerics::gradient_cfd / gradient_sobel (APRNumerics.hpp:165-215) and the
// gradient magnitudes (:218-287).  The reference convolves with a 3x1x1
// central difference (cfd), a 3x3x3 Sobel stencil (3-D data) or a 3x3x1 one
// (2-D data), rescaled by 1/2^d for level delta d (APRStencil.hpp:135-152,
// 254-299).  Here the 1-D and 2-D shapes sit in the middle of a 3x3x3 cube
// with zero taps around them, which add nothing to the tap sums, so the
// cubic convolution reproduces the reference's values bit for bit.
// ---------------------------------------------------------------------------
static std::vector<float> gradient_stencils(const aprb_apr *a, int dim, int sobel, float delta, int nlev) {
    const int nd = (a->org[0] > 1) + (a->org[1] > 1) + (a->org[2] > 1);
    const float two_d = 2.0f * delta;
    const float diff[3] = {-1.0f / two_d, 0.0f, 1.0f / two_d};
    const float smooth[3] = {0.25f, 0.5f, 0.25f};
    float base[27] = {};  // [z][x][y]
    if (sobel && nd == 3) {
        const float *bank[3] = {dim == 0 ? diff : smooth, dim == 1 ? diff : smooth, dim == 2 ? diff : smooth};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) base[(k * 3 + j) * 3 + i] = bank[0][i] * bank[1][j] * bank[2][k];
    } else if (sobel && nd == 2 && dim != 2) {
        const float *bank[2] = {dim == 0 ? diff : smooth, dim == 1 ? diff : smooth};
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) base[(1 * 3 + j) * 3 + i] = bank[0][i] * bank[1][j];
    } else {
        for (int t = 0; t < 3; ++t) {
            int idx[3] = {1, 1, 1};  // z, x, y
            idx[2 - dim] = t;
            base[(idx[0] * 3 + idx[1]) * 3 + idx[2]] = diff[t];
        }
    }
    std::vector<float> out;
    for (int d = 0; d < nlev; ++d) {
        const float step = (float)std::pow(2.0, (double)d);
        for (int k = 0; k < 27; ++k) out.push_back(base[k] / step);
    }
    return out;
}

// gradient of dimension dim, device buffers
static void gradient_dim(aprb_apr *a, const float *in, float *out, int dim, int sobel, float delta, cudaStream_t s) {
    ensure_tree(a, s);
    const int nlev = std::max(a->g.l_max - a->g.l_min, 1);
    const std::vector<float> host = gradient_stencils(a, dim, sobel, delta, nlev);
    ConvPlan plan;
    plan.nstencils = nlev;
    for (int d = 0; d < nlev; ++d) {
        plan.sides.push_back(3);
        plan.offsets.push_back(27 * d);
    }
    plan.reflect = true;
    plan.values.assign(host.begin(), host.end());
    float *dst = scratch().stencils.as<float>(host.size());
    APRB_CUDA(cudaMemcpyAsync(dst, host.data(), host.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    float *tree = scratch().tree_vals.as<float>(a->T ? a->T : 1);
    filter_apply<float>(a->g, (const uint64_t *)a->xz_end.p, (const uint16_t *)a->y_vec.p, a->tg,
                        (const uint64_t *)a->t_xz_end.p, (const uint16_t *)a->t_y_vec.p, a->fi, in, tree, &plan, dst,
                        out, 0, nullptr, scratch().fb, s);
    a->last_stale = filter_stale_count(scratch().fb, s);
}

// gradient magnitude: y^2, then + x^2 and + z^2 for axes longer than 1, then
// the square root, in the reference's order; the three directions share one
// pass (tree means, neighbourhood images, particles)
static void gradient_magnitude(aprb_apr *a, const float *in, float *out, const float *deltas, int sobel,
                               cudaStream_t s) {
    ensure_tree(a, s);
    const int nlev = std::max(a->g.l_max - a->g.l_min, 1);
    std::vector<float> st[3];
    const float *stp[3];
    int active[3];
    for (int d = 0; d < 3; ++d) {
        active[d] = d == 0 || a->org[d] > 1;
        st[d] = gradient_stencils(a, d, sobel, deltas[d], nlev);
        stp[d] = st[d].data();
    }
    float *tree = scratch().tree_vals.as<float>(a->T ? a->T : 1);
    filter_gradient_magnitude(a->g, (const uint64_t *)a->xz_end.p, (const uint16_t *)a->y_vec.p, a->tg,
                              (const uint64_t *)a->t_xz_end.p, (const uint16_t *)a->t_y_vec.p, a->fi, in, tree, stp,
                              active, nlev, out, scratch().fb, s);
    a->last_stale = filter_stale_count(scratch().fb, s);
}

template <typename T>
__global__ void fill_kernel(T *p, uint64_t n, T v) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// APRNumerics::richardson_lucy (APRNumerics.hpp:551-593) with value type T:
// float, or double as the reference's FP64 instantiation.  The PSF is given
// as float and converted to T before it is flipped and down-sampled.
template <typename T>
void rl_impl(aprb_apr *a, const uint16_t *in, T *out, const float *psf, int ks, int niter, int ds, int normalize,
             int resume, cudaStream_t s) {
    ensure_tree(a, s);
    const int n0 = ks * ks * ks;
    std::vector<T> pt(n0), flipped(n0);
    for (int i = 0; i < n0; ++i) pt[i] = (T)psf[i];
    for (int i = 0; i < n0; ++i) flipped[i] = pt[n0 - 1 - i];
    std::vector<T> hp, hf;
    ConvPlan plan = make_plan<T>(a, pt.data(), ks, ds, normalize, 1, hp);
    ConvPlan plan_f = make_plan<T>(a, flipped.data(), ks, ds, normalize, 1, hf);
    T *dp = (T *)scratch().stencils.get(hp.size() * sizeof(T));
    T *df = (T *)scratch().stencils_f.get(hf.size() * sizeof(T));
    APRB_CUDA(cudaMemcpyAsync(dp, hp.data(), hp.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    APRB_CUDA(cudaMemcpyAsync(df, hf.data(), hf.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    if (!resume && a->P) {
        fill_kernel<T><<<blocks_for(a->P, 256), 256, 0, s>>>(out, a->P, T(1));
        count_launch();
        APRB_CHECK_LAUNCH();
    }
    T *tree = (T *)scratch().tree_vals.get((a->T ? a->T : 1) * sizeof(T));
    T *rb = (T *)scratch().rb.get((a->P ? a->P : 1) * sizeof(T));
    const uint64_t *xz = (const uint64_t *)a->xz_end.p;
    const uint16_t *yv = (const uint16_t *)a->y_vec.p;
    const uint64_t *txz = (const uint64_t *)a->t_xz_end.p;
    const uint16_t *tyv = (const uint16_t *)a->t_y_vec.p;
    for (int it = 0; it < niter; ++it) {
        // rb = in / conv(psf_flipped, out); out = out * conv(psf, rb)  (APRNumerics.hpp:565-570)
        filter_apply<T>(a->g, xz, yv, a->tg, txz, tyv, a->fi, out, tree, &plan_f, df, rb, 1, in, scratch().fb, s);
        filter_apply<T>(a->g, xz, yv, a->tg, txz, tyv, a->fi, rb, tree, &plan, dp, out, 2, nullptr, scratch().fb, s);
    }
}

}  // namespace

extern "C" {

aprb_status aprb_apr_init_tree(aprb_apr *a) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a, "null apr");
        ensure_tree(a, cudaStreamPerThread);
    });
}

aprb_status aprb_apr_export_tree(aprb_apr *a, uint64_t *level_xz, uint64_t *xz_end, uint16_t *y_vec) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a, "null apr");
        ensure_tree(a, cudaStreamPerThread);
        if (level_xz) std::memcpy(level_xz, a->tg.level_xz, sizeof(uint64_t) * (a->tg.l_max + 2));
        if (xz_end) APRB_CUDA(cudaMemcpy(xz_end, a->t_xz_end.p, a->t_n_xz * sizeof(uint64_t), cudaMemcpyDeviceToHost));
        if (y_vec && a->T) APRB_CUDA(cudaMemcpy(y_vec, a->t_y_vec.p, a->T * sizeof(uint16_t), cudaMemcpyDeviceToHost));
    });
}

aprb_status aprb_fill_tree_mean_device(aprb_apr *a, const float *parts_dev, float *tree_dev, void *stream) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && parts_dev && tree_dev, "null argument");
        cudaStream_t s = (cudaStream_t)stream;
        ensure_tree(a, s);
        filter_apply<float>(a->g, (const uint64_t *)a->xz_end.p, (const uint16_t *)a->y_vec.p, a->tg,
                     (const uint64_t *)a->t_xz_end.p, (const uint16_t *)a->t_y_vec.p, a->fi, parts_dev, tree_dev, nullptr,
                     nullptr, nullptr, 0, nullptr, scratch().fb, s);
    });
}

aprb_status aprb_fill_tree_mean(aprb_apr *a, const float *parts, float *tree) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && parts && tree, "null argument");
        cudaStream_t s = cudaStreamPerThread;
        ensure_tree(a, s);
        float *dp = scratch().parts_f.as<float>(a->P ? a->P : 1);
        float *dt = scratch().out_f.as<float>(a->T ? a->T : 1);
        APRB_CUDA(cudaMemcpyAsync(dp, parts, a->P * sizeof(float), cudaMemcpyHostToDevice, s));
        filter_apply<float>(a->g, (const uint64_t *)a->xz_end.p, (const uint16_t *)a->y_vec.p, a->tg,
                     (const uint64_t *)a->t_xz_end.p, (const uint16_t *)a->t_y_vec.p, a->fi, dp, dt, nullptr, nullptr,
                     nullptr, 0, nullptr, scratch().fb, s);
        APRB_CUDA(cudaMemcpyAsync(tree, dt, a->T * sizeof(float), cudaMemcpyDeviceToHost, s));
        APRB_CUDA(cudaStreamSynchronize(s));
    });
}

aprb_status aprb_convolve_device(aprb_apr *a, const float *stencil, int ksize, const float *in_dev, float *out_dev,
                                 int reflect, int use_stencil_downsample, int normalize, void *stream) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && stencil && in_dev && out_dev, "null argument");
        convolve_impl(a, stencil, ksize, in_dev, out_dev, reflect, use_stencil_downsample, normalize,
                      (cudaStream_t)stream);
    });
}

aprb_status aprb_gradient(aprb_apr *a, const float *in, float *out, int dimension, float delta, int sobel) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && out && (in || a->P == 0), "null argument");
        ARG_CHECK(dimension >= 0 && dimension <= 2, "dimension must be 0 (y), 1 (x) or 2 (z)");
        cudaStream_t s = cudaStreamPerThread;
        float *din = scratch().parts_f.as<float>(a->P ? a->P : 1);
        float *dout = scratch().out_f.as<float>(a->P ? a->P : 1);
        if (a->P) APRB_CUDA(cudaMemcpyAsync(din, in, a->P * sizeof(float), cudaMemcpyHostToDevice, s));
        gradient_dim(a, din, dout, dimension, sobel, delta, s);
        if (a->P) APRB_CUDA(cudaMemcpyAsync(out, dout, a->P * sizeof(float), cudaMemcpyDeviceToHost, s));
        APRB_CUDA(cudaStreamSynchronize(s));
    });
}

aprb_status aprb_gradient_device(aprb_apr *a, const float *in_dev, float *out_dev, int dimension, float delta,
                                 int sobel, void *stream) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && out_dev && (in_dev || a->P == 0), "null argument");
        ARG_CHECK(dimension >= 0 && dimension <= 2, "dimension must be 0 (y), 1 (x) or 2 (z)");
        gradient_dim(a, in_dev, out_dev, dimension, sobel, delta, (cudaStream_t)stream);
    });
}

aprb_status aprb_gradient_magnitude(aprb_apr *a, const float *in, float *out, const float *deltas, int sobel) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && out && deltas && (in || a->P == 0), "null argument");
        cudaStream_t s = cudaStreamPerThread;
        float *din = scratch().parts_f.as<float>(a->P ? a->P : 1);
        float *dout = scratch().out_f.as<float>(a->P ? a->P : 1);
        if (a->P) APRB_CUDA(cudaMemcpyAsync(din, in, a->P * sizeof(float), cudaMemcpyHostToDevice, s));
        gradient_magnitude(a, din, dout, deltas, sobel, s);
        if (a->P) APRB_CUDA(cudaMemcpyAsync(out, dout, a->P * sizeof(float), cudaMemcpyDeviceToHost, s));
        APRB_CUDA(cudaStreamSynchronize(s));
    });
}

aprb_status aprb_gradient_magnitude_device(aprb_apr *a, const float *in_dev, float *out_dev, const float *deltas,
                                           int sobel, void *stream) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && out_dev && deltas && (in_dev || a->P == 0), "null argument");
        gradient_magnitude(a, in_dev, out_dev, deltas, sobel, (cudaStream_t)stream);
    });
}

aprb_status aprb_convolve(aprb_apr *a, const float *stencil, int ksize, const float *in, float *out, int reflect,
                          int use_stencil_downsample, int normalize) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && stencil && in && out, "null argument");
        cudaStream_t s = cudaStreamPerThread;
        float *di = scratch().parts_f.as<float>(a->P ? a->P : 1);
        float *dout = scratch().out_f.as<float>(a->P ? a->P : 1);
        APRB_CUDA(cudaMemcpyAsync(di, in, a->P * sizeof(float), cudaMemcpyHostToDevice, s));
        convolve_impl(a, stencil, ksize, di, dout, reflect, use_stencil_downsample, normalize, s);
        APRB_CUDA(cudaMemcpyAsync(out, dout, a->P * sizeof(float), cudaMemcpyDeviceToHost, s));
        APRB_CUDA(cudaStreamSynchronize(s));
    });
}

aprb_status aprb_richardson_lucy_device(aprb_apr *a, const uint16_t *in_dev, float *out_dev, const float *psf,
                                        int ksize, int niter, int use_stencil_downsample, int normalize, int resume,
                                        void *stream) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && in_dev && out_dev && psf && niter >= 0, "invalid argument");
        rl_impl<float>(a, in_dev, out_dev, psf, ksize, niter, use_stencil_downsample, normalize, resume,
                (cudaStream_t)stream);
    });
}

aprb_status aprb_richardson_lucy(aprb_apr *a, const uint16_t *in, float *out, const float *psf, int ksize, int niter,
                                 int use_stencil_downsample, int normalize, int resume) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && in && out && psf && niter >= 0, "invalid argument");
        cudaStream_t s = cudaStreamPerThread;
        uint16_t *di = scratch().parts_u16.as<uint16_t>(a->P ? a->P : 1);
        float *dout = scratch().out_f.as<float>(a->P ? a->P : 1);
        APRB_CUDA(cudaMemcpyAsync(di, in, a->P * sizeof(uint16_t), cudaMemcpyHostToDevice, s));
        if (resume) APRB_CUDA(cudaMemcpyAsync(dout, out, a->P * sizeof(float), cudaMemcpyHostToDevice, s));
        rl_impl<float>(a, di, dout, psf, ksize, niter, use_stencil_downsample, normalize, resume, s);
        APRB_CUDA(cudaMemcpyAsync(out, dout, a->P * sizeof(float), cudaMemcpyDeviceToHost, s));
        APRB_CUDA(cudaStreamSynchronize(s));
    });
}

aprb_status aprb_richardson_lucy_fp64_device(aprb_apr *a, const uint16_t *in_dev, double *out_dev, const float *psf,
                                             int ksize, int niter, int use_stencil_downsample, int normalize,
                                             int resume, void *stream) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && in_dev && out_dev && psf && niter >= 0, "invalid argument");
        rl_impl<double>(a, in_dev, out_dev, psf, ksize, niter, use_stencil_downsample, normalize, resume,
                        (cudaStream_t)stream);
    });
}

aprb_status aprb_richardson_lucy_fp64(aprb_apr *a, const uint16_t *in, double *out, const float *psf, int ksize,
                                      int niter, int use_stencil_downsample, int normalize, int resume) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && in && out && psf && niter >= 0, "invalid argument");
        cudaStream_t s = cudaStreamPerThread;
        uint16_t *di = scratch().parts_u16.as<uint16_t>(a->P ? a->P : 1);
        double *dout = (double *)scratch().out_f.get((a->P ? a->P : 1) * sizeof(double));
        APRB_CUDA(cudaMemcpyAsync(di, in, a->P * sizeof(uint16_t), cudaMemcpyHostToDevice, s));
        if (resume) APRB_CUDA(cudaMemcpyAsync(dout, out, a->P * sizeof(double), cudaMemcpyHostToDevice, s));
        rl_impl<double>(a, di, dout, psf, ksize, niter, use_stencil_downsample, normalize, resume, s);
        APRB_CUDA(cudaMemcpyAsync(out, dout, a->P * sizeof(double), cudaMemcpyDeviceToHost, s));
        APRB_CUDA(cudaStreamSynchronize(s));
    });
}

}  // extern "C"

namespace {

CnnGeom cnn_geom(aprb_apr *a, cudaStream_t s) {
    ensure_tree(a, s);
    if (!a->cnn_ready) {
        ARG_CHECK(a->P < 0xffffffffull, "too many particles for the learned proposal");
        uint32_t *rows = a->cnn_rows.as_pooled<uint32_t>(a->P ? a->P : 1, s);
        cnn_build_rows(a->g, (const uint64_t *)a->xz_end.p, rows, s);
        a->cnn_ready = true;
    }
    CnnGeom cg;
    cg.g = &a->g;
    cg.tg = &a->tg;
    cg.xz_end = (const uint64_t *)a->xz_end.p;
    cg.y_vec = (const uint16_t *)a->y_vec.p;
    cg.t_xz_end = (const uint64_t *)a->t_xz_end.p;
    cg.t_y_vec = (const uint16_t *)a->t_y_vec.p;
    cg.fi = &a->fi;
    cg.prow = (const uint32_t *)a->cnn_rows.p;
    for (int l = 0; l < 34; ++l) cg.level_begin[l] = 0;
    uint64_t acc = 0;
    for (int l = a->g.l_min; l <= a->g.l_max; ++l) {
        cg.level_begin[l] = acc;
        acc += a->fi.level_count[l];
    }
    cg.level_begin[a->g.l_max + 1] = acc;
    cg.T = a->T;
    return cg;
}

}  // namespace

extern "C" {

aprb_status aprb_cnn_layer_forward_device(aprb_apr *a, const float *in, const float *W, const float *bias, int relu,
                                          float *out, void *stream) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && in && W && bias && out, "null argument");
        cudaStream_t s = (cudaStream_t)stream;
        const CnnGeom cg = cnn_geom(a, s);
        cnn_layer_forward(cg, in, W, bias, relu, out, scratch().cnn, s);
    });
}

aprb_status aprb_cnn_layer_backward_device(aprb_apr *a, const float *in, const float *W, const float *out,
                                           const float *g_out, int relu, float *g_in, float *dW, float *db,
                                           void *stream) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && in && W && out && g_out && g_in && dW && db, "null argument");
        cudaStream_t s = (cudaStream_t)stream;
        const CnnGeom cg = cnn_geom(a, s);
        cnn_layer_backward(cg, in, W, out, g_out, relu, g_in, dW, db, scratch().cnn, s);
    });
}

aprb_status aprb_cnn_features_device(const aprb_apr *a, const float *u, const float *ratio, const uint16_t *raw,
                                     float *features, void *stream) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && u && ratio && raw && features, "null argument");
        cnn_features(u, ratio, raw, features, a->P, (cudaStream_t)stream);
    });
}

aprb_status aprb_cnn_loss_device(const aprb_apr *a, const float *pred, const float *u0, const float *u1, float *g_pred,
                                 double *loss_dev, void *stream) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && pred && u0 && u1 && g_pred && loss_dev, "null argument");
        cnn_loss(pred, u0, u1, g_pred, a->P, loss_dev, (cudaStream_t)stream);
    });
}

aprb_status aprb_cnn_apply_device(const aprb_apr *a, const float *pred, float *u, void *stream) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && pred && u, "null argument");
        cnn_apply(pred, u, a->P, (cudaStream_t)stream);
    });
}

aprb_status aprb_cnn_adam_device(float *params, const float *grads, float *m, float *v, const float *mask, uint64_t n,
                                 float lr, float beta1, float beta2, float eps, int step, void *stream) {
    return guarded([&] {
        require_device();
        ARG_CHECK(params && grads && m && v && step >= 1, "invalid argument");
        cnn_adam(params, grads, m, v, mask, n, lr, beta1, beta2, eps, step, (cudaStream_t)stream);
    });
}

aprb_status aprb_rl_ratio_device(aprb_apr *a, const uint16_t *in_dev, const float *u_dev, float *ratio_dev,
                                 const float *psf, int ksize, int use_stencil_downsample, int normalize,
                                 void *stream) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && in_dev && u_dev && ratio_dev && psf, "null argument");
        cudaStream_t s = (cudaStream_t)stream;
        ensure_tree(a, s);
        const int n0 = ksize * ksize * ksize;
        std::vector<float> flipped(n0);
        for (int i = 0; i < n0; ++i) flipped[i] = psf[n0 - 1 - i];
        std::vector<float> hf;
        ConvPlan plan_f = make_plan<float>(a, flipped.data(), ksize, use_stencil_downsample, normalize, 1, hf);
        float *df = (float *)scratch().stencils_f.get(hf.size() * sizeof(float));
        APRB_CUDA(cudaMemcpyAsync(df, hf.data(), hf.size() * sizeof(float), cudaMemcpyHostToDevice, s));
        float *tree = (float *)scratch().tree_vals.get((a->T ? a->T : 1) * sizeof(float));
        filter_apply<float>(a->g, (const uint64_t *)a->xz_end.p, (const uint16_t *)a->y_vec.p, a->tg,
                            (const uint64_t *)a->t_xz_end.p, (const uint16_t *)a->t_y_vec.p, a->fi, u_dev, tree,
                            &plan_f, df, ratio_dev, 1, in_dev, scratch().fb, s);
    });
}

aprb_status aprb_rl_objective_device(aprb_apr *a, const uint16_t *in_dev, const float *u_dev, const float *psf,
                                     int ksize, int use_stencil_downsample, int normalize, double *objective,
                                     void *stream) {
    return guarded([&] {
        if (a) a->quiet = false;
        require_device();
        ARG_CHECK(a && in_dev && u_dev && psf && objective, "null argument");
        cudaStream_t s = (cudaStream_t)stream;
        ensure_tree(a, s);
        const int n0 = ksize * ksize * ksize;
        std::vector<float> flipped(n0);
        for (int i = 0; i < n0; ++i) flipped[i] = psf[n0 - 1 - i];
        std::vector<float> hf;
        ConvPlan plan_f = make_plan<float>(a, flipped.data(), ksize, use_stencil_downsample, normalize, 1, hf);
        float *df = (float *)scratch().stencils_f.get(hf.size() * sizeof(float));
        APRB_CUDA(cudaMemcpyAsync(df, hf.data(), hf.size() * sizeof(float), cudaMemcpyHostToDevice, s));
        float *tree = (float *)scratch().tree_vals.get((a->T ? a->T : 1) * sizeof(float));
        float *k = (float *)scratch().rb.get((a->P ? a->P : 1) * sizeof(float));
        filter_apply<float>(a->g, (const uint64_t *)a->xz_end.p, (const uint16_t *)a->y_vec.p, a->tg,
                            (const uint64_t *)a->t_xz_end.p, (const uint16_t *)a->t_y_vec.p, a->fi, u_dev, tree,
                            &plan_f, df, k, 0, nullptr, scratch().fb, s);
        double *d = (double *)scratch().obj.get(sizeof(double));
        rl_objective_sum(k, in_dev, a->P, d, s);
        APRB_CUDA(cudaMemcpyAsync(objective, d, sizeof(double), cudaMemcpyDeviceToHost, s));
        APRB_CUDA(cudaStreamSynchronize(s));
    });
}

aprb_status aprb_synth_blobs_u16(uint16_t *img_dev, int y_num, int x_num, int z_num, int n_blobs, float sigma_lo,
                                 float sigma_hi, float amp_lo, float amp_hi, float background, uint64_t seed,
                                 void *stream) {
    return guarded([&] {
        require_device();
        ARG_CHECK(img_dev && y_num > 0 && x_num > 0 && z_num > 0 && n_blobs >= 0, "invalid argument");
        static thread_local DevBuf buf;
        launch_synth_blobs(img_dev, y_num, x_num, z_num, n_blobs, sigma_lo, sigma_hi, amp_lo, amp_hi, background,
                           seed, buf, (cudaStream_t)stream);
    });
}

aprb_status aprb_synth_blobs_f32(float *img_dev, int y_num, int x_num, int z_num, int n_blobs, float sigma_lo,
                                 float sigma_hi, float amp_lo, float amp_hi, float background, uint64_t seed,
                                 void *stream) {
    return guarded([&] {
        require_device();
        ARG_CHECK(img_dev && y_num > 0 && x_num > 0 && z_num > 0 && n_blobs >= 0, "invalid argument");
        static thread_local DevBuf buf;
        launch_synth_blobs(img_dev, y_num, x_num, z_num, n_blobs, sigma_lo, sigma_hi, amp_lo, amp_hi, background, seed,
                           buf, (cudaStream_t)stream);
    });
}

}  // extern "C"
