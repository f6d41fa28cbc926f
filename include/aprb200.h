/*
 * aprb200 -- B200-native (sm_100a) APR construction and filtering.
 *
 * C ABI of libaprb200.so.  Plain pointers and sizes only; every entry point
 * returns an aprb_status and never throws.  Each declaration names the LibAPR
 * interface it replaces (file:line in the LibAPR source tree).
 *
 * Conventions
 *  - Dense images are y-fastest, then x, then z (LibAPR PixelData order:
 *    index = z*x_num*y_num + x*y_num + y), dimensions passed as (y, x, z).
 *  - Functions without the _device suffix take HOST buffers, copy them to the
 *    GPU, run, copy results back and return when the results are on the host
 *    (the reference's calls are blocking too).  The _device variants take
 *    device pointers and a cudaStream_t (passed as void*), enqueue work on that
 *    stream and return without waiting, except where noted (a structure whose
 *    size is data-dependent reads its particle count back once).
 *  - The particle structure is the reference's linear access structure
 *    (LinearAccess.hpp:33-35): level_xz (uint64, l_max+2 entries), xz_end
 *    (uint64, inclusive particle counts per (level, z, x) row, entry 0 is a
 *    zero guard), y_vec (uint16 per particle); particle order is level
 *    ascending, then z, x, y.
 *  - One GPU, the calling thread's current CUDA device.  Handles are not
 *    thread-safe: one converter / APR handle per host thread, as one
 *    APRConverter object is not re-entrant in the reference.
 */
#ifndef APRB200_H
#define APRB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    APRB_OK = 0,
    APRB_ERR_INVALID_ARGUMENT = 1,   /* null pointer, bad enum, size mismatch            */
    APRB_ERR_DIMENSIONS = 2,         /* input dimension check failed (APRConverter.hpp:86-91)  */
    APRB_ERR_INTEGER_OVERFLOW = 3,   /* uint16 IIR under/overflow (ComputeGradient.hpp:409-412) */
    APRB_ERR_UNSUPPORTED = 4,        /* e.g. stencil side not 3 or 5 (APRNumericsGPU.cu:201-203) */
    APRB_ERR_OUT_OF_MEMORY = 5,
    APRB_ERR_CUDA = 6,               /* a CUDA runtime call failed                        */
    APRB_ERR_NO_DEVICE = 7,          /* no usable sm_100 device                           */
    APRB_ERR_INCOMPLETE_NEIGHBOURHOOD = 8 /* filter read a cell no particle covers (invalid APR) */
} aprb_status;

/* Mirror of the APRParameters fields the path reads (APRParameters.hpp:14-41). */
typedef struct {
    float dx, dy, dz;
    float psfx, psfy, psfz;
    float Ip_th, lambda, rel_error, sigma_th, sigma_th_max, grad_th;
    int reflect_bc_lis;              /* default 1 */
    int neighborhood_optimization;   /* default 1 */
    int constant_intensity_scale;    /* default 0 */
    int check_input;                 /* default 0 (APRConverter.hpp:86) */
    int swap_dimensions;             /* default 0 */
    int auto_parameters;             /* default 0 (APRParameters.hpp:32): grad_th and sigma_th
                                        by autoParametersLiEntropy before applyParameters */
} aprb_params;

/* ImageType of APRConverter<ImageType> */
enum { APRB_IMAGE_FLOAT = 0, APRB_IMAGE_U16 = 1 };

/* Intermediates kept by a converter for stage-level checks. */
enum {
    APRB_STAGE_SMOOTHED = 0,        /* full-res B-spline coefficients (IT values as float)    */
    APRB_STAGE_GRADIENT = 1,        /* ds gradient magnitude after get_gradient               */
    APRB_STAGE_DS_IMAGE = 2,        /* ds inverse-bspline image (local_scale_temp2)           */
    APRB_STAGE_LOCAL_SCALE = 3,     /* ds local intensity scale                               */
    APRB_STAGE_GRADIENT_APPLIED = 4,/* ds gradient after applyParameters                      */
    APRB_STAGE_SCALE_APPLIED = 5,   /* ds scale after applyParameters                         */
    APRB_STAGE_LEVELS = 6           /* ds particle-cell levels (compute_level_for_array)      */
};

typedef struct aprb_converter aprb_converter;
typedef struct aprb_apr aprb_apr;

typedef struct {
    int l_min, l_max;
    int org_dims[3];                 /* y, x, z */
    int y_num[32], x_num[32], z_num[32];
    uint64_t total_number_particles;
    uint64_t n_level_xz;             /* l_max + 2 */
    uint64_t n_xz;                   /* entries of xz_end */
    float bspline_offset;
    /* tree (valid after aprb_apr_init_tree) */
    int tree_l_min, tree_l_max;
    uint64_t tree_total_number_particles, tree_n_level_xz, tree_n_xz;
} aprb_apr_info;

const char *aprb_status_string(aprb_status s);
/* Text of the last error on this thread ("" when none). */
const char *aprb_last_error(void);

/* APRParameters defaults (APRParameters.hpp:14-41). */
void aprb_default_params(aprb_params *p);

/* --- construction: APRConverter<ImageType> (APRConverter.hpp:35-134) ---------- */
aprb_status aprb_converter_create(int image_type, aprb_converter **out);
aprb_status aprb_converter_destroy(aprb_converter *c);
/* keep_intermediates != 0 keeps the APRB_STAGE_* buffers after get_apr */
aprb_status aprb_converter_keep_intermediates(aprb_converter *c, int keep);

/* keep != 0: aprb_get_apr (host buffer) hands its device copy of the input image to the
 * APR it returns, and the first aprb_sample_image of that APR from the same host buffer
 * samples that copy instead of uploading the image again (the reference's call pair
 * get_apr(apr, img); sample_image(apr, img) moves the volume to the GPU once).  The caller
 * must not change the image in between; the copy is released by that sample_image or
 * with the APR.  No counterpart in the reference (a host-transfer option). */
aprb_status aprb_converter_keep_input(aprb_converter *c, int keep);

/* APRConverter<IT>::get_apr(APR&, PixelData<uint16_t>&) (APRConverter.hpp:591-600 -> get_apr_cpu :535-582) */
aprb_status aprb_get_apr(aprb_converter *c, const aprb_params *p, const uint16_t *img, int y_num, int x_num,
                         int z_num, aprb_apr **out);
/* same, image already on the device; enqueued on stream, returns after the particle count is known */
aprb_status aprb_get_apr_device(aprb_converter *c, const aprb_params *p, const uint16_t *img_dev, int y_num,
                                int x_num, int z_num, void *stream, aprb_apr **out);
/* Blocked construction, APRConverterBatch<IT> (APRConverterBatch.hpp:114-175): the pixel
 * pipeline runs per z-tile of z_block_size planes (the last tile takes the remainder) with
 * up to ghost_z planes of overlap on each side (get_apr_method_patch :190-271), every tile
 * fills the global particle-cell tree (fill_global_particle_cell_tree :282-314), then one
 * pulling scheme and one linear structure are built.  The reference reads the tiles from a
 * TIFF file (get_apr(APR&) :48-64); here the caller passes the volume.  Reference defaults:
 * z_block_size 128, ghost_z 32.  Where the reference's integer ghost cropping maps the last
 * tile one plane past a coarse level, the reference writes outside that level's array; here
 * those planes are skipped. */
aprb_status aprb_get_apr_by_block(aprb_converter *c, const aprb_params *p, const uint16_t *img, int y_num,
                                  int x_num, int z_num, int z_block_size, int ghost_z, aprb_apr **out);
aprb_status aprb_get_apr_by_block_device(aprb_converter *c, const aprb_params *p, const uint16_t *img_dev, int y_num,
                                         int x_num, int z_num, int z_block_size, int ghost_z, void *stream,
                                         aprb_apr **out);
/* many volumes of uneven sizes through the blocked converter, in order, on one stream
 * (the reference converts one file per call); outs[i] receives volume i's APR, and on an
 * error no APR is returned */
typedef struct {
    const uint16_t *img_dev;
    int y_num, x_num, z_num;
} aprb_volume;
aprb_status aprb_get_apr_batch_device(aprb_converter *c, const aprb_params *p, int n_volumes,
                                      const aprb_volume *volumes, int z_block_size, int ghost_z, void *stream,
                                      aprb_apr **outs);
/* --- the blocked converter split by z-tiles over several GPUs -------------------
 * APRConverterBatch (APRConverterBatch.hpp:114-175) fills one global particle-cell tree
 * from its z-tiles (fill_global_particle_cell_tree :282-314, PullingScheme::fill_patch
 * PullingScheme.hpp:175-247) and solves it once.  A tile only sets cells to SEED, so the
 * tree of all tiles is the element-wise maximum of the trees of any partition of the tiles:
 * each GPU fills a zeroed pyramid from its own tiles, the pyramids are combined by a MAX
 * all-reduce (one uint8 buffer), and the pulling scheme and linear structure run on the
 * result.  The layout is the converter's own: pct levels l_min .. l_max - 1, each padded
 * to 16 bytes. */
/* bytes of the pyramid buffer of a y x x x z volume */
aprb_status aprb_pyramid_bytes(int y_num, int x_num, int z_num, uint64_t *bytes);
/* get_apr_method_patch (:190-271) for tiles [first_tile, first_tile + n_tiles) of the
 * volume's tiling (z_block_size, ghost_z), filling pyramid_dev (zeroed by the caller before
 * the first fill); slab_dev holds planes [slab_z0, slab_z0 + slab_z_num) of the volume and
 * must contain the tiles' planes and ghosts.  Blocks until the overflow check is read. */
aprb_status aprb_pyramid_fill_tiles_device(aprb_converter *c, const aprb_params *p, uint8_t *pyramid_dev, int y_num,
                                           int x_num, int z_num, int z_block_size, int ghost_z, int first_tile,
                                           int n_tiles, const uint16_t *slab_dev, int slab_z0, int slab_z_num,
                                           void *stream);
/* pulling_scheme_main + generateDatastructures (APRConverter.hpp:339-363) of a filled
 * pyramid (consumed: the pulling scheme works in place) */
aprb_status aprb_get_apr_from_pyramid_device(aprb_converter *c, const aprb_params *p, uint8_t *pyramid_dev, int y_num,
                                             int x_num, int z_num, void *stream, aprb_apr **out);

/* copy one APRB_STAGE_* intermediate of the last get_apr to the host (n = element count) */
aprb_status aprb_converter_intermediate(const aprb_converter *c, int stage, float *dst, size_t n);
/* Level-decision margins of the last get_apr (needs aprb_converter_keep_intermediates).
 * computeLevels (LocalParticleCellSet.hpp:129-171) gives a down-sampled cell the level
 * floor(log2(v)), v = (grad / scale) * 2^l_max * min(dx, dy, dz) / E after applyParameters
 * (APRConverter.hpp:250-297); a computation of v that differs by a relative rel_tol can
 * decide another level only where v lies within rel_tol of a power of two 2^k (k >= 1).
 * near_boundary receives the number of such cells, active the number with v >= 1. */
aprb_status aprb_converter_level_margins(aprb_converter *c, double rel_tol, uint64_t *near_boundary,
                                         uint64_t *active);

/* --- automatic parameters (AutoParameters.hpp) ----------------------------------
 * With aprb_params.auto_parameters set, get_apr (APRConverter.hpp:556-561) and each
 * tile of the blocked converter (APRConverterBatch.hpp:243-247) replace grad_th and
 * sigma_th by Li's minimum cross entropy thresholds of the gradient and the local
 * intensity scale before applyParameters; aprb_apr_get_parameters returns them.
 * Sums are FP64 in a fixed order (the reference sums in FP32 in an order set by its
 * OpenMP thread count); with no foreground pixel both thresholds are 0 (the
 * reference divides by zero there); at most 1000 Li steps. */

/* threshold_li<T> (AutoParameters.hpp:50-100) on n host values of T held as float:
 * integer_values != 0 for T = uint16_t (tolerance 0.5), else T = float. */
aprb_status aprb_threshold_li(const float *values, uint64_t n, int integer_values, float *threshold);
/* autoParametersLiEntropy(par, image, localIntensityScale, grad, bspline_offset)
 * (AutoParameters.hpp:103-153) on n host cells: image = the down-sampled image
 * (local_scale_temp2), lis = local intensity scale, grad = gradient holding ImageType
 * values (grad_integer != 0 for uint16_t).  Sets par->grad_th and par->sigma_th. */
aprb_status aprb_auto_parameters(aprb_params *par, const float *image, const float *lis, const float *grad,
                                 uint64_t n, int grad_integer, float bspline_offset);

/* --- the APR object ------------------------------------------------------------ */
aprb_status aprb_apr_free(aprb_apr *a);
aprb_status aprb_apr_get_info(const aprb_apr *a, aprb_apr_info *info);
/* APR::get_apr_parameters (APR.hpp:99-101): the parameters the APR was built with,
 * grad_th / sigma_th as chosen by the automatic parameters when those were on */
aprb_status aprb_apr_get_parameters(const aprb_apr *a, aprb_params *par);
/* LinearAccess arrays to host (any pointer may be NULL) */
aprb_status aprb_apr_export(const aprb_apr *a, uint64_t *level_xz, uint64_t *xz_end, uint16_t *y_vec);
/* device pointers of the LinearAccess arrays (owned by the APR) */
aprb_status aprb_apr_device_arrays(const aprb_apr *a, const uint64_t **level_xz, const uint64_t **xz_end,
                                   const uint16_t **y_vec);
/* build an APR from host LinearAccess arrays (e.g. read from a .apr file) */
aprb_status aprb_apr_from_arrays(int y_num, int x_num, int z_num, const uint64_t *level_xz, uint64_t n_level_xz,
                                 const uint64_t *xz_end, uint64_t n_xz, const uint16_t *y_vec, uint64_t n_particles,
                                 aprb_apr **out);

/* --- particle sampling: ParticleData::sample_image (ParticleData.hpp:123-127) --- */
aprb_status aprb_sample_image(const aprb_apr *a, const uint16_t *img, uint16_t *parts);
aprb_status aprb_sample_image_device(const aprb_apr *a, const uint16_t *img_dev, uint16_t *parts_dev, void *stream);
/* blocked sampling, sample_parts_from_img_blocked (ParticleData.hpp:140-142, 288-372): every
 * z-tile builds its own mean pyramid and writes the particles of its rows (reference
 * defaults z_block_size 256, ghost_z 32; tiles from memory instead of a TIFF file) */
aprb_status aprb_sample_image_by_block(const aprb_apr *a, const uint16_t *img, int z_block_size, int ghost_z,
                                       uint16_t *parts);
aprb_status aprb_sample_image_by_block_device(const aprb_apr *a, const uint16_t *img_dev, int z_block_size,
                                              int ghost_z, uint16_t *parts_dev, void *stream);

/* Particle sampling that allocates no device memory.  No counterpart in the
 * reference.  For callers that cannot allocate GPU memory while they run:
 * real-time acquisition loops and plugin hosts that own a fixed device-memory
 * budget and forbid cudaMalloc and cudaFree after start-up.  It takes the
 * APR's device arrays (xz_end, y_vec, e.g. from aprb_apr_device_arrays) and
 * the image dimensions (y, x, z), and keeps its down-sampling pyramid in one
 * 64 MiB file-scope device buffer of the library.  The buffer is reserved on
 * a device when the library's module is first used there (at library load
 * only with eager module loading, CUDA_MODULE_LOADING=EAGER) and stays until
 * the process exits.  Volumes whose pyramid below l_max needs more than
 * 32 Mi uint16 values (about 2.2e8 voxels) are rejected with
 * APRB_ERR_INVALID_ARGUMENT.  The first call on a device looks the buffer up
 * for that device (which may load the module); make that first call before
 * any stream capture.  Later calls outside stream capture look it up again,
 * so a device reset (which reloads the module) is picked up.  All calls share
 * the buffer: calls that overlap on the GPU (other streams, other host
 * threads) race and must be serialised by the caller. */
aprb_status aprb_sample_image_noalloc(const uint64_t *xz_end_dev, const uint16_t *y_vec_dev, int y_num, int x_num,
                                      int z_num, const uint16_t *img_dev, uint16_t *parts_dev, void *stream);

/* --- reconstruction: APRReconstruction::reconstruct_constant
 * (APRReconstruction.hpp:80-123) and reconstruct_level (:132-170) ----------------
 * The full-resolution image (y fastest, org dims) in which every pixel takes
 * the value (or the level) of the particle whose cell covers it.  parts holds
 * P values in linear order; img holds y*x*z values. */
aprb_status aprb_reconstruct_constant_u16(const aprb_apr *a, const uint16_t *parts, uint16_t *img);
aprb_status aprb_reconstruct_constant_f32(const aprb_apr *a, const float *parts, float *img);
aprb_status aprb_reconstruct_level(const aprb_apr *a, uint8_t *img);
aprb_status aprb_reconstruct_constant_u16_device(const aprb_apr *a, const uint16_t *parts_dev, uint16_t *img_dev,
                                                 void *stream);
aprb_status aprb_reconstruct_constant_f32_device(const aprb_apr *a, const float *parts_dev, float *img_dev,
                                                 void *stream);
aprb_status aprb_reconstruct_level_device(const aprb_apr *a, uint8_t *img_dev, void *stream);

/* --- APR tree: APR::initialize_tree_dense (APR.hpp:633-689) ---------------------- */
aprb_status aprb_apr_init_tree(aprb_apr *a);
aprb_status aprb_apr_export_tree(aprb_apr *a, uint64_t *level_xz, uint64_t *xz_end, uint16_t *y_vec);
/* APRTreeNumerics::fill_tree_mean (APRTreeNumerics.hpp:63-203) */
aprb_status aprb_fill_tree_mean(aprb_apr *a, const float *parts, float *tree);
aprb_status aprb_fill_tree_mean_device(aprb_apr *a, const float *parts_dev, float *tree_dev, void *stream);

/* --- APR isotropic convolution --------------------------------------------------
 * APRFilter::convolve_pencil(apr, stencil, in, out, reflect, use_stencil_downsample, normalize)
 * (APRFilter.hpp:139-149, :1094-1216), and the GPU isotropic_convolve_333/555
 * (APRIsoConvGPU333.hpp:37-51, APRIsoConvGPU555.hpp:38-52) which it replaces.
 * stencil: ksize^3 floats in PixelData order; ksize 3 or 5.  Every level,
 * l_min included, is filtered (the CPU semantics). */
aprb_status aprb_convolve(aprb_apr *a, const float *stencil, int ksize, const float *in, float *out, int reflect,
                          int use_stencil_downsample, int normalize);
aprb_status aprb_convolve_device(aprb_apr *a, const float *stencil, int ksize, const float *in_dev, float *out_dev,
                                 int reflect, int use_stencil_downsample, int normalize, void *stream);

/* --- APR gradients: APRNumerics::gradient_cfd / gradient_sobel of one
 * dimension (0 y, 1 x, 2 z; APRNumerics.hpp:165-215) and
 * gradient_magnitude_cfd / _sobel (:218-287) with grid spacings deltas[3]
 * (y, x, z).  in and out hold P floats in linear order. */
aprb_status aprb_gradient(aprb_apr *a, const float *in, float *out, int dimension, float delta, int sobel);
aprb_status aprb_gradient_device(aprb_apr *a, const float *in_dev, float *out_dev, int dimension, float delta,
                                 int sobel, void *stream);
aprb_status aprb_gradient_magnitude(aprb_apr *a, const float *in, float *out, const float *deltas, int sobel);
aprb_status aprb_gradient_magnitude_device(aprb_apr *a, const float *in_dev, float *out_dev, const float *deltas,
                                           int sobel, void *stream);

/* --- APR Richardson-Lucy --------------------------------------------------------
 * APRNumerics::richardson_lucy (APRNumerics.hpp:576-593) /
 * APRNumericsGPU::richardson_lucy (APRNumericsGPU.hpp:105-108).  psf: ksize^3
 * floats; out holds the estimate (read as the start value when resume). */
aprb_status aprb_richardson_lucy(aprb_apr *a, const uint16_t *in, float *out, const float *psf, int ksize, int niter,
                                 int use_stencil_downsample, int normalize, int resume);
aprb_status aprb_richardson_lucy_device(aprb_apr *a, const uint16_t *in_dev, float *out_dev, const float *psf,
                                        int ksize, int niter, int use_stencil_downsample, int normalize, int resume,
                                        void *stream);
/* the reference's FP64 instantiation, APRNumerics::richardson_lucy<uint16_t, double, double>
 * (APRNumerics.hpp:551-593): stencils, tree means, intermediates and output in double; psf is
 * given as float and converted to double before it is flipped and down-sampled */
aprb_status aprb_richardson_lucy_fp64(aprb_apr *a, const uint16_t *in, double *out, const float *psf, int ksize,
                                      int niter, int use_stencil_downsample, int normalize, int resume);
aprb_status aprb_richardson_lucy_fp64_device(aprb_apr *a, const uint16_t *in_dev, double *out_dev, const float *psf,
                                             int ksize, int niter, int use_stencil_downsample, int normalize,
                                             int resume, void *stream);


/* --- learned Richardson-Lucy proposal (no counterpart in the reference) -----------------
 * A sparse CNN on the APR: every layer applies one 3x3x3 stencil of 16 x 16 channels on
 * every level, over the neighbourhood convolve_pencil uses (same-level particles, parents,
 * tree means; zero boundary).  Activations are P x 16 float, channels-last; W is
 * [27 taps][16 out][16 in] float (taps in convolve_pencil's z, x, y memory order), rounded
 * to bfloat16 for the tensor cores with float accumulation.  The network predicts
 * log(u_{i+10} / u_i) from (log(u / (1 + d)), log(ratio), log(1 + d) / 8). */
aprb_status aprb_cnn_layer_forward_device(aprb_apr *a, const float *in, const float *W, const float *bias, int relu,
                                          float *out, void *stream);
/* g_in = dL/d in (overwritten); dW, db accumulate */
aprb_status aprb_cnn_layer_backward_device(aprb_apr *a, const float *in, const float *W, const float *out,
                                           const float *g_out, int relu, float *g_in, float *dW, float *db,
                                           void *stream);
aprb_status aprb_cnn_features_device(const aprb_apr *a, const float *u, const float *ratio, const uint16_t *raw,
                                     float *features, void *stream);
/* loss_dev += mean (pred[:,0] - log(u1 / u0))^2 (zeroed first); g_pred = dloss/dpred */
aprb_status aprb_cnn_loss_device(const aprb_apr *a, const float *pred, const float *u0, const float *u1, float *g_pred,
                                 double *loss_dev, void *stream);
/* the proposal: u <- u * exp(clamp(pred[:,0], -2, 2)) */
aprb_status aprb_cnn_apply_device(const aprb_apr *a, const float *pred, float *u, void *stream);
/* Adam step on n parameters (mask, when not NULL, multiplies the gradient) */
aprb_status aprb_cnn_adam_device(float *params, const float *grads, float *m, float *v, const float *mask, uint64_t n,
                                 float lr, float beta1, float beta2, float eps, int step, void *stream);
/* the RL ratio d / conv(psf_flipped, u) of APRNumerics.hpp:565-566 */
aprb_status aprb_rl_ratio_device(aprb_apr *a, const uint16_t *in_dev, const float *u_dev, float *ratio_dev,
                                 const float *psf, int ksize, int use_stencil_downsample, int normalize,
                                 void *stream);
/* RL's Poisson data-fit objective sum(k - d log k), k = conv(psf_flipped, u); blocking */
aprb_status aprb_rl_objective_device(aprb_apr *a, const uint16_t *in_dev, const float *u_dev, const float *psf,
                                     int ksize, int use_stencil_downsample, int normalize, double *objective,
                                     void *stream);

/* --- synthetic data (benchmark inputs; no reference counterpart) ----------------
 * Background + n_blobs isotropic Gaussians (centre uniform, sigma and peak
 * uniform in the given ranges) + Poisson noise, rounded and clipped to
 * uint16, written to a device buffer of y*x*z elements. Deterministic for a
 * seed. */
aprb_status aprb_synth_blobs_u16(uint16_t *img_dev, int y_num, int x_num, int z_num, int n_blobs, float sigma_lo,
                                 float sigma_hi, float amp_lo, float amp_hi, float background, uint64_t seed,
                                 void *stream);
/* the same blobs without noise, as float intensities (ground truth of the deconvolution workload) */
aprb_status aprb_synth_blobs_f32(float *img_dev, int y_num, int x_num, int z_num, int n_blobs, float sigma_lo,
                                 float sigma_hi, float amp_lo, float amp_hi, float background, uint64_t seed,
                                 void *stream);

/* --- self-check of the division by a kernel constant ---------------------------
 * The box means divide by a window length fixed per launch with a corrected
 * reciprocal product instead of the IEEE division; this runs both on all 2^32
 * float inputs for divisor d on the current device and returns how many
 * results differ in their bits (NaNs compare equal) and the first such input. */
aprb_status aprb_check_division_by_constant(float d, uint64_t *mismatches, uint32_t *first_bits);

/* --- FP32 arithmetic peak (a measurement helper; no counterpart in the reference) ---
 * Times a kernel of independent fused multiply-add chains on the current
 * device and stream and returns its rate in TFLOP/s (two flops per FMA): the
 * denominator for the arithmetic rate of the convolutions. */
aprb_status aprb_measure_fp32_fma_peak(void *stream, double *tflops);

/* number of kernel launches this thread issued through the library so far */
uint64_t aprb_kernel_launch_count(void);

/* --- smoothing schedule (no counterpart in the reference: the kernel choice of the
 * recursive smoothing, bspline_filt_rec_y/x/z, ComputeGradient.hpp:249-779) ---------
 * For float ImageType the three passes run as one of several kernels, chosen per axis
 * (0 y, 1 x, 2 z) and line-length bucket (n <= 128, 256, 512, 1024, 2048, longer: bucket
 * 0 .. 5).  y: 0 cp.async-staged tiles, 1 / 2 TMA tiles with 2 / 3 stages in flight;
 * x and z: 0 register-staged lines, 1 .. 4 TMA segments of (boxes of 256 y, lines per
 * thread, stages) = (1, 2, 4), (2, 4, 3), (1, 1, 4), (2, 2, 3).  Every variant gives the
 * same bits; the default is variant 1 everywhere, and a layout TMA cannot take uses
 * variant 0.  libapr_b200.autotune times the variants on the device and persists the
 * fastest (libapr_b200/data/smoothing_schedule.json, loaded by the Python package).
 * The schedule is process-wide. */
aprb_status aprb_smoothing_variants(int axis, int *count);
aprb_status aprb_smoothing_schedule_set(int axis, int bucket, int variant);
aprb_status aprb_smoothing_schedule_get(int axis, int bucket, int *variant);

/* --- stage timing (the reference's APRTimer stages, APRConverter.hpp:61-65,
 * measured with CUDA events on the launching stream) -------------------------
 * When enabled, every pipeline stage records an event pair on its stream.
 * aprb_profile_read waits for the recorded events and returns, per stage
 * name (in first-seen order), the summed device milliseconds and the number
 * of recordings; it returns the number of stages (at most max). */
aprb_status aprb_profile_enable(int on);
aprb_status aprb_profile_reset(void);
int aprb_profile_read(const char **names, double *ms, uint64_t *count, int max);

#ifdef __cplusplus
}
#endif
#endif
