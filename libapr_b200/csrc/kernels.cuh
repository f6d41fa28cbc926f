// Declarations shared by the kernel translation units of libaprb200.
#pragma once

#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "host_params.hpp"

namespace aprb {

constexpr int kMaxK0 = 256;  // longest folded recursive-filter boundary vector

// particle-cell status codes (PullingScheme.hpp:16-22) and the
// equivalence-optimisation seed (LinearAccess.hpp:265)
constexpr uint8_t kEmpty = 0, kSeed = 1, kBoundary = 2, kFiller = 3, kUpsamplingSeed = 4, kAscendant = 8,
                  kPropagate = 15, kAscendantNeighbour = 16;

struct IIRDev {
    float b1, b2, norm;
    int minLen;
    const float *bc;  // folded boundary vectors bc1..bc4, [4][minLen]
};

struct LisBuffers {
    DevBuf padded, a, c, scalars;
};

// ---- iir_tma.cu
// Smoothing schedule: the kernel variant of each axis (0 y, 1 x, 2 z) per
// line-length bucket (n <= 128, 256, 512, 1024, 2048, longer).  y: 0 the
// cp.async-staged kernel, 1 / 2 TMA tiles with 2 / 3 stages; x, z: 0 the
// register-staged kernel, 1 .. 4 TMA segment shapes.  Variant 1 everywhere
// unless set (a layout TMA cannot take falls back to variant 0).
constexpr int kSchedBuckets = 6;
int sched_bucket(int n);
int smoothing_variants(int axis);
int smoothing_variant(int axis, int n);
bool set_smoothing_variant(int axis, int bucket, int v);
// The x (zaxis false) or z pass of the recursive smoothing over a float image
// with TMA-staged segments; false when the layout does not allow it (y_num not
// a multiple of 4 or below 256, fewer than 16 samples along the axis, an
// unaligned image), and the caller runs the register-staged kernel instead.
// A bounded mbarrier wait that runs out sets *d_timeout.  ckpt holds ckpt_elems
// recurrence states (16-sample segments x lines).
bool launch_strided_iir_tma(float *work, int yn, int xn, int zn, bool zaxis, const IIRDev &c, unsigned *d_timeout,
                            float2 *ckpt, uint64_t ckpt_elems, cudaStream_t s);

// ---- inv_bspline_tma.cu
// weights of the inverse B-spline filter [1/6, 4/6, 1/6] and the mirrored end weight a1 + a3
struct InvB {
    float a1, a2, a3, a13;
};
// calc_inv_bspline_y/x/z over the ds image with TMA-staged planes; false when
// the layout does not allow it (y extent not a multiple of 4 or below 256, x
// extent below 18, unaligned input), and the caller runs inv_bspline_kernel.
bool launch_inv_bspline_tma(const float *in, float *O, int yd, int xd, int zd, int ony, int onx, int onz,
                            const InvB &c, unsigned *d_timeout, cudaStream_t s);

// ---- iir_y_tma.cu
// The y pass of the recursive smoothing of a uint16 image into a float
// working image with TMA-staged tiles; false when the layout does not allow
// it (y_num not a multiple of 8 or below 64, fewer than 32 lines, unaligned
// buffers), and the caller runs the cp.async-staged kernel instead.  ckpt
// holds ckpt_elems recurrence states (64-sample tiles x lines).
bool launch_iir_y_tma(const uint16_t *img, float *work, int yn, uint64_t nlines, const IIRDev &c, unsigned *d_timeout,
                      float2 *ckpt, uint64_t ckpt_elems, cudaStream_t s);

// ---- peaks.cu
// FP32 fused multiply-add throughput of the current device (TFLOP/s, two
// flops per FMA), measured on stream s
double measure_fp32_fma_tflops(cudaStream_t s);

// ---- pipeline.cu
void launch_check_div_const(float d, unsigned long long *out, cudaStream_t s);
void launch_minmax_offset(const uint16_t *img, uint64_t n, unsigned *mm, float *offset, int apply, cudaStream_t s);
template <typename IT>
void launch_smooth(const uint16_t *img, IT *work, int yn, int xn, int zn, float lambda, const float *d_offset,
                   unsigned *d_err, DevBuf &ckpt, cudaStream_t s);
template <typename IT>
void launch_upload_smooth(const uint16_t *host, uint16_t *img, IT *work, int yn, int xn, int zn, float lambda,
                          unsigned *mm, float *d_offset, int apply, unsigned *d_err, DevBuf &ckpt,
                          cudaStream_t s, cudaStream_t up);
template <typename IT>
void launch_gradient(const IT *work, int yn, int xn, int zn, IT *grad, float *ids_raw, float *ids, int yd, int xd,
                     int zd, const aprb_params &p, unsigned *d_timeout, cudaStream_t s);
void launch_local_intensity_scale(const float *ids, float *lis, int yd, int xd, int zd, const aprb_params &p,
                                  LisBuffers &b, cudaStream_t s);
template <typename IT>
void launch_levels(IT *grad, float *lis, const float *ids, uint64_t nd, const float *d_offset, const aprb_params &p,
                   int apr_l_max, int top_level, uint8_t *level, uint8_t *status, int keep, cudaStream_t s);
// cells whose level argument lies within rel of a level boundary, and cells at level >= 1
template <typename IT>
void launch_level_margins(const IT *grad, const float *lis, uint64_t nd, const aprb_params &p, int apr_l_max,
                          double rel, unsigned long long *counts, cudaStream_t s);

// ---- structure.cu
// Particle-cell pyramid: status[l] for pct levels l_min..l_max-1 (dims of
// Geom level l); status[l_max-1] and level_top are filled by launch_levels.
struct Pyramid {
    uint8_t *status[32] = {};
    uint8_t *level[32] = {};
};
void launch_pulling_scheme(const Geom &g, Pyramid &pm, cudaStream_t s, bool fill_pyramid = true);

// z-tiles of the blocked converter (APRConverterBatch.hpp:125-160): planes
// [z0 - gl, zf + gr) of which [z0, zf) belong to the tile.
struct ZTile {
    int z0, zf, gl, gr, pz;
};
ZTile z_tile(int b, int nb, int zn, int zblock, int ghost);
void launch_fill_patch(const Geom &g, Pyramid &pm, const uint8_t *lev_top, const ZTile &t, DevBuf &tmp,
                       cudaStream_t s);
void launch_sample_by_block(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const uint16_t *img,
                            uint16_t *parts, int zblock, int ghost, DevBuf &pyr, cudaStream_t s);
// Linear access structure: writes row counts into xz_end (n_xz entries) and
// scans them; returns the particle count (synchronises the stream once).
uint64_t launch_linear_counts(const Geom &g, Pyramid &pm, uint64_t *xz_end, uint64_t n_xz, int min_type,
                              DevBuf &scan_tmp, cudaStream_t s);
void launch_linear_fill(const Geom &g, const Pyramid &pm, const uint64_t *xz_end, uint16_t *y_vec, int min_type,
                        cudaStream_t s);
void launch_full_resolution_structure(const Geom &g, uint64_t *xz_end, uint16_t *y_vec, cudaStream_t s);
void inclusive_scan_u64(uint64_t *data, uint64_t n, DevBuf &tmp, cudaStream_t s);

// sampling (ParticleData.hpp:222-261)
void launch_sample(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const uint16_t *img,
                   uint16_t *parts, DevBuf &pyr, cudaStream_t s);

// piecewise-constant (or level) image of an APR at full resolution
template <typename V>
void launch_reconstruct(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const V *parts, V *img,
                        bool level, cudaStream_t s);

// pieces of sampling for a host-buffer call that pipelines its transfers
uint16_t *sample_pyramid(const Geom &g, DevBuf &pyr, uint64_t off[32]);
void launch_sample_slab(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const uint16_t *img, int z0,
                        int z1, uint16_t *pyr_top, uint16_t *parts, cudaStream_t s);
void launch_sample_coarse(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, uint16_t *base,
                          const uint64_t off[32], uint16_t *parts, cudaStream_t s);

// sampling into caller-provided scratch (no allocation): the pyramid levels
// below l_max need sample_scratch_elems(g) uint16 elements
uint64_t sample_scratch_elems(const Geom &g);
void launch_sample_scratch(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const uint16_t *img,
                           uint16_t *parts, uint16_t *scratch, cudaStream_t s);

// tree (APR.hpp:633-689)
uint64_t launch_tree_build(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const Geom &tg,
                           uint64_t *t_xz_end, uint64_t t_n_xz, DevBuf &flags, DevBuf &scan_tmp, cudaStream_t s);
void launch_tree_fill(const Geom &tg, const DevBuf &flags, const uint64_t *t_xz_end, uint16_t *t_y_vec,
                      cudaStream_t s);

// ---- filter.cu
struct FilterBuffers {
    DevBuf dense, type, stale, stencils;
};
// APRTreeNumerics::fill_tree_mean, or (stencil != null) APRFilter::convolve_pencil
// whose epilogue is: mode 0 out = conv; mode 1 out = in_u16 / conv (RL ratio);
// mode 2 out = out * conv (RL update).
struct ConvPlan {
    int nstencils = 0;
    std::vector<int> sides;
    std::vector<int> offsets;
    int reflect = 1;
    std::vector<double> values;  // the stencils on the host (exact for float and double), at offsets
};
// Row chunk index of every APR and tree level (built once per APR) and the
// particle count of every APR level.
struct FilterIndex {
    DevBuf buf;
    uint64_t apr_off[32] = {}, tree_off[32] = {};
    uint64_t level_count[32] = {};
    bool built = false;
};
void build_filter_index(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const Geom &tg,
                        const uint64_t *t_xz_end, const uint16_t *t_y_vec, FilterIndex &fi, cudaStream_t s);
// T = float, or double for the FP64 instantiation of richardson_lucy
template <typename T>
void filter_apply(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const Geom &tg,
                  const uint64_t *t_xz_end, const uint16_t *t_y_vec, const FilterIndex &fi, const T *in, T *tree,
                  const ConvPlan *plan, const T *d_stencils, T *out, int mode, const uint16_t *rl_in,
                  FilterBuffers &fb, cudaStream_t s);
uint64_t filter_stale_count(FilterBuffers &fb, cudaStream_t s);
// gradient magnitude (APRNumerics::gradient_magnitude_*): tree means once,
// then per level one neighbourhood image and one pass over the particles with
// the three directions' 3x3x3 stencils (host arrays of nstencils x 27, level
// delta d at stencils[k] + 27 d); active[k] = direction k enters the magnitude
void filter_gradient_magnitude(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const Geom &tg,
                               const uint64_t *t_xz_end, const uint16_t *t_y_vec, const FilterIndex &fi,
                               const float *in, float *tree, const float *const stencils[3], const int active[3],
                               int nstencils, float *out, FilterBuffers &fb, cudaStream_t s);

// ---- learned.cu: the learned RL proposal (a sparse APR CNN, 16 channels)
struct CnnGeom {
    const Geom *g, *tg;
    const uint64_t *xz_end, *t_xz_end;
    const uint16_t *y_vec, *t_y_vec;
    const FilterIndex *fi;
    const uint32_t *prow;        // row (z * x_num + x) of every particle within its level
    uint64_t level_begin[34];    // first particle of each level (level_begin[l_max + 1] = P)
    uint64_t T;                  // tree nodes
};
struct CnnScratch {
    DevBuf tree, gtree, dense, gdense, gp, wt, wbf;
};
void cnn_build_rows(const Geom &g, const uint64_t *xz_end, uint32_t *prow, cudaStream_t s);
// one layer: out = act(conv3x3x3(in) + b), W[27][16 co][16 ci] fp32 (bf16 on the tensor cores)
void cnn_layer_forward(const CnnGeom &cg, const float *in, const float *W, const float *b, int relu, float *out,
                       CnnScratch &sc, cudaStream_t s);
// g_in = d/d in; dW, db accumulated
void cnn_layer_backward(const CnnGeom &cg, const float *in, const float *W, const float *out, const float *g_out,
                        int relu, float *g_in, float *dW, float *db, CnnScratch &sc, cudaStream_t s);
void cnn_adam(float *p, const float *g, float *m, float *v, const float *mask, uint64_t n, float lr, float b1,
              float b2, float eps, int step, cudaStream_t s);
void cnn_features(const float *u, const float *ratio, const uint16_t *raw, float *f, uint64_t P, cudaStream_t s);
void cnn_loss(const float *pred, const float *u0, const float *u1, float *g, uint64_t P, double *loss, cudaStream_t s);
void cnn_apply(const float *pred, float *u, uint64_t P, cudaStream_t s);
void rl_objective_sum(const float *k, const uint16_t *raw, uint64_t P, double *out, cudaStream_t s);

// ---- synth.cu
// OutT uint16_t: blobs + Poisson noise; OutT float: the noise-free intensity
template <typename OutT>
void launch_synth_blobs(OutT *img, int yn, int xn, int zn, int n_blobs, float slo, float shi, float alo, float ahi,
                        float bg, uint64_t seed, DevBuf &blobs, cudaStream_t s);

// ---- autopar.cu
// Scratch of the automatic-parameter step, kept by a converter.
struct AutoParBuffers {
    DevBuf counts, offs, sub_g, sub_l, part, res, ticket;
    bool ticket_ready = false;
};
// threshold_li (AutoParameters.hpp:50-100) on up to two device arrays of m
// values each (T values as float; integer[q] for T = uint16); inactive
// arrays give 0.  Synchronises s.
void threshold_li_pair(const float *const v[2], uint64_t m, const int integer[2], const int active[2],
                       AutoParBuffers &b, cudaStream_t s, float out[2]);
// autoParametersLiEntropy (AutoParameters.hpp:103-153) on the ds image ids,
// gradient grad (ImageType values; grad_integer for uint16_t) and local
// intensity scale lis, nd cells; synchronises s.  n_subsample (may be null)
// receives the subsample length.
template <typename IT>
void auto_parameters(const float *ids, const IT *grad, const float *lis, uint64_t nd, const float *d_off,
                     float Ip_th, int grad_integer, AutoParBuffers &b, cudaStream_t s, float *grad_th,
                     float *sigma_th, uint64_t *n_subsample);

}  // namespace aprb
