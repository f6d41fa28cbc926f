/*
 * TEST INFRASTRUCTURE ONLY -- not part of the product.
 *
 * CPU restatement (plain C, single thread, strict IEEE float: built with
 * -O2 -fno-fast-math -ffp-contract=off) of LibAPR's APR construction and
 * filtering path.  It is the checker for the CUDA implementation in
 * libapr_b200/: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  Each function in apr_oracle.c cites the
 * reference file:line it restates (paths relative to the LibAPR source tree).
 *
 * Memory order of every dense image is the reference's PixelData order:
 * y fastest, then x, then z  (index = z*x_num*y_num + x*y_num + y).
 */
#ifndef APR_ORACLE_H
#define APR_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Mirror of the APRParameters fields the path reads
 * (src/algorithm/APRParameters.hpp:14-41). */
typedef struct {
    float dx, dy, dz;
    float psfx, psfy, psfz;
    float Ip_th, lambda, rel_error, sigma_th, sigma_th_max, grad_th;
    int reflect_bc_lis;
    int neighborhood_optimization;
    int constant_intensity_scale;
} orc_params;

#define ORC_MAX_LEVELS 32

/* Linear access structure (src/data_structures/APR/access/LinearAccess.hpp:33-35)
 * plus the level geometry of GenInfo (src/data_structures/APR/GenInfo.hpp). */
typedef struct {
    int l_min, l_max;
    int org[3];                       /* y, x, z */
    int y_num[ORC_MAX_LEVELS], x_num[ORC_MAX_LEVELS], z_num[ORC_MAX_LEVELS];
    uint64_t level_xz[ORC_MAX_LEVELS + 2];
    uint64_t n_xz;
    uint64_t *xz_end;
    uint64_t P;
    uint16_t *y_vec;
} orc_access;

typedef struct orc_apr orc_apr;

/* error codes */
#define ORC_OK 0
#define ORC_ERR_DIMS 1
#define ORC_ERR_OVERFLOW 2
#define ORC_ERR_ALLOC 3
#define ORC_ERR_ARG 4

/* Full get_apr (APRConverter<IT>::get_apr_cpu) on a uint16 input.
 * image_type: 0 = float ImageType, 1 = uint16 ImageType. */
int orc_get_apr(const uint16_t *img, int y, int x, int z, const orc_params *p,
                int image_type, orc_apr **out);

/* APR from a precomputed down-sampled gradient (IT-valued, stored as float)
 * and local intensity scale, as APRConverter::get_apr_custom_grad_scale
 * (src/algorithm/APRConverter.hpp:170-191) with bspline_offset = 0. */
int orc_get_apr_custom(const float *grad_ds, const float *lis_ds, int y, int x, int z,
                       const orc_params *p, orc_apr **out);

/* Blocked construction, APRConverterBatch<IT> (src/algorithm/APRConverterBatch.hpp:114-175,
 * 190-271, 282-314) with the z-tiles cut from the in-memory volume instead of
 * read from a TIFF file: z tiles of zblock planes (the last one takes the
 * remainder) with up to ghost planes of overlap on each side. */
int orc_get_apr_by_block(const uint16_t *img, int y, int x, int z, const orc_params *p, int image_type,
                         int zblock, int ghost, orc_apr **out);

void orc_free(orc_apr *a);
/* the blocked converter split by tiles: bytes of the flat particle-cell tree,
 * tiles [first, first + count) filling it (slab = planes [slab_z0, ...) of the
 * volume), and the APR of a filled tree (pulling scheme in place) */
size_t orc_pyramid_bytes(int y, int x, int z);
int orc_pyramid_fill_tiles(const uint16_t *slab, int slab_z0, int y, int x, int z, const orc_params *p,
                           int image_type, int zblock, int ghost, int first, int count, uint8_t *pyramid);
int orc_apr_from_pyramid(uint8_t *pyramid, int y, int x, int z, const orc_params *p, orc_apr **out);
const orc_access *orc_get_access(const orc_apr *a);
/* Intermediates kept by orc_get_apr (ds = ceil(dim/2) per axis):
 * which: 0 smoothed full-res image (IT values as float), 1 ds gradient after
 * get_gradient, 2 ds inverse-bspline image (local_scale_temp2), 3 ds local
 * intensity scale after get_local_intensity_scale, 4 ds gradient after
 * applyParameters, 5 ds local intensity scale after applyParameters,
 * 6 ds levels (compute_level_for_array output). */
int orc_copy_intermediate(const orc_apr *a, int which, float *dst, size_t n);
float orc_bspline_offset(const orc_apr *a);

/* Particle sampling: ParticleData::sample_image with the default mean
 * pyramid (src/data_structures/APR/particles/ParticleData.hpp:123-127). */
int orc_sample_image(const orc_access *acc, const uint16_t *img, uint16_t *parts);

/* Blocked sampling, sample_parts_from_img_blocked
 * (src/data_structures/APR/particles/ParticleData.hpp:288-372), tiles from memory. */
int orc_sample_image_by_block(const orc_access *acc, const uint16_t *img, int zblock, int ghost, uint16_t *parts);

/* APR tree of an access structure (APR::initialize_tree_dense,
 * src/data_structures/APR/APR.hpp:633-689); the caller frees with
 * orc_access_free. */
int orc_tree_init(const orc_access *acc, orc_access *tree);
void orc_access_free(orc_access *acc);

/* APRTreeNumerics::fill_tree_mean (src/numerics/APRTreeNumerics.hpp:63-203). */
int orc_fill_tree_mean(const orc_access *acc, const orc_access *tree,
                       const float *parts, float *tree_data);

/* APRStencil::get_downsampled_stencils for a cubic stencil of side ks
 * (src/numerics/APRStencil.hpp:81-95); out receives nlevels stencils packed
 * back to back, sizes in out_sizes (side lengths). Returns total floats. */
int orc_downsampled_stencils(const float *stencil, int ks, int nlevels, int normalize,
                             float *out, int *out_sides);

/* APRFilter::convolve_pencil (src/numerics/APRFilter.hpp:1094-1216) with the
 * per-level stencils of orc_downsampled_stencils.  stale_reads counts
 * neighbourhood cells that the reference would leave unfilled. */
int orc_convolve(const orc_access *acc, const orc_access *tree, const float *stencils,
                 const int *sides, int nstencils, const float *in, float *out,
                 int reflect, uint64_t *stale_reads);

/* APRNumerics::richardson_lucy (src/numerics/APRNumerics.hpp:551-593) in FP32
 * (use_double = 0) or FP64 (use_double = 1) arithmetic. out holds the
 * estimate (as double when use_double, else float); resume keeps it. */
int orc_richardson_lucy(const orc_access *acc, const orc_access *tree, const uint16_t *in,
                        void *out, const float *psf, int ks, int niter, int use_stencil_ds,
                        int normalize, int resume, int use_double);

/* ComputeGradient IIR passes on a float image holding IT values
 * (src/algorithm/ComputeGradient.hpp:249-779); returns overflow count. */
uint64_t orc_bspline_axis(float *img, int y, int x, int z, int axis, float lambda, int is_u16);

/* Li's minimum cross entropy threshold, threshold_li<T>
 * (src/algorithm/AutoParameters.hpp:50-100), on T values held as float.
 * integer_values selects T = uint16 (tolerance 0.5, initial value raised
 * towards 1.5, :63-78), else T = float.  fp32_sums = 1 sums in float in index
 * order, as the reference does at one OpenMP thread (std::accumulate :71,
 * compute_means :17-36); fp32_sums = 0 sums in double and rounds each mean to
 * float once, as libaprb200 does.  At most 1000 Li steps. */
float orc_threshold_li(const float *v, size_t n, int integer_values, int fp32_sums);

/* autoParametersLiEntropy (src/algorithm/AutoParameters.hpp:103-153): the
 * gradient and local intensity scale at the pixels whose ds image value
 * exceeds threshold (= Ip_th + bspline_offset), uniformly subsampled to at
 * most 32*512*512 values, each thresholded by orc_threshold_li.  sub_grad and
 * sub_lis (capacity n, may be NULL) receive the subsample, *m its length. */
int orc_auto_parameters(const float *image, const float *lis, const float *grad, size_t n, float threshold,
                        int grad_integer, int fp32_sums, float *grad_th, float *sigma_th, float *sub_grad,
                        float *sub_lis, size_t *m);

#ifdef __cplusplus
}
#endif
#endif
