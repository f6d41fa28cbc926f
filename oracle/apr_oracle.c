/*
 * TEST INFRASTRUCTURE ONLY -- not part of the product.
 *
 * Plain-C restatement of LibAPR's APR construction (get_apr) and filtering
 * (fill_tree_mean, convolve_pencil, richardson_lucy) CPU path.  It is the
 * checker the CUDA implementation is compared against; it must be compiled
 * with -O2 -fno-fast-math -ffp-contract=off so that every float operation
 * rounds exactly where the reference's strict-IEEE build rounds.
 *
 * Citations are file:line in the LibAPR source tree.  Where the reference
 * evaluates an expression through the double-precision libm overloads
 * (unqualified sqrt/pow/cos/log/atan on float arguments resolve to the
 * double functions in the global namespace), this file makes the double
 * evaluation explicit.
 *
 * Parity of this restatement is pinned in tests/ against (a) the reference's
 * golden TIFF fixtures (gradient/scale/level/coordinate/intensity images of
 * the sphere test volumes) and (b) the reference's own CPU code compiled
 * from its headers into oracle/_ref by oracle/Makefile.
 */
#include "apr_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define IDX(y, x, z, yn, xn) ((size_t)(z) * (size_t)(xn) * (size_t)(yn) + (size_t)(x) * (size_t)(yn) + (size_t)(y))

/* ------------------------------------------------------------------------ */
/* ImageType emulation.  The working image is kept as float; when ImageType  */
/* is uint16 every store converts like the x86-64 g++ build of the          */
/* reference does (cvttss2si to 32 bit, low 16 bits kept).                   */
/* ------------------------------------------------------------------------ */
static inline float cvt_u16(float v) {
    if (!(v > -2147483648.0f && v < 2147483648.0f)) return 0.0f;
    return (float)(uint16_t)(int32_t)v;
}

/* double -> uint16_t (cvttsd2si to 32 bit, low 16 bits kept) */
static inline float cvt_u16d(double v) {
    if (!(v > -2147483648.0 && v < 2147483648.0)) return 0.0f;
    return (float)(uint16_t)(int32_t)v;
}

static inline float store_it(float v, int is_u16) { return is_u16 ? cvt_u16(v) : v; }

/* round<T> (src/algorithm/ComputeGradient.hpp:220-244) */
static inline float round_it(float v, int is_u16, uint64_t *err) {
    if (!is_u16) return v;
    v = roundf(v);
    if (v < 0.0f || v > 65535.0f) (*err)++;
    return cvt_u16(v);
}

/* float -> uint32_t as emitted by g++ on x86-64 (cvttss2si to 64 bit, low 32
 * bits kept; NaN and |v| >= 2^63 give 0x8000000000000000). */
static inline uint32_t cvt_u32(float v) {
    if (!(v > -9223372036854775808.0f && v < 9223372036854775808.0f)) return 0u;
    return (uint32_t)(int64_t)v;
}

/* ------------------------------------------------------------------------ */
/* Level geometry: GenInfo::init / init_tree (src/data_structures/APR/GenInfo.hpp:33-98) */
/* ------------------------------------------------------------------------ */
static double powr(double num, double p) { return round(pow(num, p)); }

static void geninfo_init(orc_access *a, int y, int x, int z) {
    memset(a, 0, sizeof(*a));
    a->org[0] = y; a->org[1] = x; a->org[2] = z;
    int max_dim = x > y ? x : y;
    if (z > max_dim) max_dim = z;
    int lm = (int)ceil(log2((double)max_dim));
    if (lm < 1) lm = 1;
    a->l_min = 1;
    a->l_max = lm;
    for (int l = a->l_min; l <= a->l_max; ++l) {
        double cell = powr(2, lm - l);
        a->y_num[l] = (int)ceil((double)(uint64_t)y / cell);
        a->x_num[l] = (int)ceil((double)(uint64_t)x / cell);
        a->z_num[l] = (int)ceil((double)(uint64_t)z / cell);
    }
}

static void geninfo_init_tree(orc_access *a, int y, int x, int z) {
    memset(a, 0, sizeof(*a));
    a->org[0] = y; a->org[1] = x; a->org[2] = z;
    int max_dim = x > y ? x : y;
    if (z > max_dim) max_dim = z;
    int lm = (int)ceil(log2((double)max_dim));
    a->l_min = 0;
    a->l_max = lm - 1 > 0 ? lm - 1 : 0;
    for (int l = a->l_min; l <= a->l_max; ++l) {
        double cell = powr(2, a->l_max - l + 1);
        a->y_num[l] = (int)ceil((double)(uint64_t)y / cell);
        a->x_num[l] = (int)ceil((double)(uint64_t)x / cell);
        a->z_num[l] = (int)ceil((double)(uint64_t)z / cell);
    }
}

/* LinearAccess::initialize_xz_linear (src/data_structures/APR/access/LinearAccess.hpp:37-54) */
static int init_xz_linear(orc_access *a) {
    uint64_t counter = 1;
    memset(a->level_xz, 0, sizeof(a->level_xz));
    a->level_xz[0] = 1;
    for (int i = 0; i <= a->l_max; ++i) {
        counter += (uint64_t)a->x_num[i] * (uint64_t)a->z_num[i];
        a->level_xz[i + 1] = counter;
    }
    a->n_xz = counter;
    a->xz_end = (uint64_t *)calloc(counter, sizeof(uint64_t));
    return a->xz_end ? ORC_OK : ORC_ERR_ALLOC;
}

void orc_access_free(orc_access *acc) {
    if (!acc) return;
    free(acc->xz_end);
    free(acc->y_vec);
    acc->xz_end = NULL;
    acc->y_vec = NULL;
}

static inline uint64_t row_begin(const orc_access *a, int l, int z, int x) {
    return a->xz_end[a->level_xz[l] + (uint64_t)z * a->x_num[l] + x - 1];
}
static inline uint64_t row_end(const orc_access *a, int l, int z, int x) {
    return a->xz_end[a->level_xz[l] + (uint64_t)z * a->x_num[l] + x];
}

/* ------------------------------------------------------------------------ */
/* a2: smoothing B-spline recursive filter coefficients                      */
/* (src/algorithm/ComputeGradient.hpp:256-330, 176-186)                      */
/* ------------------------------------------------------------------------ */
typedef struct {
    float b1, b2, norm;
    size_t k0, minLen;
    float *bc1, *bc2, *bc3, *bc4;
} iir_t;

static float impulse_resp(float k, float rho, float omg) {
    float ak = fabsf(k);
    return (float)((pow((double)rho, (double)ak) * sin((double)((ak + 1) * omg))) / sin((double)omg));
}

static float impulse_resp_back(float k, float rho, float omg, float gamma, float c0) {
    float ak = fabsf(k);
    double p2 = pow((double)rho, 2.0);
    double den = pow((1.0 - 2.0 * (double)rho * cos((double)omg) + p2), 2.0);
    return (float)((double)c0 * pow((double)rho, (double)ak) *
                   (cos((double)(omg * ak)) + (double)gamma * sin((double)(omg * ak))) * (1.0 / den));
}

static int iir_setup(float lambda, size_t dim, iir_t *c) {
    const float tol = 0.0001f;
    float xi = (float)((double)(1.0f - 96.0f * lambda) +
                       (double)(24.0f * lambda) * sqrt((double)(3.0f + 144.0f * lambda)));
    double inner = (double)(48.0f * lambda) + (double)(24.0f * lambda) * sqrt((double)(3.0f + 144.0f * lambda));
    float rho = (float)(((double)(24.0f * lambda - 1.0f) - sqrt((double)xi)) / (double)(24.0f * lambda) *
                        sqrt((double)(1.0f / xi) * inner));
    float omg = (float)atan(sqrt((double)((1.0f / xi) * (144.0f * lambda - 1.0f))));
    double p2 = pow((double)rho, 2.0);
    double cw = cos((double)omg);
    float c0 = (float)((1.0 + p2) / (1.0 - p2) * (1.0 - (double)(2.0f * rho) * cw + p2) /
                       (1.0 + (double)(2.0f * rho) * cw + p2));
    float gamma = (float)((1.0 - p2) / (1.0 + p2) * (1.0 / tan((double)omg)));
    c->b1 = (float)((double)(2.0f * rho) * cw);
    c->b2 = (float)(-pow((double)rho, 2.0));
    size_t k0 = (size_t)ceil(fabs(log((double)tol) / log((double)rho)));
    c->k0 = k0;
    c->minLen = k0 < dim ? k0 : dim;
    c->norm = (float)pow((1.0 - 2.0 * (double)rho * cw + p2), 2.0);

    float *irf = (float *)calloc(k0 + 3, sizeof(float));
    float *irb = (float *)calloc(k0 + 3, sizeof(float));
    c->bc1 = (float *)calloc(k0, sizeof(float));
    c->bc2 = (float *)calloc(k0, sizeof(float));
    c->bc3 = (float *)calloc(k0, sizeof(float));
    c->bc4 = (float *)calloc(k0, sizeof(float));
    if (!irf || !irb || !c->bc1 || !c->bc2 || !c->bc3 || !c->bc4 || k0 < 2) {
        free(irf); free(irb);
        return ORC_ERR_ALLOC;
    }
    for (size_t k = 0; k < k0 + 3; ++k) irf[k] = impulse_resp((float)k, rho, omg);
    for (size_t k = 0; k < k0 + 3; ++k) irb[k] = impulse_resp_back((float)k, rho, omg, gamma, c0);
    size_t m = c->minLen;
    c->bc1[1] = irf[0];
    for (size_t k = 0; k < k0; ++k) c->bc1[k] += irf[k + 1];
    for (size_t k = m; k < k0; ++k) c->bc1[m - 1] += c->bc1[k];
    for (size_t k = 0; k < k0; ++k) c->bc2[k] = irf[k];
    for (size_t k = m; k < k0; ++k) c->bc2[m - 1] += c->bc2[k];
    c->bc3[0] = irb[1];
    for (size_t k = 0; k < k0 - 1; ++k) c->bc3[k + 1] += irb[k] + irb[k + 2];
    for (size_t k = m; k < k0; ++k) c->bc3[m - 1] += c->bc3[k];
    c->bc4[0] = irb[0];
    for (size_t k = 1; k < k0; ++k) c->bc4[k] += 2 * irb[k];
    for (size_t k = m; k < k0; ++k) c->bc4[m - 1] += c->bc4[k];
    free(irf); free(irb);
    return ORC_OK;
}

static void iir_free(iir_t *c) {
    free(c->bc1); free(c->bc2); free(c->bc3); free(c->bc4);
}

/* bspline_filt_rec_y (src/algorithm/ComputeGradient.hpp:249-413) */
static uint64_t bspline_y(float *im, int yn, int xn, int zn, float lambda, int is_u16) {
    iir_t c;
    if (iir_setup(lambda, (size_t)yn, &c) != ORC_OK) return (uint64_t)-1;
    uint64_t err = 0;
    const size_t m = c.minLen;
    for (int z = 0; z < zn; ++z) {
        for (int x = 0; x < xn; ++x) {
            float *I = im + IDX(0, x, z, yn, xn);
            float t1 = 0, t2 = 0, t3 = 0, t4 = 0;
            for (size_t k = 0; k < m; ++k) {
                t1 += c.bc1[k] * I[k];
                t2 += c.bc2[k] * I[k];
            }
            for (size_t k = 0; k < m; ++k) {
                t3 += c.bc3[k] * I[yn - 1 - k];
                t4 += c.bc4[k] * I[yn - 1 - k];
            }
            I[0] = store_it(t2, is_u16);
            I[1] = store_it(t1, is_u16);
            for (int k = 2; k < yn; ++k) {
                float temp = t1 * c.b1 + t2 * c.b2 + I[k];
                I[k] = round_it(temp, is_u16, &err);
                t2 = t1;
                t1 = temp;
            }
            I[yn - 2] = round_it(t3 * c.norm, is_u16, &err);
            I[yn - 1] = round_it(t4 * c.norm, is_u16, &err);
        }
    }
    for (int z = zn - 1; z >= 0; --z) {
        for (int x = xn - 1; x >= 0; --x) {
            float *I = im + IDX(0, x, z, yn, xn);
            float t2 = I[yn - 1] / c.norm;
            float t1 = I[yn - 2] / c.norm;
            for (int k = yn - 3; k >= 0; --k) {
                float temp = t1 * c.b1 + t2 * c.b2 + I[k];
                I[k] = round_it(temp * c.norm, is_u16, &err);
                t2 = t1;
                t1 = temp;
            }
        }
    }
    iir_free(&c);
    return err;
}

/* bspline_filt_rec_x (src/algorithm/ComputeGradient.hpp:602-779) and
 * bspline_filt_rec_z (:416-599): identical recursions along a strided axis.
 * Runs one line of n samples at stride s. */
static void bspline_strided_line(float *I, size_t s, int n, const iir_t *c, int is_u16, uint64_t *err) {
    const size_t m = c->minLen;
    float v1 = 0, v2 = 0, v3 = 0, v4 = 0;
    for (size_t i = 0; i < m; ++i) {
        v1 += c->bc1[i] * I[i * s];
        v2 += c->bc2[i] * I[i * s];
        v3 += c->bc3[i] * I[(n - 1 - i) * s];
        v4 += c->bc4[i] * I[(n - 1 - i) * s];
    }
    I[0] = round_it(v2, is_u16, err);
    I[s] = round_it(v1, is_u16, err);
    for (int i = 2; i < n; ++i) {
        float nv = round_it(I[i * s] + c->b1 * v1 + c->b2 * v2, is_u16, err);
        v2 = v1;
        v1 = nv;
        I[i * s] = nv;
    }
    I[(n - 1) * s] = round_it(v4 * c->norm, is_u16, err);
    I[(n - 2) * s] = round_it(v3 * c->norm, is_u16, err);
    for (int i = n - 3; i >= 0; --i) {
        float temp = (I[i * s] + c->b1 * v3 + c->b2 * v4);
        I[i * s] = round_it(temp * c->norm, is_u16, err);
        v4 = v3;
        v3 = temp;
    }
}

uint64_t orc_bspline_axis(float *img, int yn, int xn, int zn, int axis, float lambda, int is_u16) {
    if (axis == 0) return bspline_y(img, yn, xn, zn, lambda, is_u16);
    iir_t c;
    int n = axis == 1 ? xn : zn;
    if (iir_setup(lambda, (size_t)n, &c) != ORC_OK) return (uint64_t)-1;
    uint64_t err = 0;
    if (axis == 1) {
        for (int z = 0; z < zn; ++z)
            for (int y = 0; y < yn; ++y)
                bspline_strided_line(img + IDX(y, 0, z, yn, xn), (size_t)yn, xn, &c, is_u16, &err);
    } else {
        for (int x = 0; x < xn; ++x)
            for (int y = 0; y < yn; ++y)
                bspline_strided_line(img + IDX(y, x, 0, yn, xn), (size_t)yn * xn, zn, &c, is_u16, &err);
    }
    iir_free(&c);
    return err;
}

/* ------------------------------------------------------------------------ */
/* a3: calc_bspline_fd_ds_mag (src/algorithm/ComputeGradient.hpp:976-1051)  */
/* ------------------------------------------------------------------------ */
static void gradient_ds(const float *im, int yn, int xn, int zn, float *grad, int yd, int xd, int zd,
                        float hx, float hy, float hz, int is_u16) {
    float *temp = (float *)calloc((size_t)yn, sizeof(float));
    memset(grad, 0, sizeof(float) * (size_t)yd * xd * zd);
    for (int z = 0; z < zn; ++z) {
        int zm = z > 0 ? z - 1 : 0;
        int zp = z + 1 < zn - 1 ? z + 1 : zn - 1;
        for (int x = 0; x < xn; ++x) {
            int xl = x > 0 ? x - 1 : 0;
            int xr = x + 1 < xn - 1 ? x + 1 : xn - 1;
            const float *left = im + IDX(0, xl, z, yn, xn);
            const float *center = im + IDX(0, x, z, yn, xn);
            const float *right = im + IDX(0, xr, z, yn, xn);
            const float *up = im + IDX(0, x, zm, yn, xn);
            const float *down = im + IDX(0, x, zp, yn, xn);
            for (int y = 0; y < yn; ++y) {
                int ym, yp;
                if (yn < 2) { temp[0] = 0; break; }
                ym = y > 0 ? y - 1 : 0;
                yp = y < yn - 1 ? y + 1 : yn - 1;
                float gx = (right[y] - left[y]) / (2 * hx);
                float gz = (down[y] - up[y]) / (2 * hz);
                float gy = (center[yp] - center[ym]) / (2 * hy);
                double s = pow((double)gx, 2.0) + pow((double)gz, 2.0) + pow((double)gy, 2.0);
                temp[y] = is_u16 ? cvt_u16d(sqrt(s)) : (float)sqrt(s);
            }
            for (int k = 0; k < yd; ++k) {
                int ks = 2 * k + 1 < yn - 1 ? 2 * k + 1 : yn - 1;
                size_t idx = IDX(k, x / 2, z / 2, yd, xd);
                float a = temp[ks] > grad[idx] ? temp[ks] : grad[idx];
                grad[idx] = temp[2 * k] > a ? temp[2 * k] : a;
            }
        }
    }
    free(temp);
}

/* ------------------------------------------------------------------------ */
/* a4: downsample (src/data_structures/Mesh/PixelData.hpp:916-967)            */
/* ------------------------------------------------------------------------ */
enum { DS_MEAN_D8 = 0, DS_MAX = 1, DS_MEAN_U16 = 2 };

static void downsample2(const float *in, int yn, int xn, int zn, float *out, int mode) {
    int yd = (int)ceil(yn / 2.0), xd = (int)ceil(xn / 2.0), zd = (int)ceil(zn / 2.0);
    for (int z = 0; z < zd; ++z) {
        for (int x = 0; x < xd; ++x) {
            int shx = 2 * x + 1 < xn - 1 ? 2 * x + 1 : xn - 1;
            int shz = 2 * z + 1 < zn - 1 ? 2 * z + 1 : zn - 1;
            for (int y = 0; y < yd; ++y) {
                int shy = 2 * y + 1 < yn - 1 ? 2 * y + 1 : yn - 1;
                float v[8] = {in[IDX(2 * y, 2 * x, 2 * z, yn, xn)], in[IDX(shy, 2 * x, 2 * z, yn, xn)],
                              in[IDX(2 * y, shx, 2 * z, yn, xn)],   in[IDX(shy, shx, 2 * z, yn, xn)],
                              in[IDX(2 * y, 2 * x, shz, yn, xn)],   in[IDX(shy, 2 * x, shz, yn, xn)],
                              in[IDX(2 * y, shx, shz, yn, xn)],     in[IDX(shy, shx, shz, yn, xn)]};
                float r = v[0];
                if (mode == DS_MAX) {
                    for (int i = 1; i < 8; ++i) r = r > v[i] ? r : v[i];
                    out[IDX(y, x, z, yd, xd)] = r;
                } else {
                    for (int i = 1; i < 8; ++i) r = r + v[i];
                    if (mode == DS_MEAN_D8)
                        out[IDX(y, x, z, yd, xd)] = (float)((double)r / 8.0);
                    else
                        out[IDX(y, x, z, yd, xd)] = cvt_u16(r / 8.0f);
                }
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* a5: calc_inv_bspline_y/x/z (src/algorithm/ComputeGradient.hpp:785-964)    */
/* ------------------------------------------------------------------------ */
static void inv_bspline_y(float *im, int yn, int xn, int zn) {
    const float a1 = (float)(1.0 / 6.0), a2 = (float)(4.0 / 6.0), a3 = (float)(1.0 / 6.0);
    float *t = (float *)malloc(sizeof(float) * (size_t)yn);
    for (int z = 0; z < zn; ++z)
        for (int x = 0; x < xn; ++x) {
            float *I = im + IDX(0, x, z, yn, xn);
            memcpy(t, I, sizeof(float) * (size_t)yn);
            I[0] = a2 * t[0];
            I[0] += (a1 + a3) * t[1];
            for (int k = 1; k < yn - 1; ++k) I[k] = a1 * t[k - 1] + a2 * t[k] + a3 * t[k + 1];
            I[yn - 1] = (a1 + a3) * t[yn - 2];
            I[yn - 1] += a2 * t[yn - 1];
        }
    free(t);
}

/* x and z share one form: leading mirror folded into the first tap. */
static void inv_bspline_strided(float *I, size_t s, int n) {
    const float a1 = (float)(1.0 / 6.0), a2 = (float)(4.0 / 6.0), a3 = (float)(1.0 / 6.0);
    float t1 = I[s], t2 = I[0];
    for (int j = 0; j < n - 1; ++j) {
        float t3 = I[(j + 1) * s];
        I[j * s] = a1 * t1 + a2 * t2 + a3 * t3;
        t1 = t2;
        t2 = t3;
    }
    I[(n - 1) * s] = (a1 + a3) * t1;
    I[(n - 1) * s] += a2 * t2;
}

/* ------------------------------------------------------------------------ */
/* a6: local intensity scale (src/algorithm/LocalIntensityScale.hpp)        */
/* ------------------------------------------------------------------------ */
typedef struct {
    int active[3];
    int win1[3], win2[3];
    int n_active;
    float rescale;
} lis_win_t;

/* get_window_alt (:250-303) */
static void lis_window(const orc_params *p, int yn, int xn, int zn, lis_win_t *w) {
    static const double r3[6] = {12.8214, 26.1256, 40.2795, 23.3692, 36.2061, 27.0385};
    static const double r2[6] = {13.2421, 28.7069, 52.0385, 24.4272, 34.9565, 21.1891};
    static const double r1[6] = {13.9040, 31.2843, 57.4037, 30.3767, 45.9930, 29.0890};
    static const int w1[6] = {1, 1, 1, 2, 2, 3};
    static const int w2[6] = {2, 3, 4, 4, 5, 6};
    float fi = (float)(round((double)(p->psfx / p->dx)) - 1);
    int psf_ind = (int)(fi > 0.0f ? fi : 0.0f);
    if (psf_ind > 5) psf_ind = 5;
    int win_val = w1[psf_ind] > w2[psf_ind] ? w1[psf_ind] : w2[psf_ind];
    int dims[3] = {yn, xn, zn};
    w->n_active = 0;
    for (int a = 0; a < 3; ++a) {
        w->active[a] = dims[a] > win_val;
        w->win1[a] = w->active[a] ? w1[psf_ind] : 0;
        w->win2[a] = w->active[a] ? w2[psf_ind] : 0;
        w->n_active += w->active[a];
    }
    if (w->n_active == 3) w->rescale = (float)r3[psf_ind];
    else if (w->n_active == 2) w->rescale = (float)r2[psf_ind];
    else w->rescale = (float)r1[psf_ind];
}

/* calc_sat_mean_y (:311-362) */
static void sat_mean_y(float *im, int yn, int xn, int zn, size_t off) {
    float *cs = (float *)malloc(sizeof(float) * (size_t)yn);
    float divisor = (float)(2 * off + 1);
    for (int z = 0; z < zn; ++z)
        for (int x = 0; x < xn; ++x) {
            float *I = im + IDX(0, x, z, yn, xn);
            float temp = 0;
            for (int k = 0; k < yn; ++k) { temp += I[k]; cs[k] = temp; }
            for (size_t k = 0; k <= off; ++k) I[k] = 0;
            for (size_t k = off + 1; k < (size_t)yn; ++k) I[k] = -cs[k - off - 1] / divisor;
            for (size_t k = 0; k < (size_t)yn - off; ++k) I[k] += cs[k + off] / divisor;
            float counter = 0;
            for (size_t k = (size_t)yn - off; k < (size_t)yn; ++k) {
                counter++;
                I[k] *= divisor;
                I[k] += cs[yn - 1];
                I[k] = (float)((double)I[k] * (1.0 / (double)(divisor - counter)));
            }
            for (size_t k = 1; k <= off; ++k) I[k] = (float)((double)I[k] * ((double)divisor / ((double)k + (double)off + 1.0)));
            I[0] = (float)((double)I[0] * ((double)divisor / ((double)off + 1.0)));
        }
    free(cs);
}

/* calc_sat_mean_x (:364-427) and calc_sat_mean_z (:429-494): ring of 2*off+1
 * cumulative sums along a strided axis; one line of n samples at stride s. */
static void sat_mean_strided_line(float *I, size_t s, size_t n, size_t off, float *ring) {
    size_t w = 2 * off + 1;
    ring[0] = I[0];
    for (size_t i = 1; i < w; ++i) ring[i] = I[i * s] + ring[i - 1];
    for (size_t i = 0; i < off + 1; ++i) I[i * s] = ring[i + off] / (float)(i + off + 1);
    size_t cur = off + 1, im = 0;
    for (size_t i = off + 1; i < n - off; ++i) {
        im = (cur + off) % w;
        size_t prev = (cur + off - 1) % w;
        float temp = I[(i + off) * s] + ring[prev];
        I[i * s] = (temp - ring[im]) / (float)(2 * off + 1);
        ring[im] = temp;
        cur = (cur + 1) % w;
    }
    cur = (cur + off) % w;
    for (size_t i = n - off; i < n; ++i) {
        I[i * s] = (ring[im] - ring[cur]) / (float)(n - i + off);
        cur = (cur + 1) % w;
    }
}

/* paddPixels (src/data_structures/Mesh/PixelData.hpp:1071-1178): reflection
 * about the edge sample, size bounded by dim-1. */
static float *pad_reflect(const float *in, int yn, int xn, int zn, int *sy, int *sx, int *sz, int *py, int *px, int *pz) {
    *sy = yn > 1 ? (*sy < yn - 1 ? *sy : yn - 1) : 0;
    *sx = xn > 1 ? (*sx < xn - 1 ? *sx : xn - 1) : 0;
    *sz = zn > 1 ? (*sz < zn - 1 ? *sz : zn - 1) : 0;
    *py = yn + 2 * *sy; *px = xn + 2 * *sx; *pz = zn + 2 * *sz;
    float *out = (float *)malloc(sizeof(float) * (size_t)*py * *px * *pz);
    for (int z = 0; z < *pz; ++z) {
        int rz = z - *sz; if (rz < 0) rz = -rz; if (rz > zn - 1) rz = 2 * (zn - 1) - rz;
        for (int x = 0; x < *px; ++x) {
            int rx = x - *sx; if (rx < 0) rx = -rx; if (rx > xn - 1) rx = 2 * (xn - 1) - rx;
            for (int y = 0; y < *py; ++y) {
                int ry = y - *sy; if (ry < 0) ry = -ry; if (ry > yn - 1) ry = 2 * (yn - 1) - ry;
                out[IDX(y, x, z, *py, *px)] = in[IDX(ry, rx, rz, yn, xn)];
            }
        }
    }
    return out;
}

static void sat_mean_axis(float *im, int yn, int xn, int zn, int axis, int off) {
    if (axis == 0) { sat_mean_y(im, yn, xn, zn, (size_t)off); return; }
    float *ring = (float *)malloc(sizeof(float) * (2 * (size_t)off + 1));
    if (axis == 1) {
        for (int z = 0; z < zn; ++z)
            for (int y = 0; y < yn; ++y)
                sat_mean_strided_line(im + IDX(y, 0, z, yn, xn), (size_t)yn, (size_t)xn, (size_t)off, ring);
    } else {
        for (int x = 0; x < xn; ++x)
            for (int y = 0; y < yn; ++y)
                sat_mean_strided_line(im + IDX(y, x, 0, yn, xn), (size_t)yn * xn, (size_t)zn, (size_t)off, ring);
    }
    free(ring);
}

/* get_local_intensity_scale (:26-150): returns the scale in lis (ds dims);
 * ids (the inverse-bspline image) is left unchanged. */
static void local_intensity_scale(const float *ids, int yn, int xn, int zn, const orc_params *p, float *lis) {
    lis_win_t w;
    lis_window(p, yn, xn, zn, &w);
    size_t n = (size_t)yn * xn * zn;
    if (p->constant_intensity_scale || w.n_active == 0) {
        float min_val = 660000;
        double sum = 0;
        for (size_t i = 0; i < n; ++i) {
            float t = ids[i];
            sum += t;
            if (t < min_val) min_val = t;
        }
        float numel = (float)(yn * xn * zn);
        float sv = (float)(sum / numel - min_val);
        for (size_t i = 0; i < n; ++i) lis[i] = sv;
        return;
    }
    int sy = w.win1[0] > w.win2[0] ? w.win1[0] : w.win2[0];
    int sx = w.win1[1] > w.win2[1] ? w.win1[1] : w.win2[1];
    int sz = w.win1[2] > w.win2[2] ? w.win1[2] : w.win2[2];
    int py = yn, px = xn, pz = zn;
    float *a, *b;
    if (p->reflect_bc_lis) {
        a = pad_reflect(ids, yn, xn, zn, &sy, &sx, &sz, &py, &px, &pz);
        b = (float *)malloc(sizeof(float) * (size_t)py * px * pz);
        memcpy(b, a, sizeof(float) * (size_t)py * px * pz);
    } else {
        sy = sx = sz = 0;
        a = (float *)malloc(sizeof(float) * n);
        b = (float *)malloc(sizeof(float) * n);
        memcpy(a, ids, sizeof(float) * n);
        memcpy(b, ids, sizeof(float) * n);
    }
    size_t pn = (size_t)py * px * pz;
    for (int ax = 0; ax < 3; ++ax)
        if (w.active[ax]) sat_mean_axis(a, py, px, pz, ax, w.win1[ax]);
    for (size_t i = 0; i < pn; ++i) a[i] = fabsf(a[i] - b[i]);
    for (int ax = 0; ax < 3; ++ax)
        if (w.active[ax]) sat_mean_axis(a, py, px, pz, ax, w.win2[ax]);
    for (size_t i = 0; i < pn; ++i) a[i] = a[i] * w.rescale;
    int oy = (py - yn) / 2, ox = (px - xn) / 2, oz = (pz - zn) / 2;
    for (int z = 0; z < zn; ++z)
        for (int x = 0; x < xn; ++x)
            for (int y = 0; y < yn; ++y) lis[IDX(y, x, z, yn, xn)] = a[IDX(y + oy, x + ox, z + oz, py, px)];
    free(a);
    free(b);
}

/* ------------------------------------------------------------------------ */
/* a9-a11: particle-cell pyramid, pulling scheme, linear structure          */
/* ------------------------------------------------------------------------ */
#define PS_EMPTY 0
#define PS_SEED 1
#define PS_BOUNDARY 2
#define PS_FILLER 3
#define PS_ASCENDANT 8
#define PS_PROPOGATE 15
#define PS_ASCENDANTNEIGHBOUR 16

typedef struct {
    int l_min, l_max;
    int y_num[ORC_MAX_LEVELS], x_num[ORC_MAX_LEVELS], z_num[ORC_MAX_LEVELS];
    uint8_t *m[ORC_MAX_LEVELS];
} pct_t;

static void pct_free(pct_t *t) {
    for (int l = 0; l < ORC_MAX_LEVELS; ++l) free(t->m[l]);
}

/* PullingScheme::initialize_particle_cell_tree (src/algorithm/PullingScheme.hpp:92-104) */
static void pct_init(pct_t *t, const orc_access *g) {
    memset(t, 0, sizeof(*t));
    t->l_max = g->l_max - 1;
    t->l_min = g->l_min;
    for (int l = t->l_min; l <= t->l_max; ++l) {
        double cell = powr(2, t->l_max - l + 1);
        t->y_num[l] = (int)ceil(g->org[0] / cell);
        t->x_num[l] = (int)ceil(g->org[1] / cell);
        t->z_num[l] = (int)ceil(g->org[2] / cell);
        t->m[l] = (uint8_t *)calloc((size_t)t->y_num[l] * t->x_num[l] * t->z_num[l], 1);
    }
}

/* PullingScheme::fill (:137-168) */
static void pct_fill(pct_t *t, int k, const float *lv) {
    size_t n = (size_t)t->y_num[k] * t->x_num[k] * t->z_num[k];
    float kf = (float)k;
    for (size_t i = 0; i < n; ++i) {
        int s;
        if (k == t->l_max) s = lv[i] >= kf;
        else if (k == t->l_min) s = lv[i] <= kf;
        else s = lv[i] == kf;
        if (s) t->m[k][i] = PS_SEED;
    }
}

/* LocalParticleCellSet::get_local_particle_cell_set (src/algorithm/LocalParticleCellSet.hpp:59-91) */
static void local_particle_cell_set(pct_t *t, const float *levels, int yd, int xd, int zd) {
    pct_fill(t, t->l_max, levels);
    size_t n = (size_t)yd * xd * zd;
    float *cur = (float *)malloc(sizeof(float) * n);
    memcpy(cur, levels, sizeof(float) * n);
    int cy = yd, cx = xd, cz = zd;
    for (int l = t->l_max - 1; l >= t->l_min; --l) {
        int ny = (int)ceil(cy / 2.0), nx = (int)ceil(cx / 2.0), nz = (int)ceil(cz / 2.0);
        float *nxt = (float *)malloc(sizeof(float) * (size_t)ny * nx * nz);
        downsample2(cur, cy, cx, cz, nxt, DS_MAX);
        pct_fill(t, l, nxt);
        free(cur);
        cur = nxt;
        cy = ny; cx = nx; cz = nz;
    }
    free(cur);
}

/* set_ascendant_neighbours (:250-289), set_filler (:291-343),
 * fill_neighbours (:345-381), fill_parent (:383-393) */
static void ps_set_ascendant_neighbours(pct_t *t, int l) {
    int yn = t->y_num[l], xn = t->x_num[l], zn = t->z_num[l];
    uint8_t *m = t->m[l];
    for (int z = 0; z < zn; ++z)
        for (int x = 0; x < xn; ++x)
            for (int y = 0; y < yn; ++y) {
                if (m[IDX(y, x, z, yn, xn)] != PS_ASCENDANT) continue;
                for (int dz = (z == 0 ? 0 : -1); dz < (z == zn - 1 ? 1 : 2); ++dz)
                    for (int dx = (x == 0 ? 0 : -1); dx < (x == xn - 1 ? 1 : 2); ++dx)
                        for (int dy = (y == 0 ? 0 : -1); dy < (y == yn - 1 ? 1 : 2); ++dy) {
                            uint8_t *q = &m[IDX(y + dy, x + dx, z + dz, yn, xn)];
                            if (*q == PS_EMPTY) *q = PS_ASCENDANTNEIGHBOUR;
                            if (*q == PS_SEED) *q = PS_PROPOGATE;
                        }
            }
}

static void ps_set_filler(pct_t *t, int l) {
    int yn = t->y_num[l], xn = t->x_num[l], zn = t->z_num[l];
    int cy = t->y_num[l + 1], cx = t->x_num[l + 1], cz = t->z_num[l + 1];
    for (int z = 0; z < zn; ++z)
        for (int x = 0; x < xn; ++x)
            for (int y = 0; y < yn; ++y) {
                uint8_t s = t->m[l][IDX(y, x, z, yn, xn)];
                if (s != PS_ASCENDANTNEIGHBOUR && s != PS_PROPOGATE) continue;
                for (int jz = 2 * z; jz < 2 * z + 2 && jz < cz; ++jz)
                    for (int jx = 2 * x; jx < 2 * x + 2 && jx < cx; ++jx)
                        for (int jy = 2 * y; jy < 2 * y + 2 && jy < cy; ++jy) {
                            uint8_t *q = &t->m[l + 1][IDX(jy, jx, jz, cy, cx)];
                            if (*q == PS_EMPTY) *q = PS_FILLER;
                        }
            }
}

static void ps_fill_parent(pct_t *t, int z, int x, int y, int xn, int yn, int nl) {
    if (nl < t->l_min) return;
    size_t nx = (size_t)(xn + 1) / 2, ny = (size_t)(yn + 1) / 2;
    size_t i = (size_t)(z / 2) * nx * ny + (size_t)(x / 2) * ny + (size_t)(y / 2);
    if (t->m[nl][i] != PS_SEED) t->m[nl][i] = PS_ASCENDANT;
}

static void ps_fill_neighbours(pct_t *t, int l) {
    int yn = t->y_num[l], xn = t->x_num[l], zn = t->z_num[l];
    uint8_t *m = t->m[l];
    for (int z = 0; z < zn; ++z)
        for (int x = 0; x < xn; ++x)
            for (int y = 0; y < yn; ++y) {
                uint8_t s = m[IDX(y, x, z, yn, xn)];
                if (s == PS_SEED || s == PS_PROPOGATE) {
                    for (int dz = (z == 0 ? 0 : -1); dz < (z == zn - 1 ? 1 : 2); ++dz)
                        for (int dx = (x == 0 ? 0 : -1); dx < (x == xn - 1 ? 1 : 2); ++dx)
                            for (int dy = (y == 0 ? 0 : -1); dy < (y == yn - 1 ? 1 : 2); ++dy) {
                                uint8_t *q = &m[IDX(y + dy, x + dx, z + dz, yn, xn)];
                                if (*q == PS_EMPTY) *q = PS_BOUNDARY;
                            }
                    ps_fill_parent(t, z, x, y, xn, yn, l - 1);
                } else if (s == PS_ASCENDANT) {
                    ps_fill_parent(t, z, x, y, xn, yn, l - 1);
                }
            }
}

/* pulling_scheme_main (:111-132) */
static void pulling_scheme(pct_t *t) {
    for (int l = t->l_max; l >= t->l_min; --l) {
        if (l != t->l_max) {
            ps_set_ascendant_neighbours(t, l);
            ps_set_filler(t, l);
        }
        ps_fill_neighbours(t, l);
    }
}

/* LinearAccess::initialize_linear_structure (src/data_structures/APR/access/LinearAccess.hpp:210-524) */
static int linear_structure(orc_access *a, pct_t *t, int neighborhood_optimization) {
    const uint8_t min_type = neighborhood_optimization ? 1 : 2;
    const uint8_t US = 4;
    if (init_xz_linear(a) != ORC_OK) return ORC_ERR_ALLOC;
    int L = a->l_max;
    if (L <= 2) {
        uint64_t counter = 0, ls = a->level_xz[L];
        for (int z = 0; z < a->z_num[L]; ++z)
            for (int x = 0; x < a->x_num[L]; ++x) {
                counter += (uint64_t)a->y_num[L];
                a->xz_end[ls + (uint64_t)z * a->x_num[L] + x] = counter;
            }
        a->P = counter;
        a->y_vec = (uint16_t *)malloc(sizeof(uint16_t) * (counter ? counter : 1));
        counter = 0;
        for (int z = 0; z < a->z_num[L]; ++z)
            for (int x = 0; x < a->x_num[L]; ++x)
                for (int y = 0; y < a->y_num[L]; ++y) a->y_vec[counter++] = (uint16_t)y;
        return ORC_OK;
    }
    /* first step: equivalence optimisation, levels ascending */
    for (int l = a->l_min + 1; l < L; ++l) {
        int yl = a->y_num[l], xl = a->x_num[l], zl = a->z_num[l];
        int yu = a->y_num[l - 1], xu = a->x_num[l - 1];
        for (int z = 0; z < zl; ++z)
            for (int x = 0; x < xl; ++x)
                for (int y = 0; y < yu; ++y) {
                    uint8_t s = t->m[l - 1][IDX(y, x / 2, z / 2, yu, xu)];
                    if (s > 0 && s <= min_type) {
                        int y2p = 2 * y + 1 < yl - 1 ? 2 * y + 1 : yl - 1;
                        t->m[l][IDX(2 * y, x, z, yl, xl)] = US;
                        t->m[l][IDX(y2p, x, z, yl, xl)] = US;
                    }
                }
    }
    /* second step: row counts */
    for (int l = a->l_min; l < L - 1; ++l) {
        int yl = a->y_num[l], xl = a->x_num[l], zl = a->z_num[l];
        for (int z = 0; z < zl; ++z)
            for (int x = 0; x < xl; ++x) {
                uint64_t c = 0;
                for (int y = 0; y < yl; ++y) {
                    uint8_t s = t->m[l][IDX(y, x, z, yl, xl)];
                    if (s > min_type && s <= US) c++;
                }
                a->xz_end[a->level_xz[l] + (uint64_t)z * xl + x] = c;
            }
    }
    int lm1 = L - 1;
    int yl = a->y_num[lm1], xl = a->x_num[lm1], zl = a->z_num[lm1];
    int ylm = a->y_num[L], xlm = a->x_num[L], zlm = a->z_num[L];
    uint64_t *tmax = (uint64_t *)calloc((size_t)zl * xl, sizeof(uint64_t));
    for (int z = 0; z < zl; ++z)
        for (int x = 0; x < xl; ++x) {
            uint64_t c = 0, cl = 0;
            for (int y = 0; y < yl; ++y) {
                uint8_t s = t->m[lm1][IDX(y, x, z, yl, xl)];
                if (s > min_type && s <= US) c++;
                else if (s > 0 && s <= min_type) {
                    cl++;
                    if (2 * y < ylm - 1) cl++;
                }
            }
            a->xz_end[a->level_xz[lm1] + (uint64_t)z * xl + x] = c;
            tmax[(size_t)z * xl + x] = cl;
        }
    for (int z = 0; z < zlm; ++z)
        for (int x = 0; x < xlm; ++x)
            a->xz_end[a->level_xz[L] + (uint64_t)z * xlm + x] = tmax[(size_t)(z / 2) * xl + x / 2];
    free(tmax);
    for (uint64_t i = 1; i < a->n_xz; ++i) a->xz_end[i] += a->xz_end[i - 1];
    a->P = a->xz_end[a->n_xz - 1];
    a->y_vec = (uint16_t *)calloc(a->P ? a->P : 1, sizeof(uint16_t));
    if (!a->y_vec) return ORC_ERR_ALLOC;
    for (int l = a->l_min; l < L - 1; ++l) {
        int yy = a->y_num[l], xx = a->x_num[l], zz = a->z_num[l];
        for (int z = 0; z < zz; ++z)
            for (int x = 0; x < xx; ++x) {
                uint64_t o = row_begin(a, l, z, x), c = 0;
                for (int y = 0; y < yy; ++y) {
                    uint8_t s = t->m[l][IDX(y, x, z, yy, xx)];
                    if (s > min_type && s <= US) a->y_vec[o + c++] = (uint16_t)y;
                }
            }
    }
    for (int z = 0; z < zl; ++z)
        for (int x = 0; x < xl; ++x) {
            uint64_t o = row_begin(a, lm1, z, x), om = row_begin(a, L, 2 * z, 2 * x), c = 0, cl = 0;
            for (int y = 0; y < yl; ++y) {
                uint8_t s = t->m[lm1][IDX(y, x, z, yl, xl)];
                if (s > min_type && s <= US) a->y_vec[o + c++] = (uint16_t)y;
                else if (s > 0 && s <= min_type) {
                    a->y_vec[om + cl++] = (uint16_t)(2 * y);
                    if (2 * y < ylm - 1) a->y_vec[om + cl++] = (uint16_t)(2 * y + 1);
                }
            }
        }
    for (int z = 0; z < zlm; ++z)
        for (int x = 0; x < xlm; ++x) {
            if ((z % 2) == 0 && (x % 2) == 0) continue;
            uint64_t bf = row_begin(a, L, (z / 2) * 2, (x / 2) * 2), ef = row_end(a, L, (z / 2) * 2, (x / 2) * 2);
            uint64_t b = row_begin(a, L, z, x);
            memcpy(a->y_vec + b, a->y_vec + bf, sizeof(uint16_t) * (ef - bf));
        }
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* get_apr pipeline (src/algorithm/APRConverter.hpp:195-363, 535-582)        */
/* ------------------------------------------------------------------------ */
struct orc_apr {
    orc_access acc;
    float offset;
    int yd, xd, zd, yn, xn, zn;
    float *inter[7];
};

void orc_free(orc_apr *a) {
    if (!a) return;
    orc_access_free(&a->acc);
    for (int i = 0; i < 7; ++i) free(a->inter[i]);
    free(a);
}

const orc_access *orc_get_access(const orc_apr *a) { return &a->acc; }
float orc_bspline_offset(const orc_apr *a) { return a->offset; }

int orc_copy_intermediate(const orc_apr *a, int which, float *dst, size_t n) {
    if (which < 0 || which > 6 || !a->inter[which]) return ORC_ERR_ARG;
    size_t need = which == 0 ? (size_t)a->yn * a->xn * a->zn : (size_t)a->yd * a->xd * a->zd;
    if (n != need) return ORC_ERR_ARG;
    memcpy(dst, a->inter[which], sizeof(float) * n);
    return ORC_OK;
}

static float *dup_f(const float *s, size_t n) {
    float *d = (float *)malloc(sizeof(float) * n);
    memcpy(d, s, sizeof(float) * n);
    return d;
}

/* applyParameters (src/algorithm/APRConverter.hpp:250-297) and computeLevels
 * (src/algorithm/LocalParticleCellSet.hpp:129-171): grad and lis (ds) are
 * thresholded in place and lis receives the level image.  ids may be NULL
 * (custom gradient entry point: no intensity threshold). */
static void apply_and_levels(orc_apr *keep_r, float *grad, float *lis, const float *ids, size_t nd, float offset,
                             const orc_params *p, int apr_l_max) {
    float th = p->Ip_th + offset;
    if (ids)
        for (size_t i = 0; i < nd; ++i)
            if (ids[i] <= th) grad[i] = 0;
    for (size_t i = 0; i < nd; ++i) {
        float v = lis[i];
        if (v < p->sigma_th) lis[i] = (v < p->sigma_th_max) ? 60000.0f : p->sigma_th;
    }
    for (size_t i = 0; i < nd; ++i)
        if (grad[i] < p->grad_th) grad[i] = 0;
    if (keep_r) { keep_r->inter[4] = dup_f(grad, nd); keep_r->inter[5] = dup_f(lis, nd); }
    float mxz = p->dz < p->dx ? p->dz : p->dx;          /* std::min(dx, dz) */
    float min_dim = mxz < p->dy ? mxz : p->dy;            /* std::min(dy, .) */
    float level_factor = (float)(pow(2.0, (double)apr_l_max) * (double)min_dim);
    float mult = level_factor / p->rel_error;
    for (size_t i = 0; i < nd; ++i) {
        float q = grad[i] / lis[i];
        uint32_t u = cvt_u32(q * mult);
        lis[i] = (float)(u == 0 ? 0u : (uint32_t)(31 - __builtin_clz(u)));
    }
    if (keep_r) keep_r->inter[6] = dup_f(lis, nd);
}

/* solveForAPR (APRConverter.hpp:301-336) after the levels, and
 * generateDatastructures (:339-363) */
static int finish_apr(orc_apr *r, float *grad, float *lis, const float *ids, const orc_params *p, int keep) {
    size_t nd = (size_t)r->yd * r->xd * r->zd;
    apply_and_levels(keep ? r : NULL, grad, lis, ids, nd, r->offset, p, r->acc.l_max);
    pct_t t;
    pct_init(&t, &r->acc);
    if (t.l_max >= t.l_min) {
        local_particle_cell_set(&t, lis, r->yd, r->xd, r->zd);
        pulling_scheme(&t);
    }
    int e = linear_structure(&r->acc, &t, p->neighborhood_optimization);
    pct_free(&t);
    return e;
}

/* The pixel stages of one image (the whole volume, or one z-tile of the
 * blocked converter, APRConverterBatch.hpp:190-271): offset, smoothing,
 * gradient + ds image, inverse B-spline, local intensity scale.  Returns
 * ORC_ERR_OVERFLOW on a uint16 smoothing overflow.  On success *grad, *ids and
 * *lis hold ds images the caller frees; keep_r (optional) receives the
 * smoothed image and the stage intermediates. */
static int pixel_stages(const uint16_t *img, int yn, int xn, int zn, const orc_params *p, int is_u16,
                        float *offset, float **grad_out, float **ids_out, float **lis_out, orc_apr *keep_r) {
    int yd = (int)ceil(yn / 2.0), xd = (int)ceil(xn / 2.0), zd = (int)ceil(zn / 2.0);
    size_t n = (size_t)yn * xn * zn, nd = (size_t)yd * xd * zd;
    float *im = (float *)malloc(sizeof(float) * n);
    /* offset (:216-223) and compute_bspline_offset (src/algorithm/AutoParameters.hpp:186-197) */
    *offset = 0;
    if (is_u16) {
        if (p->lambda > 0) {
            uint16_t mn = 65535, mx = 0;
            for (size_t i = 0; i < n; ++i) { if (img[i] > mx) mx = img[i]; if (img[i] < mn) mn = img[i]; }
            float off = (float)((65535 - (mx - mn)) / 2 - mn);
            off = off < 100.f ? off : 100.f;
            *offset = off > -100.f ? off : -100.f;
        }
        for (size_t i = 0; i < n; ++i) im[i] = cvt_u16((float)img[i] + *offset);
    } else {
        for (size_t i = 0; i < n; ++i) im[i] = (float)img[i];
    }
    /* get_gradient (src/algorithm/ComputeGradient.hpp:71-119) */
    if (p->lambda > 0) {
        uint64_t err = 0;
        if (yn > 2) err += orc_bspline_axis(im, yn, xn, zn, 0, p->lambda, is_u16);
        if (xn > 2) err += orc_bspline_axis(im, yn, xn, zn, 1, p->lambda, is_u16);
        if (zn > 2) err += orc_bspline_axis(im, yn, xn, zn, 2, p->lambda, is_u16);
        if (err) { free(im); return ORC_ERR_OVERFLOW; }
    }
    if (keep_r) keep_r->inter[0] = dup_f(im, n);
    float *grad = (float *)malloc(sizeof(float) * nd);
    gradient_ds(im, yn, xn, zn, grad, yd, xd, zd, p->dx, p->dy, p->dz, is_u16);
    float *ids = (float *)malloc(sizeof(float) * nd);
    downsample2(im, yn, xn, zn, ids, DS_MEAN_D8);
    free(im);
    if (p->lambda > 0) {
        if (yn > 2) inv_bspline_y(ids, yd, xd, zd);
        if (xn > 2)
            for (int z = 0; z < zd; ++z)
                for (int y = 0; y < yd; ++y) inv_bspline_strided(ids + IDX(y, 0, z, yd, xd), (size_t)yd, xd);
        if (zn > 2)
            for (int x = 0; x < xd; ++x)
                for (int y = 0; y < yd; ++y)
                    inv_bspline_strided(ids + IDX(y, x, 0, yd, xd), (size_t)yd * xd, zd);
    }
    if (keep_r) { keep_r->inter[1] = dup_f(grad, nd); keep_r->inter[2] = dup_f(ids, nd); }
    float *lis = (float *)malloc(sizeof(float) * nd);
    local_intensity_scale(ids, yd, xd, zd, p, lis);
    if (keep_r) keep_r->inter[3] = dup_f(lis, nd);
    *grad_out = grad; *ids_out = ids; *lis_out = lis;
    return ORC_OK;
}

int orc_get_apr(const uint16_t *img, int yn, int xn, int zn, const orc_params *p, int image_type, orc_apr **out) {
    *out = NULL;
    if (yn < 1 || xn < 1 || zn < 1) return ORC_ERR_DIMS;
    int nd3 = (yn > 1) + (xn > 1) + (zn > 1);
    if (nd3 == 0) return ORC_ERR_DIMS;
    orc_apr *r = (orc_apr *)calloc(1, sizeof(orc_apr));
    geninfo_init(&r->acc, yn, xn, zn);
    r->yn = yn; r->xn = xn; r->zn = zn;
    r->yd = (int)ceil(yn / 2.0); r->xd = (int)ceil(xn / 2.0); r->zd = (int)ceil(zn / 2.0);
    float *grad, *ids, *lis;
    int e = pixel_stages(img, yn, xn, zn, p, image_type == 1, &r->offset, &grad, &ids, &lis, r);
    if (e != ORC_OK) { orc_free(r); return e; }
    e = finish_apr(r, grad, lis, ids, p, 1);
    free(grad); free(lis); free(ids);
    if (e != ORC_OK) { orc_free(r); return e; }
    *out = r;
    return ORC_OK;
}

/* PullingScheme::fill_patch (src/algorithm/PullingScheme.hpp:175-247) for a
 * z-tile (no x/y ghost): level image lv of the tile at pct level k, tile dims
 * (py, px, pz) at that level; the ghost is cropped by integer division. */
static int pct_fill_patch(pct_t *t, int k, const float *lv, int py, int px, int pz, int ghost_l, int ghost_r,
                          int z0) {
    int lf = (int)powr(2, t->l_max + 1 - k);
    int zgl = ghost_l / lf, zgr = ghost_r / lf;
    int offz = z0 / lf - zgl;  /* (z_offset + z_ghost_l) / lf - z_ghost_l / lf */
    float kf = (float)k;
    for (int z = zgl; z < pz - zgr; ++z) {
        /* planes past the level: the reference writes beyond its array there */
        if (z + offz < 0 || z + offz >= t->z_num[k]) continue;
        for (int x = 0; x < px; ++x)
            for (int y = 0; y < py; ++y) {
                float v = lv[IDX(y, x, z, py, px)];
                int sd;
                if (k == t->l_max) sd = v >= kf;
                else if (k == t->l_min) sd = v <= kf;
                else sd = v == kf;
                if (sd) t->m[k][IDX(y, x, z + offz, t->y_num[k], t->x_num[k])] = PS_SEED;
            }
    }
    return ORC_OK;
}

/* z-tiling of APRConverterBatch::get_apr_batch_method_from_file
 * (src/algorithm/APRConverterBatch.hpp:125-160) */
static void z_block(int b, int nb, int zn, int zblock, int ghost, int *z0, int *zf, int *gl, int *gr) {
    *z0 = b * zblock;
    *zf = (b == nb - 1) ? zn : (b + 1) * zblock;
    *gl = *z0 < ghost ? *z0 : ghost;
    *gr = (zn - *zf) < ghost ? (zn - *zf) : ghost;
}

/* get_apr_method_patch (APRConverterBatch.hpp:190-271) for tiles [first, first +
 * count) of the blocked tiling, each filling the global particle-cell tree t
 * (fill_global_particle_cell_tree :282-314); slab holds planes [slab_z0, ...)
 * of the volume.  *offset receives the last tile's bspline offset. */
static int fill_tiles(pct_t *t, const uint16_t *slab, int slab_z0, int yn, int xn, int zn, const orc_params *p,
                      int image_type, int zblock, int ghost, int first, int count, int l_max, float *offset) {
    int nb = zn / zblock > 1 ? zn / zblock : 1;
    int e = ORC_OK;
    for (int b = first; b < first + count && b < nb && e == ORC_OK; ++b) {
        int z0, zf, gl, gr;
        z_block(b, nb, zn, zblock, ghost, &z0, &zf, &gl, &gr);
        int pz = zf + gr - (z0 - gl);
        float *grad, *ids, *lis;
        e = pixel_stages(slab + (size_t)(z0 - gl - slab_z0) * xn * yn, yn, xn, pz, p, image_type == 1, offset, &grad,
                         &ids, &lis, NULL);
        if (e != ORC_OK) break;
        int cy = (int)ceil(yn / 2.0), cx = (int)ceil(xn / 2.0), cz = (int)ceil(pz / 2.0);
        apply_and_levels(NULL, grad, lis, ids, (size_t)cy * cx * cz, *offset, p, l_max);
        free(grad); free(ids);
        float *cur = lis;
        if (t->l_max >= t->l_min) {
            e = pct_fill_patch(t, t->l_max, cur, cy, cx, cz, gl, gr, z0);
            for (int l = t->l_max - 1; l >= t->l_min && e == ORC_OK; --l) {
                int ny = (int)ceil(cy / 2.0), nx = (int)ceil(cx / 2.0), nz = (int)ceil(cz / 2.0);
                float *nxt = (float *)malloc(sizeof(float) * (size_t)ny * nx * nz);
                downsample2(cur, cy, cx, cz, nxt, DS_MAX);
                free(cur);
                cur = nxt;
                cy = ny; cx = nx; cz = nz;
                e = pct_fill_patch(t, l, cur, cy, cx, cz, gl, gr, z0);
            }
        }
        free(cur);
    }
    return e;
}

/* APRConverterBatch<IT>: get_apr_method_patch per z-tile
 * (APRConverterBatch.hpp:190-271), fill_global_particle_cell_tree (:282-314),
 * then one pulling scheme and linear structure for the whole volume. */
int orc_get_apr_by_block(const uint16_t *img, int yn, int xn, int zn, const orc_params *p, int image_type,
                         int zblock, int ghost, orc_apr **out) {
    *out = NULL;
    if (yn < 1 || xn < 1 || zn < 1 || zblock < 1 || ghost < 0) return ORC_ERR_ARG;
    orc_apr *r = (orc_apr *)calloc(1, sizeof(orc_apr));
    geninfo_init(&r->acc, yn, xn, zn);
    r->yn = yn; r->xn = xn; r->zn = zn;
    r->yd = (int)ceil(yn / 2.0); r->xd = (int)ceil(xn / 2.0); r->zd = (int)ceil(zn / 2.0);
    pct_t t;
    pct_init(&t, &r->acc);
    int nb = zn / zblock > 1 ? zn / zblock : 1;
    int e = fill_tiles(&t, img, 0, yn, xn, zn, p, image_type, zblock, ghost, 0, nb, r->acc.l_max, &r->offset);
    if (e == ORC_OK) {
        if (t.l_max >= t.l_min) pulling_scheme(&t);
        e = linear_structure(&r->acc, &t, p->neighborhood_optimization);
    }
    pct_free(&t);
    if (e != ORC_OK) { orc_free(r); return e; }
    *out = r;
    return ORC_OK;
}

/* The particle-cell tree in one caller buffer: levels l_min .. l_max - 1 of the
 * tree, each y_num x x_num x z_num bytes, concatenated (the arrays of
 * PullingScheme::particle_cell_tree, PullingScheme.hpp:92-104). */
static size_t pct_view(pct_t *t, const orc_access *g, uint8_t *buf) {
    memset(t, 0, sizeof(*t));
    t->l_max = g->l_max - 1;
    t->l_min = g->l_min;
    size_t tot = 0;
    for (int l = t->l_min; l <= t->l_max; ++l) {
        double cell = powr(2, t->l_max - l + 1);
        t->y_num[l] = (int)ceil(g->org[0] / cell);
        t->x_num[l] = (int)ceil(g->org[1] / cell);
        t->z_num[l] = (int)ceil(g->org[2] / cell);
        if (buf) t->m[l] = buf + tot;
        tot += (size_t)t->y_num[l] * t->x_num[l] * t->z_num[l];
    }
    return tot;
}

size_t orc_pyramid_bytes(int yn, int xn, int zn) {
    orc_access g;
    memset(&g, 0, sizeof(g));
    geninfo_init(&g, yn, xn, zn);
    pct_t t;
    size_t n = pct_view(&t, &g, NULL);
    free(g.xz_end);
    return n;
}

int orc_pyramid_fill_tiles(const uint16_t *slab, int slab_z0, int yn, int xn, int zn, const orc_params *p,
                           int image_type, int zblock, int ghost, int first, int count, uint8_t *pyramid) {
    if (yn < 1 || xn < 1 || zn < 1 || zblock < 1 || ghost < 0 || first < 0 || count < 0) return ORC_ERR_ARG;
    orc_access g;
    memset(&g, 0, sizeof(g));
    geninfo_init(&g, yn, xn, zn);
    pct_t t;
    pct_view(&t, &g, pyramid);
    float offset = 0;
    int e = fill_tiles(&t, slab, slab_z0, yn, xn, zn, p, image_type, zblock, ghost, first, count, g.l_max, &offset);
    free(g.xz_end);
    return e;
}

int orc_apr_from_pyramid(uint8_t *pyramid, int yn, int xn, int zn, const orc_params *p, orc_apr **out) {
    *out = NULL;
    orc_apr *r = (orc_apr *)calloc(1, sizeof(orc_apr));
    geninfo_init(&r->acc, yn, xn, zn);
    r->yn = yn; r->xn = xn; r->zn = zn;
    r->yd = (int)ceil(yn / 2.0); r->xd = (int)ceil(xn / 2.0); r->zd = (int)ceil(zn / 2.0);
    pct_t t;
    pct_view(&t, &r->acc, pyramid);
    if (t.l_max >= t.l_min) pulling_scheme(&t);
    int e = linear_structure(&r->acc, &t, p->neighborhood_optimization);
    if (e != ORC_OK) { orc_free(r); return e; }
    *out = r;
    return ORC_OK;
}

int orc_get_apr_custom(const float *grad_ds, const float *lis_ds, int yn, int xn, int zn, const orc_params *p, orc_apr **out) {
    *out = NULL;
    if (yn < 1 || xn < 1 || zn < 1) return ORC_ERR_DIMS;
    orc_apr *r = (orc_apr *)calloc(1, sizeof(orc_apr));
    geninfo_init(&r->acc, yn, xn, zn);
    r->yn = yn; r->xn = xn; r->zn = zn;
    r->yd = (int)ceil(yn / 2.0); r->xd = (int)ceil(xn / 2.0); r->zd = (int)ceil(zn / 2.0);
    size_t nd = (size_t)r->yd * r->xd * r->zd;
    r->offset = 0;
    float *grad = dup_f(grad_ds, nd), *lis = dup_f(lis_ds, nd);
    /* The threshold step reads local_scale_temp2, which in this entry point
     * holds padded LIS work memory of an earlier call; the reference tests
     * use Ip_th = 0 with a positive image, so the step is skipped here. */
    int e = finish_apr(r, grad, lis, NULL, p, 1);
    free(grad); free(lis);
    if (e != ORC_OK) { orc_free(r); return e; }
    *out = r;
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* a12: sample_image (src/data_structures/APR/particles/ParticleData.hpp:222-261) */
/* ------------------------------------------------------------------------ */
int orc_sample_image(const orc_access *a, const uint16_t *img, uint16_t *parts) {
    int L = a->l_max;
    float *lev[ORC_MAX_LEVELS] = {0};
    size_t n = (size_t)a->y_num[L] * a->x_num[L] * a->z_num[L];
    lev[L] = (float *)malloc(sizeof(float) * n);
    for (size_t i = 0; i < n; ++i) lev[L][i] = (float)img[i];
    for (int l = L; l > a->l_min; --l) {
        lev[l - 1] = (float *)malloc(sizeof(float) * (size_t)a->y_num[l - 1] * a->x_num[l - 1] * a->z_num[l - 1]);
        downsample2(lev[l], a->y_num[l], a->x_num[l], a->z_num[l], lev[l - 1], DS_MEAN_U16);
    }
    for (int l = a->l_min; l <= L; ++l)
        for (int z = 0; z < a->z_num[l]; ++z)
            for (int x = 0; x < a->x_num[l]; ++x)
                for (uint64_t i = row_begin(a, l, z, x); i < row_end(a, l, z, x); ++i)
                    parts[i] = (uint16_t)lev[l][IDX(a->y_vec[i], x, z, a->y_num[l], a->x_num[l])];
    for (int l = 0; l < ORC_MAX_LEVELS; ++l) free(lev[l]);
    return ORC_OK;
}

/* sample_parts_from_img_downsampled_patch
 * (src/data_structures/APR/particles/ParticleData.hpp:330-372) over the
 * z-tiles of sample_parts_from_img_blocked_gen (:288-322): every tile builds
 * its own uint16 mean pyramid and writes the particles of its rows; a later
 * tile overwrites an earlier one where their cropped rows overlap. */
int orc_sample_image_by_block(const orc_access *a, const uint16_t *img, int zblock, int ghost, uint16_t *parts) {
    int L = a->l_max, yn = a->org[0], xn = a->org[1], zn = a->org[2];
    if (zblock < 1 || ghost < 0) return ORC_ERR_ARG;
    int nb = zn / zblock > 1 ? zn / zblock : 1;
    for (int b = 0; b < nb; ++b) {
        int z0, zf, gl, gr;
        z_block(b, nb, zn, zblock, ghost, &z0, &zf, &gl, &gr);
        int pz = zf + gr - (z0 - gl);
        float *lev[ORC_MAX_LEVELS] = {0};
        int ly[ORC_MAX_LEVELS], lx[ORC_MAX_LEVELS], lz[ORC_MAX_LEVELS];
        size_t n = (size_t)yn * xn * pz;
        lev[L] = (float *)malloc(sizeof(float) * n);
        const uint16_t *src = img + (size_t)(z0 - gl) * xn * yn;
        for (size_t i = 0; i < n; ++i) lev[L][i] = (float)src[i];
        ly[L] = yn; lx[L] = xn; lz[L] = pz;
        for (int l = L; l > a->l_min; --l) {
            ly[l - 1] = (int)ceil(ly[l] / 2.0); lx[l - 1] = (int)ceil(lx[l] / 2.0); lz[l - 1] = (int)ceil(lz[l] / 2.0);
            lev[l - 1] = (float *)malloc(sizeof(float) * (size_t)ly[l - 1] * lx[l - 1] * lz[l - 1]);
            downsample2(lev[l], ly[l], lx[l], lz[l], lev[l - 1], DS_MEAN_U16);
        }
        int err = 0;
        for (int l = a->l_min; l <= L && !err; ++l) {
            int lf = (int)powr(2, L - l);
            int zgl = gl / lf, zgr = gr / lf, offz = z0 / lf - zgl;
            for (int z = zgl; z < lz[l] - zgr && !err; ++z) {
                /* rows past the level: the reference reads beyond its row index there */
                if (z + offz < 0 || z + offz >= a->z_num[l]) continue;
                for (int x = 0; x < lx[l]; ++x)
                    for (uint64_t i = row_begin(a, l, z + offz, x); i < row_end(a, l, z + offz, x); ++i)
                        parts[i] = (uint16_t)lev[l][IDX(a->y_vec[i], x, z, ly[l], lx[l])];
            }
        }
        for (int l = 0; l < ORC_MAX_LEVELS; ++l) free(lev[l]);
        if (err) return ORC_ERR_ARG;
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* a14: APR::initialize_tree_dense (src/data_structures/APR/APR.hpp:633-689)  */
/* + LinearAccess::initialize_tree_access_dense (LinearAccess.hpp:67-122)    */
/* ------------------------------------------------------------------------ */
int orc_tree_init(const orc_access *a, orc_access *t) {
    geninfo_init_tree(t, a->org[0], a->org[1], a->org[2]);
    uint8_t *pm[ORC_MAX_LEVELS] = {0};
    for (int l = t->l_min; l <= t->l_max; ++l)
        pm[l] = (uint8_t *)calloc((size_t)t->y_num[l] * t->x_num[l] * t->z_num[l], 1);
    for (int l = a->l_max; l >= a->l_min; --l)
        for (int z = 0; z < a->z_num[l]; ++z)
            for (int x = 0; x < a->x_num[l]; ++x)
                for (uint64_t i = row_begin(a, l, z, x); i < row_end(a, l, z, x); ++i)
                    pm[l - 1][IDX(a->y_vec[i] / 2, x / 2, z / 2, t->y_num[l - 1], t->x_num[l - 1])] = 1;
    for (int l = t->l_max - 1; l >= t->l_min; --l)
        for (int z = 0; z < t->z_num[l]; ++z)
            for (int x = 0; x < t->x_num[l]; ++x)
                for (int y = 0; y < t->y_num[l]; ++y)
                    pm[l][IDX(y, x, z, t->y_num[l], t->x_num[l])] |=
                        pm[l + 1][IDX(2 * y, 2 * x, 2 * z, t->y_num[l + 1], t->x_num[l + 1])];
    if (init_xz_linear(t) != ORC_OK) return ORC_ERR_ALLOC;
    for (int l = t->l_max; l >= t->l_min; --l)
        for (int z = 0; z < t->z_num[l]; ++z)
            for (int x = 0; x < t->x_num[l]; ++x) {
                uint64_t c = 0;
                for (int y = 0; y < t->y_num[l]; ++y) c += pm[l][IDX(y, x, z, t->y_num[l], t->x_num[l])];
                t->xz_end[t->level_xz[l] + (uint64_t)z * t->x_num[l] + x] = c;
            }
    for (uint64_t i = 1; i < t->n_xz; ++i) t->xz_end[i] += t->xz_end[i - 1];
    t->P = t->xz_end[t->n_xz - 1];
    t->y_vec = (uint16_t *)calloc(t->P ? t->P : 1, sizeof(uint16_t));
    for (int l = t->l_max; l >= t->l_min; --l)
        for (int z = 0; z < t->z_num[l]; ++z)
            for (int x = 0; x < t->x_num[l]; ++x) {
                uint64_t o = row_begin(t, l, z, x);
                for (int y = 0; y < t->y_num[l]; ++y)
                    if (pm[l][IDX(y, x, z, t->y_num[l], t->x_num[l])]) t->y_vec[o++] = (uint16_t)y;
            }
    for (int l = 0; l < ORC_MAX_LEVELS; ++l) free(pm[l]);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* a15: fill_tree_mean (src/numerics/APRTreeNumerics.hpp:63-203)             */
/* Generic over the value type so the FP64 RL oracle can reuse it.           */
/* ------------------------------------------------------------------------ */
#define DEFINE_TREE_MEAN(NAME, VT)                                                                         \
static void NAME(const orc_access *a, const orc_access *t, const VT *parts, VT *tree) {                    \
    memset(tree, 0, sizeof(VT) * (t->P ? t->P : 1));                                                       \
    for (int pass = 0; pass < 2; ++pass) {                                                                 \
        const orc_access *c = pass == 0 ? a : t;                                                           \
        const VT *cv = pass == 0 ? parts : tree;                                                           \
        int lhi = pass == 0 ? a->l_max : t->l_max;                                                         \
        int llo = pass == 0 ? a->l_min : t->l_min + 1;                                                     \
        for (int l = lhi; l >= llo; --l) {                                                                 \
            int pl = l - 1;                                                                                \
            for (int zd = 0; zd < t->z_num[pl]; ++zd)                                                      \
                for (int z = 2 * zd; z <= (2 * zd + 1 < c->z_num[l] - 1 ? 2 * zd + 1 : c->z_num[l] - 1); ++z) \
                    for (int xd = 0; xd < t->x_num[pl]; ++xd)                                              \
                        for (int x = 2 * xd; x <= (2 * xd + 1 < c->x_num[l] - 1 ? 2 * xd + 1 : c->x_num[l] - 1); ++x) { \
                            uint64_t pb = row_begin(t, pl, z / 2, x / 2), pe = row_end(t, pl, z / 2, x / 2); \
                            float sxz = (float)((((2 * t->x_num[pl] != c->x_num[l]) && ((x / 2) == (t->x_num[pl] - 1))) + \
                                                 ((2 * t->z_num[pl] != c->z_num[l]) && ((z / 2) == (t->z_num[pl] - 1)))) * 2); \
                            if (sxz == 0) sxz = 1;                                                         \
                            float syxz = sxz;                                                              \
                            if (2 * t->y_num[pl] != c->y_num[l]) syxz = sxz * 2;                           \
                            uint64_t pi = pb;                                                              \
                            for (uint64_t i = row_begin(c, l, z, x); i < row_end(c, l, z, x); ++i) {       \
                                while (pi < pe && t->y_vec[pi] != c->y_vec[i] / 2) pi++;                   \
                                VT v = cv[i];                                                              \
                                if (t->y_vec[pi] == t->y_num[pl] - 1) tree[pi] = syxz * v / 8.0f + tree[pi]; \
                                else tree[pi] = sxz * v / 8.0f + tree[pi];                                  \
                            }                                                                              \
                        }                                                                                  \
        }                                                                                                  \
    }                                                                                                      \
}
DEFINE_TREE_MEAN(tree_mean_f, float)
DEFINE_TREE_MEAN(tree_mean_d, double)

int orc_fill_tree_mean(const orc_access *a, const orc_access *t, const float *parts, float *tree) {
    tree_mean_f(a, t, parts, tree);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* a16: stencils (src/numerics/APRStencil.hpp:13-95; PixelData::normalize    */
/* src/data_structures/Mesh/PixelData.hpp:771-778)                           */
/* ------------------------------------------------------------------------ */
#define DEFINE_DS_STENCIL(NAME, ST)                                                                        \
static int NAME(const ST *in, int n, int level_delta, int normalize, ST *out) {                           \
    int ndim = 3;                                                                                          \
    int step = (int)powf(2.0f, (float)level_delta);                                                        \
    int factor = (int)powf((float)step, (float)ndim);                                                      \
    int nd = 2 * (((n - 1) / 2 + step - 1) / step) + 1;                                                    \
    if (nd < 3) nd = 3;                                                                                    \
    for (int i = 0; i < nd * nd * nd; ++i) out[i] = 0;                                                     \
    int off = (nd / 2) * step - n / 2;                                                                     \
    for (int iz = 0; iz < n; ++iz)                                                                         \
        for (int ix = 0; ix < n; ++ix)                                                                     \
            for (int iy = 0; iy < n; ++iy)                                                                 \
                for (int dz = 0; dz < nd; ++dz) {                                                          \
                    int zs = dz * step > off + iz ? dz * step : off + iz;                                  \
                    int ze = dz * step + step < off + iz + step ? dz * step + step : off + iz + step;      \
                    float oz = (float)(ze - zs > 0 ? ze - zs : 0);                                         \
                    for (int dx = 0; dx < nd; ++dx) {                                                      \
                        int xs = dx * step > off + ix ? dx * step : off + ix;                              \
                        int xe = dx * step + step < off + ix + step ? dx * step + step : off + ix + step;  \
                        float ox = (float)(xe - xs > 0 ? xe - xs : 0);                                     \
                        for (int dy = 0; dy < nd; ++dy) {                                                  \
                            int ys = dy * step > off + iy ? dy * step : off + iy;                          \
                            int ye = dy * step + step < off + iy + step ? dy * step + step : off + iy + step; \
                            float oy = (float)(ye - ys > 0 ? ye - ys : 0);                                 \
                            float ov = ox * oy * oz;                                                       \
                            out[(dz * nd + dx) * nd + dy] += ov * in[(iz * n + ix) * n + iy];              \
                        }                                                                                  \
                    }                                                                                      \
                }                                                                                          \
    float sum = 0;                                                                                         \
    for (int i = 0; i < nd * nd * nd; ++i) { out[i] /= factor; sum += out[i]; }                            \
    if (normalize) {                                                                                       \
        float nf = 1.0f / sum;                                                                             \
        for (int i = 0; i < nd * nd * nd; ++i) out[i] *= nf;                                               \
    }                                                                                                      \
    return nd;                                                                                             \
}
DEFINE_DS_STENCIL(ds_stencil_f, float)
DEFINE_DS_STENCIL(ds_stencil_d, double)

#define DEFINE_GET_STENCILS(NAME, ST, DSF)                                                                 \
static int NAME(const ST *in, int ks, int nlevels, int normalize, ST *out, int *sides) {                 \
    int total = 0;                                                                                         \
    int n0 = ks * ks * ks;                                                                                 \
    for (int i = 0; i < n0; ++i) out[i] = in[i];                                                           \
    if (normalize) {                                                                                       \
        float s = 0.0f;                                                                                    \
        for (int i = 0; i < n0; ++i) s = (float)(s + out[i]);                                              \
        if (fabsf(s) > 1e-6 && s != 1.0f)                                                                  \
            for (int i = 0; i < n0; ++i) out[i] = out[i] / s;                                              \
    }                                                                                                      \
    sides[0] = ks;                                                                                         \
    total = n0;                                                                                            \
    for (int d = 1; d < nlevels; ++d) {                                                                    \
        int nd = DSF(in, ks, d, normalize, out + total);                                                   \
        sides[d] = nd;                                                                                     \
        total += nd * nd * nd;                                                                             \
    }                                                                                                      \
    return total;                                                                                          \
}
DEFINE_GET_STENCILS(get_stencils_f, float, ds_stencil_f)
DEFINE_GET_STENCILS(get_stencils_d, double, ds_stencil_d)

int orc_downsampled_stencils(const float *stencil, int ks, int nlevels, int normalize, float *out, int *sides) {
    if (nlevels < 1) nlevels = 1;
    return get_stencils_f(stencil, ks, nlevels, normalize, out, sides);
}

/* ------------------------------------------------------------------------ */
/* a17: convolve_pencil (src/numerics/APRFilter.hpp:1094-1216, helpers       */
/* :287-849).  Each level's isotropic neighbourhood is built as a dense      */
/* image: same-level particles, parents up to num_parent_levels coarser      */
/* (piecewise constant in y, :766-793), and tree means at the same level    */
/* (:802-818); out-of-domain samples reflect about the edge sample or are    */
/* zero (:287-504).                                                          */
/* ------------------------------------------------------------------------ */
static inline int bc_index(int i, int n, int reflect, int *ok) {
    if (i >= 0 && i < n) return i;
    if (!reflect) { *ok = 0; return 0; }
    int r = i < 0 ? -i : 2 * (n - 1) - i;
    if (r < 0 || r >= n) { *ok = -1; return 0; }
    return r;
}

#define DEFINE_CONV(NAME, VT)                                                                              \
static uint64_t NAME(const orc_access *a, const orc_access *t, const VT *st, const int *sides, int ns,     \
                     const VT *in, const VT *tree, VT *out, int reflect) {                                  \
    uint64_t stale = 0;                                                                                    \
    int offs[ORC_MAX_LEVELS];                                                                              \
    offs[0] = 0;                                                                                           \
    for (int i = 1; i < ns; ++i) offs[i] = offs[i - 1] + sides[i - 1] * sides[i - 1] * sides[i - 1];       \
    for (int l = a->l_max; l >= a->l_min; --l) {                                                           \
        int sn = ns - 1 < a->l_max - l ? ns - 1 : a->l_max - l;                                            \
        int s = sides[sn], r = (s - 1) / 2;                                                                \
        const VT *S = st + offs[sn];                                                                       \
        int mnp = (int)ceil(log2((double)(r + 2)) - 1);                                                    \
        int npl = mnp < l - a->l_min ? mnp : l - a->l_min;                                                 \
        int yn = a->y_num[l], xn = a->x_num[l], zn = a->z_num[l];                                          \
        if (row_begin(a, l, 0, 0) == row_end(a, l, zn - 1, xn - 1)) continue;                              \
        size_t n = (size_t)yn * xn * zn;                                                                   \
        VT *D = (VT *)malloc(sizeof(VT) * n);                                                              \
        uint8_t *F = (uint8_t *)calloc(n, 1);                                                              \
        for (int z = 0; z < zn; ++z)                                                                       \
            for (int x = 0; x < xn; ++x) {                                                                 \
                for (uint64_t i = row_begin(a, l, z, x); i < row_end(a, l, z, x); ++i) {                   \
                    size_t q = IDX(a->y_vec[i], x, z, yn, xn); D[q] = in[i]; F[q] = 1;                     \
                }                                                                                          \
                for (int d = 1; d <= npl; ++d) {                                                           \
                    int step = (int)pow(2.0, (double)d);                                                   \
                    int pl = l - d;                                                                        \
                    for (uint64_t i = row_begin(a, pl, z / step, x / step); i < row_end(a, pl, z / step, x / step); ++i) { \
                        int y0 = step * a->y_vec[i];                                                       \
                        int y1 = y0 + step < yn ? y0 + step : yn;                                          \
                        for (int y = y0; y < y1; ++y) { size_t q = IDX(y, x, z, yn, xn); D[q] = in[i]; F[q] = 1; } \
                    }                                                                                      \
                }                                                                                          \
                if (l < a->l_max)                                                                          \
                    for (uint64_t i = row_begin(t, l, z, x); i < row_end(t, l, z, x); ++i) {               \
                        size_t q = IDX(t->y_vec[i], x, z, yn, xn); D[q] = tree[i]; F[q] = 1;               \
                    }                                                                                      \
            }                                                                                              \
        for (int z = 0; z < zn; ++z)                                                                       \
            for (int x = 0; x < xn; ++x)                                                                   \
                for (uint64_t i = row_begin(a, l, z, x); i < row_end(a, l, z, x); ++i) {                   \
                    int y = a->y_vec[i];                                                                   \
                    VT val = 0;                                                                            \
                    int cnt = 0;                                                                           \
                    for (int iz = 0; iz < s; ++iz) {                                                       \
                        int okz = 1; int zz = bc_index(z + iz - r, zn, reflect, &okz);                     \
                        for (int ix = 0; ix < s; ++ix) {                                                   \
                            int okx = 1; int xx = bc_index(x + ix - r, xn, reflect, &okx);                 \
                            for (int iy = 0; iy < s; ++iy) {                                               \
                                int oky = 1; int yy = bc_index(y + iy - r, yn, reflect, &oky);             \
                                VT v = 0;                                                                  \
                                if (okz == 1 && okx == 1 && oky == 1) {                                    \
                                    size_t q = IDX(yy, xx, zz, yn, xn);                                    \
                                    if (F[q]) v = D[q]; else stale++;                                      \
                                } else if (okz < 0 || okx < 0 || oky < 0) stale++;                         \
                                val += v * S[cnt++];                                                       \
                            }                                                                              \
                        }                                                                                  \
                    }                                                                                      \
                    out[i] = val;                                                                          \
                }                                                                                          \
        free(D); free(F);                                                                                  \
    }                                                                                                      \
    return stale;                                                                                          \
}
DEFINE_CONV(conv_f, float)
DEFINE_CONV(conv_d, double)

int orc_convolve(const orc_access *a, const orc_access *t, const float *stencils, const int *sides, int ns,
                 const float *in, float *out, int reflect, uint64_t *stale_reads) {
    float *tree = (float *)malloc(sizeof(float) * (t->P ? t->P : 1));
    tree_mean_f(a, t, in, tree);
    uint64_t s = conv_f(a, t, stencils, sides, ns, in, tree, out, reflect);
    if (stale_reads) *stale_reads = s;
    free(tree);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* a19: richardson_lucy (src/numerics/APRNumerics.hpp:551-593)               */
/* ------------------------------------------------------------------------ */
int orc_richardson_lucy(const orc_access *a, const orc_access *t, const uint16_t *in, void *outv, const float *psf,
                        int ks, int niter, int use_stencil_ds, int normalize, int resume, int use_double) {
    int nlev = use_stencil_ds ? a->l_max - a->l_min : 1;
    if (nlev < 1) nlev = 1;
    int n0 = ks * ks * ks;
    int sides[ORC_MAX_LEVELS], sides2[ORC_MAX_LEVELS];
    size_t cap = (size_t)n0 * (nlev + 1);
    uint64_t P = a->P;
    if (!use_double) {
        float *pf = (float *)malloc(sizeof(float) * n0), *pv = (float *)malloc(sizeof(float) * cap);
        float *fv = (float *)malloc(sizeof(float) * cap);
        for (int i = 0; i < n0; ++i) pf[i] = psf[n0 - 1 - i];
        get_stencils_f(psf, ks, nlev, normalize, pv, sides);
        get_stencils_f(pf, ks, nlev, normalize, fv, sides2);
        float *out = (float *)outv;
        if (!resume) for (uint64_t i = 0; i < P; ++i) out[i] = 1.0f;
        float *rb = (float *)malloc(sizeof(float) * (P ? P : 1)), *er = (float *)malloc(sizeof(float) * (P ? P : 1));
        float *tree = (float *)malloc(sizeof(float) * (t->P ? t->P : 1));
        for (int it = 0; it < niter; ++it) {
            tree_mean_f(a, t, out, tree);
            conv_f(a, t, fv, sides2, nlev, out, tree, rb, 1);
            for (uint64_t i = 0; i < P; ++i) rb[i] = (float)in[i] / rb[i];
            tree_mean_f(a, t, rb, tree);
            conv_f(a, t, pv, sides, nlev, rb, tree, er, 1);
            for (uint64_t i = 0; i < P; ++i) out[i] = out[i] * er[i];
        }
        free(pf); free(pv); free(fv); free(rb); free(er); free(tree);
    } else {
        double *pd = (double *)malloc(sizeof(double) * n0), *pfd = (double *)malloc(sizeof(double) * n0);
        double *pv = (double *)malloc(sizeof(double) * cap), *fv = (double *)malloc(sizeof(double) * cap);
        for (int i = 0; i < n0; ++i) pd[i] = (double)psf[i];
        for (int i = 0; i < n0; ++i) pfd[i] = pd[n0 - 1 - i];
        get_stencils_d(pd, ks, nlev, normalize, pv, sides);
        get_stencils_d(pfd, ks, nlev, normalize, fv, sides2);
        double *out = (double *)outv;
        if (!resume) for (uint64_t i = 0; i < P; ++i) out[i] = 1.0;
        double *rb = (double *)malloc(sizeof(double) * (P ? P : 1)), *er = (double *)malloc(sizeof(double) * (P ? P : 1));
        double *tree = (double *)malloc(sizeof(double) * (t->P ? t->P : 1));
        for (int it = 0; it < niter; ++it) {
            tree_mean_d(a, t, out, tree);
            conv_d(a, t, fv, sides2, nlev, out, tree, rb, 1);
            for (uint64_t i = 0; i < P; ++i) rb[i] = (double)in[i] / rb[i];
            tree_mean_d(a, t, rb, tree);
            conv_d(a, t, pv, sides, nlev, rb, tree, er, 1);
            for (uint64_t i = 0; i < P; ++i) out[i] = out[i] * er[i];
        }
        free(pd); free(pfd); free(pv); free(fv); free(rb); free(er); free(tree);
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------ automatic parameters */

/* Means of the values above / at-or-below t (compute_means,
 * src/algorithm/AutoParameters.hpp:17-36): float sums in index order, or
 * double sums. */
static void li_means(const float *v, size_t n, float t, int fp32_sums, float *mean_back, float *mean_fore) {
    if (fp32_sums) {
        float sf = 0.f, sb = 0.f;
        size_t cf = 0, cb = 0;
        for (size_t i = 0; i < n; ++i) {
            if (v[i] > t) { sf += v[i]; cf++; } else { sb += v[i]; cb++; }
        }
        *mean_fore = sf / (float)cf;
        *mean_back = sb / (float)cb;
    } else {
        double sf = 0, sb = 0;
        size_t cf = 0, cb = 0;
        for (size_t i = 0; i < n; ++i) {
            if (v[i] > t) { sf += v[i]; cf++; } else { sb += v[i]; cb++; }
        }
        *mean_fore = (float)(sf / (double)cf);
        *mean_back = (float)(sb / (double)cb);
    }
}

/* threshold_li<T> (src/algorithm/AutoParameters.hpp:50-100) with the
 * iteration bounded by ORC_LI_MAX_ITER steps. */
#define ORC_LI_MAX_ITER 1000
float orc_threshold_li(const float *v, size_t n, int integer_values, int fp32_sums) {
    if (n == 0) return 0.f;
    float mn = v[0], mx = v[0];
    for (size_t i = 1; i < n; ++i) {
        if (v[i] < mn) mn = v[i];
        if (v[i] > mx) mx = v[i];
    }
    if (mn == mx) return mn;
    float tol = 0.5f;
    if (!integer_values) {
        const float range = mx - mn;
        tol = fminf(0.01f, range * 1e-4f);
    }
    float t_next;
    if (fp32_sums) {
        float s = 0.f;
        for (size_t i = 0; i < n; ++i) s += v[i];
        t_next = s / (float)n;
    } else {
        double s = 0;
        for (size_t i = 0; i < n; ++i) s += v[i];
        t_next = (float)(s / (double)n);
    }
    float t_curr = -2.f * tol;
    if (integer_values && t_next < 1.f) {
        const float mid = (mn + mx) / 2.f;
        t_next = mid < 1.5f ? mid : 1.5f;
    }
    for (int it = 0; it < ORC_LI_MAX_ITER && fabsf(t_next - t_curr) > tol; ++it) {
        t_curr = t_next;
        float mb, mf;
        li_means(v, n, t_curr, fp32_sums, &mb, &mf);
        if (mb == 0) return t_curr;
        t_next = (mf - mb) / (logf(mf) - logf(mb));
    }
    return t_next;
}

/* autoParametersLiEntropy (src/algorithm/AutoParameters.hpp:103-153). */
int orc_auto_parameters(const float *image, const float *lis, const float *grad, size_t n, float threshold,
                        int grad_integer, int fp32_sums, float *grad_th, float *sigma_th, float *sub_grad,
                        float *sub_lis, size_t *m_out) {
    float *fg = (float *)malloc(sizeof(float) * (n ? n : 1)), *fl = (float *)malloc(sizeof(float) * (n ? n : 1));
    if (!fg || !fl) { free(fg); free(fl); return ORC_ERR_ALLOC; }
    size_t nf = 0;
    for (size_t i = 0; i < n; ++i)
        if (image[i] > threshold) { fg[nf] = grad[i]; fl[nf] = lis[i]; nf++; }
    const size_t cap = (size_t)32 * 512 * 512;
    const size_t m = nf < cap ? nf : cap;
    /* the reference divides by m here; with no foreground pixel both
     * thresholds are those of an empty input */
    const size_t delta = m ? nf / m : 0;
    for (size_t i = 0; i < m; ++i) { fg[i] = fg[i * delta]; fl[i] = fl[i * delta]; }
    *grad_th = orc_threshold_li(fg, m, grad_integer, fp32_sums);
    *sigma_th = orc_threshold_li(fl, m, 0, fp32_sums);
    if (sub_grad) memcpy(sub_grad, fg, sizeof(float) * m);
    if (sub_lis) memcpy(sub_lis, fl, sizeof(float) * m);
    if (m_out) *m_out = m;
    free(fg); free(fl);
    return ORC_OK;
}
