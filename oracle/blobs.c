/* TEST INFRASTRUCTURE ONLY.
 *
 * CPU twin of the library's seeded synthetic-volume generator
 * (aprb_synth_blobs_u16 / aprb_synth_blobs_f32): background + isotropic
 * Gaussian blobs (+ Poisson noise, rounded and clipped to uint16).  It
 * performs the same IEEE operations in the same order as the device code --
 * splitmix64 blob parameters, 16^3 bricks summing the blobs whose 4-sigma box
 * meets them in blob order, Cody-Waite exponentials with Taylor polynomials,
 * atanh-series logarithms, Stirling log-factorials, Hoermann's PTRS Poisson
 * sampler -- so it writes the same bytes, and a CPU run (the reference's own
 * code timed on the host) gets the benchmark volume without a GPU or the
 * library.  Compile without contraction (-ffp-contract=off, no fast-math).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define BRICK 16

typedef struct {
    float cz, cx, cy, inv2s2, amp;
} blob_t;

static uint64_t splitmix64(uint64_t *s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double unif(uint64_t *s) { return (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0); }

static uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double rng_next(uint64_t *s) {
    *s += 0x9E3779B97F4A7C15ull;
    return (double)(mix64(*s) >> 11) * (1.0 / 9007199254740992.0);
}

static float bits_f(uint32_t b) {
    float f;
    memcpy(&f, &b, 4);
    return f;
}
static double bits_d(uint64_t b) {
    double d;
    memcpy(&d, &b, 8);
    return d;
}
static uint64_t d_bits(double d) {
    uint64_t b;
    memcpy(&b, &d, 8);
    return b;
}

static float exp_nonpos_f(float x) {
    if (!(x > -87.0f)) return 0.0f;
    const float kf = floorf(x * 1.44269504f + 0.5f);
    const int k = (int)kf;
    const float r = (x - kf * 0.693145751953125f) - kf * 1.42860677e-06f;
    float p = 1.98412701e-04f;
    p = p * r + 1.38888892e-03f;
    p = p * r + 8.33333377e-03f;
    p = p * r + 4.16666679e-02f;
    p = p * r + 1.66666672e-01f;
    p = p * r + 0.5f;
    p = p * r + 1.0f;
    p = p * r + 1.0f;
    return p * bits_f((uint32_t)(k + 127) << 23);
}

static double exp_nonpos_d(double x) {
    if (!(x > -700.0)) return 0.0;
    const double kf = floor(x * 1.4426950408889634 + 0.5);
    const long long k = (long long)kf;
    const double r = (x - kf * 0.6931471803691238) - kf * 1.9082149292705877e-10;
    double p = 1.6059043836821613e-10;
    p = p * r + 2.08767569878681e-09;
    p = p * r + 2.505210838544172e-08;
    p = p * r + 2.755731922398589e-07;
    p = p * r + 2.7557319223985893e-06;
    p = p * r + 2.48015873015873e-05;
    p = p * r + 0.0001984126984126984;
    p = p * r + 0.001388888888888889;
    p = p * r + 0.008333333333333333;
    p = p * r + 0.041666666666666664;
    p = p * r + 0.16666666666666666;
    p = p * r + 0.5;
    p = p * r + 1.0;
    p = p * r + 1.0;
    return p * bits_d((uint64_t)(k + 1023) << 52);
}

static double log_d(double x) {
    if (!(x > 0.0)) return x == 0.0 ? -INFINITY : NAN;
    if (x == INFINITY) return x;
    int e = 0;
    if (x < 2.2250738585072014e-308) {
        x *= 18014398509481984.0;
        e = -54;
    }
    const uint64_t b = d_bits(x);
    e += (int)((b >> 52) & 0x7ff) - 1023;
    double m = bits_d((b & 0xfffffffffffffull) | 0x3ff0000000000000ull);
    if (m > 1.4142135623730951) {
        m = m * 0.5;
        e += 1;
    }
    const double s = (m - 1.0) / (m + 1.0);
    const double s2 = s * s;
    double p = 0.043478260869565216;
    p = p * s2 + 0.047619047619047616;
    p = p * s2 + 0.05263157894736842;
    p = p * s2 + 0.058823529411764705;
    p = p * s2 + 0.06666666666666667;
    p = p * s2 + 0.07692307692307693;
    p = p * s2 + 0.09090909090909091;
    p = p * s2 + 0.1111111111111111;
    p = p * s2 + 0.14285714285714285;
    p = p * s2 + 0.2;
    p = p * s2 + 0.3333333333333333;
    p = p * s2 + 1.0;
    const double ed = (double)e;
    return ed * 0.6931471803691238 + ((2.0 * s) * p + ed * 1.9082149292705877e-10);
}

static double log_factorial(long long k) {
    if (k < 2) return 0.0;
    if (k < 18) {
        double f = 1.0;
        for (long long i = 2; i <= k; ++i) f = f * (double)i;
        return log_d(f);
    }
    const double n = (double)(k + 1);
    const double inv = 1.0 / n, inv2 = inv * inv;
    const double series =
        inv * (0.08333333333333333 +
               inv2 * (-0.002777777777777778 + inv2 * (0.0007936507936507937 + inv2 * -0.0005952380952380953)));
    return (((n - 0.5) * log_d(n) - n) + 0.9189385332046727) + series;
}

static int poisson(double lam, uint64_t *r) {
    if (lam <= 0) return 0;
    if (lam < 10.0) {
        const double L = exp_nonpos_d(-lam);
        double p = 1.0;
        int k = 0;
        do {
            ++k;
            p = p * rng_next(r);
        } while (p > L && k < 1000);
        return k - 1;
    }
    const double slam = sqrt(lam), loglam = log_d(lam);
    const double b = 0.931 + 2.53 * slam, a = -0.059 + 0.02483 * b;
    const double invalpha = 1.1239 + 1.1328 / (b - 3.4), vr = 0.9277 - 3.6224 / (b - 2.0);
    const double log_invalpha = log_d(invalpha);
    for (int it = 0; it < 1000; ++it) {
        const double U = rng_next(r) - 0.5, V = rng_next(r);
        const double us = 0.5 - fabs(U);
        const long long k = (long long)floor(((2.0 * a) / us + b) * U + lam + 0.43);
        if (us >= 0.07 && V <= vr) return (int)k;
        if (k < 0 || (us < 0.013 && V > us)) continue;
        const double lhs = (log_d(V) + log_invalpha) - log_d(a / (us * us) + b);
        const double rhs = (-lam + (double)k * loglam) - log_factorial(k);
        if (lhs <= rhs) return (int)k;
    }
    return (int)lam;
}

static int imax(int a, int b) { return a > b ? a : b; }
static int imin(int a, int b) { return a < b ? a : b; }

/* out_u16 (noise) or out_f32 (noise-free intensities); returns 0 or 1 on
 * allocation failure. */
static int render(uint16_t *out_u16, float *out_f32, int yn, int xn, int zn, int n_blobs, float slo, float shi,
                  float alo, float ahi, float bg, uint64_t seed) {
    uint64_t st = seed * 0x2545F4914F6CDD1Dull + 0x632BE59BD9B4E019ull;
    const int by = (yn + BRICK - 1) / BRICK, bx = (xn + BRICK - 1) / BRICK, bz = (zn + BRICK - 1) / BRICK;
    const uint64_t nb = (uint64_t)by * bx * bz;
    blob_t *blobs = (blob_t *)malloc(sizeof(blob_t) * (size_t)(n_blobs > 0 ? n_blobs : 1));
    int *lo = (int *)malloc(sizeof(int) * 6 * (size_t)(n_blobs > 0 ? n_blobs : 1));
    uint32_t *count = (uint32_t *)calloc(nb + 1, sizeof(uint32_t));
    if (!blobs || !lo || !count) {
        free(blobs), free(lo), free(count);
        return 1;
    }
    for (int i = 0; i < n_blobs; ++i) {
        blob_t *B = &blobs[i];
        B->cz = (float)(unif(&st) * zn);
        B->cx = (float)(unif(&st) * xn);
        B->cy = (float)(unif(&st) * yn);
        const float sg = (float)(slo + unif(&st) * (shi - slo));
        B->amp = (float)(alo + unif(&st) * (ahi - alo));
        B->inv2s2 = 1.0f / (2.0f * sg * sg);
        const float r = 4.0f * sg;
        int *q = &lo[6 * (size_t)i];
        q[0] = imax(0, (int)floorf((B->cz - r) / BRICK));
        q[1] = imin(bz - 1, (int)floorf((B->cz + r) / BRICK));
        q[2] = imax(0, (int)floorf((B->cx - r) / BRICK));
        q[3] = imin(bx - 1, (int)floorf((B->cx + r) / BRICK));
        q[4] = imax(0, (int)floorf((B->cy - r) / BRICK));
        q[5] = imin(by - 1, (int)floorf((B->cy + r) / BRICK));
        for (int a = q[0]; a <= q[1]; ++a)
            for (int b = q[2]; b <= q[3]; ++b)
                for (int c = q[4]; c <= q[5]; ++c) count[((uint64_t)a * bx + b) * by + c + 1]++;
    }
    for (uint64_t i = 1; i <= nb; ++i) count[i] += count[i - 1];
    uint32_t *idx = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(count[nb] ? count[nb] : 1));
    uint32_t *fill = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)nb);
    if (!idx || !fill) {
        free(blobs), free(lo), free(count), free(idx), free(fill);
        return 1;
    }
    memcpy(fill, count, sizeof(uint32_t) * (size_t)nb);
    for (int i = 0; i < n_blobs; ++i) {
        const int *q = &lo[6 * (size_t)i];
        for (int a = q[0]; a <= q[1]; ++a)
            for (int b = q[2]; b <= q[3]; ++b)
                for (int c = q[4]; c <= q[5]; ++c) idx[fill[((uint64_t)a * bx + b) * by + c]++] = (uint32_t)i;
    }
#pragma omp parallel for schedule(dynamic, 4)
    for (long long brick = 0; brick < (long long)nb; ++brick) {
        const int bYi = (int)(brick % by), bXi = (int)((brick / by) % bx), bZi = (int)(brick / ((long long)by * bx));
        const uint32_t b0 = count[brick], b1 = count[brick + 1];
        for (int t = 0; t < BRICK * BRICK * BRICK; ++t) {
            const int y = bYi * BRICK + (t % BRICK), x = bXi * BRICK + ((t / BRICK) % BRICK),
                      z = bZi * BRICK + t / (BRICK * BRICK);
            if (y >= yn || x >= xn || z >= zn) continue;
            float v = bg;
            const float fy = y + 0.5f, fx = x + 0.5f, fz = z + 0.5f;
            for (uint32_t k = b0; k < b1; ++k) {
                const blob_t B = blobs[idx[k]];
                const float dy = fy - B.cy, dx = fx - B.cx, dz = fz - B.cz;
                v = v + B.amp * exp_nonpos_f(-((dy * dy + dx * dx) + dz * dz) * B.inv2s2);
            }
            const uint64_t vox = ((uint64_t)z * xn + x) * yn + y;
            if (out_u16) {
                uint64_t r = mix64(seed ^ mix64(vox + 0x1234567ull));
                int p = poisson((double)v, &r);
                p = p < 0 ? 0 : (p > 65535 ? 65535 : p);
                out_u16[vox] = (uint16_t)p;
            } else {
                out_f32[vox] = v;
            }
        }
    }
    free(blobs), free(lo), free(count), free(idx), free(fill);
    return 0;
}

int blobs_render_u16(uint16_t *img, int yn, int xn, int zn, int n_blobs, float slo, float shi, float alo, float ahi,
                     float bg, uint64_t seed) {
    return render(img, NULL, yn, xn, zn, n_blobs, slo, shi, alo, ahi, bg, seed);
}

int blobs_render_f32(float *img, int yn, int xn, int zn, int n_blobs, float slo, float shi, float alo, float ahi,
                     float bg, uint64_t seed) {
    return render(NULL, img, yn, xn, zn, n_blobs, slo, shi, alo, ahi, bg, seed);
}
