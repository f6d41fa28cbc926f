// Seeded synthetic benchmark volumes: background + isotropic Gaussian blobs +
// Poisson noise, rounded and clipped to uint16.  Blob parameters come from a
// host splitmix64 stream; each 16^3 brick of the volume sums the blobs whose
// 4-sigma box meets it, in blob order, so the image is deterministic.  Poisson
// deviates use a counter-based generator per voxel: multiplication of
// uniforms for small means, Hoermann's transformed rejection (PTRS, 1993)
// otherwise.
//
// The exponentials, logarithms and log-factorials are this file's own
// (Cody-Waite range reduction with Taylor, atanh and Stirling series) and
// use only IEEE-rounded additions, multiplications, divisions, square roots
// and floors, with no contraction (-fmad=false), so a host program that
// performs the same operations in the same order reproduces every voxel bit
// for bit: a CPU run of the same workload can be fed the same bytes without
// a GPU.
#include <math_constants.h>

#include <type_traits>
#include <vector>

#include "kernels.cuh"

namespace aprb {

namespace {

constexpr int kBrick = 16;

struct Blob {
    float cz, cx, cy, inv2s2, amp;
};

uint64_t splitmix64(uint64_t &s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double unif(uint64_t &s) { return (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0); }

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct Rng {
    uint64_t s;
    __device__ double next() {
        s += 0x9E3779B97F4A7C15ull;
        return (double)(mix64(s) >> 11) * (1.0 / 9007199254740992.0);
    }
};

// exp(x) for x <= 0 in float: x = k ln2 + r with the Cody-Waite split of
// ln2 (|r| <= ln2/2), exp(r) by its Taylor polynomial of degree 7 (truncation
// below 6e-9 relative), times 2^k built from the exponent bits.  Below -87 the
// result is 0 (exp(-87) < 2^-125).
__device__ __forceinline__ float exp_nonpos_f(float x) {
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
    return p * __int_as_float((k + 127) << 23);
}

// exp(x) for -700 < x <= 0 in double: the same reduction with the fdlibm
// split of ln2 and the Taylor polynomial of degree 13.
__device__ __forceinline__ double exp_nonpos_d(double x) {
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
    return p * __longlong_as_double((k + 1023) << 52);
}

// log(x) in double: x = m 2^e with m in [sqrt(1/2), sqrt(2)), log(m) =
// 2 atanh(s), s = (m - 1)/(m + 1), |s| <= 0.1716, by its series to s^23.
__device__ __forceinline__ double log_d(double x) {
    if (!(x > 0.0)) return x == 0.0 ? -CUDART_INF : CUDART_NAN;
    if (x == CUDART_INF) return x;
    int e = 0;
    if (x < 2.2250738585072014e-308) {
        x *= 18014398509481984.0;  // 2^54
        e = -54;
    }
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    e += (int)((b >> 52) & 0x7ff) - 1023;
    double m = __longlong_as_double((long long)((b & 0xfffffffffffffull) | 0x3ff0000000000000ull));
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

// log(k!) for k >= 0: the exact product below 18! (exactly representable),
// else Stirling's series for lgamma(k + 1) to the 1/n^7 term.
__device__ __forceinline__ double log_factorial(long long k) {
    if (k < 2) return 0.0;
    if (k < 18) {
        double f = 1.0;
        for (long long i = 2; i <= k; ++i) f = f * (double)i;
        return log_d(f);
    }
    const double n = (double)(k + 1);
    const double inv = 1.0 / n, inv2 = inv * inv;
    const double series =
        inv * (0.08333333333333333 + inv2 * (-0.002777777777777778 +
                                             inv2 * (0.0007936507936507937 + inv2 * -0.0005952380952380953)));
    return (((n - 0.5) * log_d(n) - n) + 0.9189385332046727) + series;
}

__device__ int poisson(double lam, Rng &r) {
    if (lam <= 0) return 0;
    if (lam < 10.0) {
        const double L = exp_nonpos_d(-lam);
        double p = 1.0;
        int k = 0;
        do {
            ++k;
            p = p * r.next();
        } while (p > L && k < 1000);
        return k - 1;
    }
    const double slam = sqrt(lam), loglam = log_d(lam);
    const double b = 0.931 + 2.53 * slam, a = -0.059 + 0.02483 * b;
    const double invalpha = 1.1239 + 1.1328 / (b - 3.4), vr = 0.9277 - 3.6224 / (b - 2.0);
    const double log_invalpha = log_d(invalpha);
    for (int it = 0; it < 1000; ++it) {
        const double U = r.next() - 0.5, V = r.next();
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

// NOISE: Poisson deviate clipped to uint16 (OutT uint16_t); otherwise the
// noise-free intensity (OutT float), the ground truth of the deconvolution
// workload.
template <bool NOISE, typename OutT>
__global__ void render_kernel(OutT *__restrict__ img, int yn, int xn, int zn, const Blob *__restrict__ blobs,
                              const uint32_t *__restrict__ boff, const uint32_t *__restrict__ bidx, int bx, int by,
                              float bg, uint64_t seed) {
    const int brick = blockIdx.x;
    const int bYi = brick % by, bXi = (brick / by) % bx, bZi = brick / (by * bx);
    const uint32_t b0 = boff[brick], b1 = boff[brick + 1];
    for (int t = threadIdx.x; t < kBrick * kBrick * kBrick; t += blockDim.x) {
        const int y = bYi * kBrick + (t % kBrick), x = bXi * kBrick + ((t / kBrick) % kBrick),
                  z = bZi * kBrick + t / (kBrick * kBrick);
        if (y >= yn || x >= xn || z >= zn) continue;
        float v = bg;
        const float fy = y + 0.5f, fx = x + 0.5f, fz = z + 0.5f;
        for (uint32_t k = b0; k < b1; ++k) {
            const Blob B = blobs[bidx[k]];
            const float dy = fy - B.cy, dx = fx - B.cx, dz = fz - B.cz;
            v = v + B.amp * exp_nonpos_f(-((dy * dy + dx * dx) + dz * dz) * B.inv2s2);
        }
        const uint64_t vox = idx3(y, x, z, yn, xn);
        if (NOISE) {
            Rng r{mix64(seed ^ mix64(vox + 0x1234567ull))};
            int p = poisson((double)v, r);
            p = p < 0 ? 0 : (p > 65535 ? 65535 : p);
            img[vox] = (OutT)p;
        } else {
            img[vox] = (OutT)v;
        }
    }
}

}  // namespace

template <typename OutT>
void launch_synth_blobs(OutT *img, int yn, int xn, int zn, int n_blobs, float slo, float shi, float alo, float ahi,
                        float bg, uint64_t seed, DevBuf &buf, cudaStream_t s) {
    uint64_t st = seed * 0x2545F4914F6CDD1Dull + 0x632BE59BD9B4E019ull;
    std::vector<Blob> blobs((size_t)n_blobs);
    const int by = (yn + kBrick - 1) / kBrick, bx = (xn + kBrick - 1) / kBrick, bz = (zn + kBrick - 1) / kBrick;
    const uint64_t nb = (uint64_t)by * bx * bz;
    std::vector<uint32_t> count(nb + 1, 0);
    std::vector<int> lo(6 * (size_t)n_blobs);
    for (int i = 0; i < n_blobs; ++i) {
        Blob &B = blobs[i];
        B.cz = (float)(unif(st) * zn);
        B.cx = (float)(unif(st) * xn);
        B.cy = (float)(unif(st) * yn);
        const float sg = (float)(slo + unif(st) * (shi - slo));
        B.amp = (float)(alo + unif(st) * (ahi - alo));
        B.inv2s2 = 1.0f / (2.0f * sg * sg);
        const float r = 4.0f * sg;
        int *q = &lo[6 * (size_t)i];
        q[0] = std::max(0, (int)std::floor((B.cz - r) / kBrick));
        q[1] = std::min(bz - 1, (int)std::floor((B.cz + r) / kBrick));
        q[2] = std::max(0, (int)std::floor((B.cx - r) / kBrick));
        q[3] = std::min(bx - 1, (int)std::floor((B.cx + r) / kBrick));
        q[4] = std::max(0, (int)std::floor((B.cy - r) / kBrick));
        q[5] = std::min(by - 1, (int)std::floor((B.cy + r) / kBrick));
        for (int a = q[0]; a <= q[1]; ++a)
            for (int b = q[2]; b <= q[3]; ++b)
                for (int c = q[4]; c <= q[5]; ++c) count[((uint64_t)a * bx + b) * by + c + 1]++;
    }
    for (uint64_t i = 1; i <= nb; ++i) count[i] += count[i - 1];
    std::vector<uint32_t> idx(count[nb]);
    std::vector<uint32_t> fill(count.begin(), count.end() - 1);
    for (int i = 0; i < n_blobs; ++i) {
        const int *q = &lo[6 * (size_t)i];
        for (int a = q[0]; a <= q[1]; ++a)
            for (int b = q[2]; b <= q[3]; ++b)
                for (int c = q[4]; c <= q[5]; ++c) idx[fill[((uint64_t)a * bx + b) * by + c]++] = (uint32_t)i;
    }
    const size_t bytes_blobs = sizeof(Blob) * blobs.size(), bytes_off = sizeof(uint32_t) * count.size(),
                 bytes_idx = sizeof(uint32_t) * idx.size();
    char *d = (char *)buf.get(bytes_blobs + bytes_off + bytes_idx + 64);
    Blob *dB = (Blob *)d;
    uint32_t *dO = (uint32_t *)(d + ((bytes_blobs + 15) & ~size_t(15)));
    uint32_t *dI = dO + count.size();
    APRB_CUDA(cudaMemcpyAsync(dB, blobs.data(), bytes_blobs, cudaMemcpyHostToDevice, s));
    APRB_CUDA(cudaMemcpyAsync(dO, count.data(), bytes_off, cudaMemcpyHostToDevice, s));
    if (bytes_idx) APRB_CUDA(cudaMemcpyAsync(dI, idx.data(), bytes_idx, cudaMemcpyHostToDevice, s));
    render_kernel<std::is_same<OutT, uint16_t>::value, OutT>
        <<<(unsigned)nb, 256, 0, s>>>(img, yn, xn, zn, dB, dO, dI, bx, by, bg, seed);
    count_launch();
    APRB_CHECK_LAUNCH();
    APRB_CUDA(cudaStreamSynchronize(s));  // host vectors go out of scope
}

template void launch_synth_blobs<uint16_t>(uint16_t *, int, int, int, int, float, float, float, float, float, uint64_t,
                                           DevBuf &, cudaStream_t);
template void launch_synth_blobs<float>(float *, int, int, int, int, float, float, float, float, float, uint64_t,
                                        DevBuf &, cudaStream_t);

}  // namespace aprb
