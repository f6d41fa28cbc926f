// Pixel stages of get_apr on the GPU: offset, smoothing-spline recursive
// filters along y/x/z, gradient magnitude fused with the 2x max and mean
// down-sampling, inverse B-spline at ds resolution, local intensity scale,
// and the fused applyParameters + computeLevels + top-level seeding.
//
// Bit-exactness: each kernel performs the reference's float operations in the
// reference's order (ComputeGradient.hpp, LocalIntensityScale.hpp,
// LocalParticleCellSet.hpp, APRConverter.hpp); recurrences that the reference
// runs sequentially along a line run sequentially in one thread here.
#include <map>
#include <mutex>
#include <type_traits>
#include <vector>

#include "kernels.cuh"

namespace aprb {

// ---------------------------------------------------------------------------
// a1: compute_bspline_offset (AutoParameters.hpp:164-197) -- min/max reduction
// then the clamped offset, kept on the device.
// ---------------------------------------------------------------------------
__global__ void minmax_u16_kernel(const uint16_t *__restrict__ img, uint64_t n, unsigned *mm) {
    unsigned mn = 0xffffu, mx = 0u;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        unsigned v = img[i];
        mn = v < mn ? v : mn;
        mx = v > mx ? v : mx;
    }
    mn = __reduce_min_sync(0xffffffffu, mn);
    mx = __reduce_max_sync(0xffffffffu, mx);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&mm[0], mn);
        atomicMax(&mm[1], mx);
    }
}

__global__ void offset_kernel(const unsigned *mm, float *offset, int apply) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (!apply) {
        *offset = 0.0f;
        return;
    }
    int mn = (int)mm[0], mx = (int)mm[1];
    float off = (float)((65535 - (mx - mn)) / 2 - mn);
    off = off < 100.f ? off : 100.f;
    *offset = off > -100.f ? off : -100.f;
}

// Working-image value of the raw input: image_temp = IT(input + offset) for
// integer IT, a plain copy for float IT (APRConverter.hpp:218-223).
template <typename IT>
__device__ __forceinline__ float raw_to_it(uint16_t v, float off);
template <>
__device__ __forceinline__ float raw_to_it<uint16_t>(uint16_t v, float off) {
    return cvt_u16((float)v + off);
}
template <>
__device__ __forceinline__ float raw_to_it<float>(uint16_t v, float) {
    return (float)v;
}

template <typename IT>
__device__ __forceinline__ float rnd_it(float v, unsigned &err);
template <>
__device__ __forceinline__ float rnd_it<uint16_t>(float v, unsigned &err) {
    return round_u16(v, err);
}
template <>
__device__ __forceinline__ float rnd_it<float>(float v, unsigned &) {
    return v;
}
template <typename IT>
__device__ __forceinline__ float store_cvt(float v);
template <>
__device__ __forceinline__ float store_cvt<uint16_t>(float v) {
    return cvt_u16(v);
}
template <>
__device__ __forceinline__ float store_cvt<float>(float v) {
    return v;
}
template <typename IT>
__device__ __forceinline__ IT to_it(float v) {
    return (IT)v;
}

// ---------------------------------------------------------------------------
// a2 (y): bspline_filt_rec_y (ComputeGradient.hpp:249-413).
// One thread owns one y-line (the recurrence is sequential); a warp owns 32
// consecutive lines and moves them through shared memory in 32 x 64 tiles
// (coalesced loads/stores), prefetching the next tile into registers while
// the current one runs.  The forward pass stores its values; the backward pass
// reads them back (through L2, __ldcg).
// ---------------------------------------------------------------------------
constexpr int kTile = 32;
constexpr int kYW = 64;  // y extent of a tile
constexpr int kYWarps = 4;

template <typename IT>
__device__ __forceinline__ float ld_it(const IT *p) {
    return (float)__ldcg(p);
}

template <typename IT>
__global__ void __launch_bounds__(kYWarps * 32) iir_y_kernel(const uint16_t *__restrict__ src, IT *__restrict__ dst,
                                                              int yn, uint64_t nlines, IIRDev c,
                                                              const float *__restrict__ d_offset, unsigned *err_out) {
    __shared__ float tile[kYWarps][kTile][kYW + 1];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t line0 = ((uint64_t)blockIdx.x * kYWarps + w) * kTile;
    if (line0 >= nlines) return;
    const uint64_t myline = line0 + lane;
    const bool valid = myline < nlines;
    const int nl = (int)min((uint64_t)kTile, nlines - line0);  // lines of this warp
    const float off = d_offset ? *d_offset : 0.0f;
    float(*T)[kYW + 1] = tile[w];
    unsigned err = 0;

    float t1 = 0, t2 = 0, t3 = 0, t4 = 0;
    if (valid) {
        const uint16_t *L = src + myline * (uint64_t)yn;
        for (int k = 0; k < c.minLen; ++k) {
            float v = raw_to_it<IT>(L[k], off);
            t1 = t1 + __ldg(c.bc + k) * v;
            t2 = t2 + __ldg(c.bc + c.minLen + k) * v;
        }
        for (int k = 0; k < c.minLen; ++k) {
            float v = raw_to_it<IT>(L[yn - 1 - k], off);
            t3 = t3 + __ldg(c.bc + 2 * c.minLen + k) * v;
            t4 = t4 + __ldg(c.bc + 3 * c.minLen + k) * v;
        }
    }
    const int ya = 2 * lane, yb = 2 * lane + 1;  // columns this lane moves
    // ---- forward (causal) pass
    uint16_t pa[kTile], pb[kTile];
#pragma unroll
    for (int j = 0; j < kTile; ++j) {
        const uint16_t *L = src + (line0 + j) * (uint64_t)yn;
        pa[j] = (j < nl && ya < yn) ? L[ya] : 0;
        pb[j] = (j < nl && yb < yn) ? L[yb] : 0;
    }
    for (int y0 = 0; y0 < yn; y0 += kYW) {
#pragma unroll
        for (int j = 0; j < kTile; ++j) {
            T[j][ya] = raw_to_it<IT>(pa[j], off);
            T[j][yb] = raw_to_it<IT>(pb[j], off);
        }
        __syncwarp();
        const int n0 = y0 + kYW;
        if (n0 < yn) {
#pragma unroll
            for (int j = 0; j < kTile; ++j) {
                const uint16_t *L = src + (line0 + j) * (uint64_t)yn + n0;
                pa[j] = (j < nl && n0 + ya < yn) ? L[ya] : 0;
                pb[j] = (j < nl && n0 + yb < yn) ? L[yb] : 0;
            }
        }
        if (valid) {
            const int kend = min(kYW, yn - y0);
            for (int k = 0; k < kend; ++k) {
                const int y = y0 + k;
                float out;
                if (y == 0) {
                    out = store_cvt<IT>(t2);
                } else if (y == 1) {
                    out = store_cvt<IT>(t1);
                } else {
                    float temp = t1 * c.b1 + t2 * c.b2 + T[lane][k];
                    out = rnd_it<IT>(temp, err);
                    t2 = t1;
                    t1 = temp;
                }
                if (y == yn - 2) out = rnd_it<IT>(t3 * c.norm, err);
                if (y == yn - 1) out = rnd_it<IT>(t4 * c.norm, err);
                T[lane][k] = out;
            }
        }
        __syncwarp();
#pragma unroll 4
        for (int j = 0; j < nl; ++j) {
            IT *L = dst + (line0 + j) * (uint64_t)yn + y0;
            if (y0 + ya < yn) L[ya] = to_it<IT>(T[j][ya]);
            if (y0 + yb < yn) L[yb] = to_it<IT>(T[j][yb]);
        }
        __syncwarp();
    }
    // ---- backward (anti-causal) pass
    float b2v = 0, b1v = 0;
    if (valid) {
        const IT *L = dst + myline * (uint64_t)yn;
        b2v = ld_it(&L[yn - 1]) / c.norm;
        b1v = ld_it(&L[yn - 2]) / c.norm;
    }
    const int last0 = ((yn - 1) / kYW) * kYW;
    float fa[kTile], fb[kTile];
#pragma unroll
    for (int j = 0; j < kTile; ++j) {
        const IT *L = dst + (line0 + j) * (uint64_t)yn + last0;
        fa[j] = (j < nl && last0 + ya < yn) ? ld_it(&L[ya]) : 0.0f;
        fb[j] = (j < nl && last0 + yb < yn) ? ld_it(&L[yb]) : 0.0f;
    }
    for (int y0 = last0; y0 >= 0; y0 -= kYW) {
#pragma unroll
        for (int j = 0; j < kTile; ++j) {
            T[j][ya] = fa[j];
            T[j][yb] = fb[j];
        }
        __syncwarp();
        const int p0 = y0 - kYW;
        if (p0 >= 0) {
#pragma unroll
            for (int j = 0; j < kTile; ++j) {
                const IT *L = dst + (line0 + j) * (uint64_t)yn + p0;
                fa[j] = (j < nl) ? ld_it(&L[ya]) : 0.0f;
                fb[j] = (j < nl) ? ld_it(&L[yb]) : 0.0f;
            }
        }
        if (valid) {
            const int kend = min(kYW, yn - y0);
            for (int k = kend - 1; k >= 0; --k) {
                const int y = y0 + k;
                if (y > yn - 3) continue;
                float temp = b1v * c.b1 + b2v * c.b2 + T[lane][k];
                T[lane][k] = rnd_it<IT>(temp * c.norm, err);
                b2v = b1v;
                b1v = temp;
            }
        }
        __syncwarp();
#pragma unroll 4
        for (int j = 0; j < nl; ++j) {
            IT *L = dst + (line0 + j) * (uint64_t)yn + y0;
            if (y0 + ya < yn) L[ya] = to_it<IT>(T[j][ya]);
            if (y0 + yb < yn) L[yb] = to_it<IT>(T[j][yb]);
        }
        __syncwarp();
    }
    if (err) atomicAdd(err_out, err);
}

// ---------------------------------------------------------------------------
// a2 (x, z): bspline_filt_rec_x (ComputeGradient.hpp:602-779) and
// bspline_filt_rec_z (:416-599).  One thread per line along the strided axis;
// neighbouring threads own neighbouring y so every step is a coalesced row.
// In place.
// ---------------------------------------------------------------------------
// The same x / z recurrences without the round trip of the causal values
// through memory: the causal sweep reads the line and keeps only the
// recurrence state at the start of every kRC-sample segment (ckpt,
// [segment][line] pairs); the anti-causal sweep walks the segments from the
// end, recomputes each segment's causal values from its saved state and the
// still untouched input -- the same operations on the same values -- and
// writes the results over it.  Traffic per sample: 4 B read twice and 4 B
// written, plus 16 B of state per 16 samples, instead of 16 B.
constexpr int kRC = 16;
template <typename IT>
__global__ void __launch_bounds__(128) iir_strided_rc_kernel(IT *__restrict__ im, int yn, int n, uint64_t stride,
                                                             uint64_t outer_stride, uint64_t nlines, IIRDev c,
                                                             unsigned *err_out, float2 *__restrict__ ckpt) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nlines) return;
    const uint64_t y = g % (uint64_t)yn, o = g / (uint64_t)yn;
    IT *L = im + o * outer_stride + y;
    unsigned err = 0, scratch_err = 0;
    float v1 = 0, v2 = 0, v3 = 0, v4 = 0;
    for (int i = 0; i < c.minLen; ++i) {
        float a = (float)L[(uint64_t)i * stride];
        float b = (float)L[(uint64_t)(n - 1 - i) * stride];
        v1 = v1 + __ldg(c.bc + i) * a;
        v2 = v2 + __ldg(c.bc + c.minLen + i) * a;
        v3 = v3 + __ldg(c.bc + 2 * c.minLen + i) * b;
        v4 = v4 + __ldg(c.bc + 3 * c.minLen + i) * b;
    }
    const int nseg = (n + kRC - 1) / kRC;
    // ---- causal sweep: the state at every segment start
    float p1 = v1, p2 = v2;
    for (int sgm = 0; sgm < nseg; ++sgm) {
        const int i0 = sgm * kRC;
        ckpt[(uint64_t)sgm * nlines + g] = make_float2(p1, p2);
        const IT *P = L + (uint64_t)i0 * stride;
        if (i0 >= 2 && i0 + kRC <= n) {
            float buf[kRC];
            const IT *q = P;
#pragma unroll
            for (int u = 0; u < kRC; ++u, q += stride) buf[u] = (float)*q;
#pragma unroll
            for (int u = 0; u < kRC; ++u) {
                const float nv = rnd_it<IT>(buf[u] + c.b1 * p1 + c.b2 * p2, scratch_err);
                p2 = p1;
                p1 = nv;
            }
        } else {
            const int i1 = min(n, i0 + kRC);
            for (int i = max(i0, 2); i < i1; ++i) {
                const float nv = rnd_it<IT>((float)L[(uint64_t)i * stride] + c.b1 * p1 + c.b2 * p2, scratch_err);
                p2 = p1;
                p1 = nv;
            }
        }
    }
    // ---- anti-causal sweep, recomputing each segment's causal values
    float q3 = v3, q4 = v4;
    for (int sgm = nseg - 1; sgm >= 0; --sgm) {
        const int i0 = sgm * kRC;
        const float2 st = ckpt[(uint64_t)sgm * nlines + g];
        float r1 = st.x, r2 = st.y;
        IT *P = L + (uint64_t)i0 * stride;
        if (i0 >= 2 && i0 + kRC <= n - 2) {
            float buf[kRC];
            const IT *q = P;
#pragma unroll
            for (int u = 0; u < kRC; ++u, q += stride) buf[u] = (float)*q;
#pragma unroll
            for (int u = 0; u < kRC; ++u) {
                const float nv = rnd_it<IT>(buf[u] + c.b1 * r1 + c.b2 * r2, err);
                r2 = r1;
                r1 = nv;
                buf[u] = nv;
            }
#pragma unroll
            for (int u = kRC - 1; u >= 0; --u) {
                const float temp = (buf[u] + c.b1 * q3 + c.b2 * q4);
                buf[u] = rnd_it<IT>(temp * c.norm, err);
                q4 = q3;
                q3 = temp;
            }
            IT *w = P;
#pragma unroll
            for (int u = 0; u < kRC; ++u, w += stride) *w = to_it<IT>(buf[u]);
        } else {
            const int i1 = min(n, i0 + kRC);
            float buf[kRC];
#pragma unroll
            for (int u = 0; u < kRC; ++u) {
                const int i = i0 + u;
                if (i >= i1) break;
                float f;
                if (i == 0) {
                    f = rnd_it<IT>(v2, err);
                } else if (i == 1) {
                    f = rnd_it<IT>(v1, err);
                } else {
                    f = rnd_it<IT>((float)P[(uint64_t)u * stride] + c.b1 * r1 + c.b2 * r2, err);
                    r2 = r1;
                    r1 = f;
                }
                buf[u] = f;
            }
#pragma unroll
            for (int u = kRC - 1; u >= 0; --u) {
                const int i = i0 + u;
                if (i >= i1) continue;
                float out;
                if (i == n - 1) {
                    out = rnd_it<IT>(v4 * c.norm, err);
                } else if (i == n - 2) {
                    out = rnd_it<IT>(v3 * c.norm, err);
                } else {
                    const float temp = (buf[u] + c.b1 * q3 + c.b2 * q4);
                    out = rnd_it<IT>(temp * c.norm, err);
                    q4 = q3;
                    q3 = temp;
                }
                buf[u] = out;
            }
#pragma unroll
            for (int u = 0; u < kRC; ++u)
                if (i0 + u < i1) P[(uint64_t)u * stride] = to_it<IT>(buf[u]);
        }
    }
    if (err) atomicAdd(err_out, err);
}

// V neighbouring lines (y .. y + V - 1) per thread, V = 2 or 4: the same
// recurrences as iir_strided_rc_kernel, each line's operations in the same
// order, with the V samples of a step moved as one 8- or 16-byte access, so
// that a block of 128 threads covers 128 V consecutive y of each plane (the
// longer contiguous runs per plane raise the DRAM efficiency of the strided
// access).  Needs yn a multiple of V and the image aligned to V samples.
template <typename IT, int V>
struct VecL;
template <>
struct VecL<float, 2> {
    __device__ __forceinline__ static void get(const float *p, float *a) {
        const float2 v = *reinterpret_cast<const float2 *>(p);
        a[0] = v.x;
        a[1] = v.y;
    }
    __device__ __forceinline__ static void put(float *p, const float *a) {
        *reinterpret_cast<float2 *>(p) = make_float2(a[0], a[1]);
    }
};
template <>
struct VecL<float, 4> {
    __device__ __forceinline__ static void get(const float *p, float *a) {
        const float4 v = *reinterpret_cast<const float4 *>(p);
        a[0] = v.x;
        a[1] = v.y;
        a[2] = v.z;
        a[3] = v.w;
    }
    __device__ __forceinline__ static void put(float *p, const float *a) {
        *reinterpret_cast<float4 *>(p) = make_float4(a[0], a[1], a[2], a[3]);
    }
};
template <>
struct VecL<uint16_t, 2> {
    __device__ __forceinline__ static void get(const uint16_t *p, float *a) {
        const ushort2 v = *reinterpret_cast<const ushort2 *>(p);
        a[0] = (float)v.x;
        a[1] = (float)v.y;
    }
    __device__ __forceinline__ static void put(uint16_t *p, const float *a) {
        *reinterpret_cast<ushort2 *>(p) = make_ushort2(to_it<uint16_t>(a[0]), to_it<uint16_t>(a[1]));
    }
};
template <>
struct VecL<uint16_t, 4> {
    __device__ __forceinline__ static void get(const uint16_t *p, float *a) {
        const ushort4 v = *reinterpret_cast<const ushort4 *>(p);
        a[0] = (float)v.x;
        a[1] = (float)v.y;
        a[2] = (float)v.z;
        a[3] = (float)v.w;
    }
    __device__ __forceinline__ static void put(uint16_t *p, const float *a) {
        *reinterpret_cast<ushort4 *>(p) = make_ushort4(to_it<uint16_t>(a[0]), to_it<uint16_t>(a[1]),
                                                       to_it<uint16_t>(a[2]), to_it<uint16_t>(a[3]));
    }
};

template <typename IT, int V>
__global__ void __launch_bounds__(128) iir_strided_rcv_kernel(IT *__restrict__ im, int yn, int n, uint64_t stride,
                                                              uint64_t outer_stride, uint64_t nlines, IIRDev c,
                                                              unsigned *err_out, float2 *__restrict__ ckpt) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;  // pair index
    const uint64_t hy = (uint64_t)(yn / V);
    if (g >= nlines / V) return;
    const uint64_t y = V * (g % hy), o = g / hy;
    const uint64_t line = V * g;  // o * yn + y
    IT *L = im + o * outer_stride + y;
    unsigned err = 0, scratch_err = 0;
    float v1[V] = {}, v2[V] = {}, v3[V] = {}, v4[V] = {};
    for (int i = 0; i < c.minLen; ++i) {
        float a[V], b[V];
        VecL<IT, V>::get(L + (uint64_t)i * stride, a);
        VecL<IT, V>::get(L + (uint64_t)(n - 1 - i) * stride, b);
        const float k1 = __ldg(c.bc + i), k2 = __ldg(c.bc + c.minLen + i);
        const float k3 = __ldg(c.bc + 2 * c.minLen + i), k4 = __ldg(c.bc + 3 * c.minLen + i);
#pragma unroll
        for (int h = 0; h < V; ++h) {
            v1[h] = v1[h] + k1 * a[h];
            v2[h] = v2[h] + k2 * a[h];
            v3[h] = v3[h] + k3 * b[h];
            v4[h] = v4[h] + k4 * b[h];
        }
    }
    const int nseg = (n + kRC - 1) / kRC;
    // ---- causal sweep: the state at every segment start
    float p1[V], p2[V];
#pragma unroll
    for (int h = 0; h < V; ++h) {
        p1[h] = v1[h];
        p2[h] = v2[h];
    }
    for (int sgm = 0; sgm < nseg; ++sgm) {
        const int i0 = sgm * kRC;
        float2 *ck = ckpt + (uint64_t)sgm * nlines + line;
#pragma unroll
        for (int h = 0; h < V; ++h) ck[h] = make_float2(p1[h], p2[h]);
        const IT *P = L + (uint64_t)i0 * stride;
        if (i0 >= 2 && i0 + kRC <= n) {
            float buf[kRC][V];
            const IT *q = P;
#pragma unroll
            for (int u = 0; u < kRC; ++u, q += stride) VecL<IT, V>::get(q, buf[u]);
#pragma unroll
            for (int u = 0; u < kRC; ++u)
#pragma unroll
                for (int h = 0; h < V; ++h) {
                    const float nv = rnd_it<IT>(buf[u][h] + c.b1 * p1[h] + c.b2 * p2[h], scratch_err);
                    p2[h] = p1[h];
                    p1[h] = nv;
                }
        } else {
            const int i1 = min(n, i0 + kRC);
            for (int i = max(i0, 2); i < i1; ++i) {
                float a[V];
                VecL<IT, V>::get(L + (uint64_t)i * stride, a);
#pragma unroll
                for (int h = 0; h < V; ++h) {
                    const float nv = rnd_it<IT>(a[h] + c.b1 * p1[h] + c.b2 * p2[h], scratch_err);
                    p2[h] = p1[h];
                    p1[h] = nv;
                }
            }
        }
    }
    // ---- anti-causal sweep, recomputing each segment's causal values
    float q3[V], q4[V];
#pragma unroll
    for (int h = 0; h < V; ++h) {
        q3[h] = v3[h];
        q4[h] = v4[h];
    }
    for (int sgm = nseg - 1; sgm >= 0; --sgm) {
        const int i0 = sgm * kRC;
        const float2 *ck = ckpt + (uint64_t)sgm * nlines + line;
        float r1[V], r2[V];
#pragma unroll
        for (int h = 0; h < V; ++h) {
            const float2 st = ck[h];
            r1[h] = st.x;
            r2[h] = st.y;
        }
        IT *P = L + (uint64_t)i0 * stride;
        if (i0 >= 2 && i0 + kRC <= n - 2) {
            float buf[kRC][V];
            const IT *q = P;
#pragma unroll
            for (int u = 0; u < kRC; ++u, q += stride) VecL<IT, V>::get(q, buf[u]);
#pragma unroll
            for (int u = 0; u < kRC; ++u)
#pragma unroll
                for (int h = 0; h < V; ++h) {
                    const float nv = rnd_it<IT>(buf[u][h] + c.b1 * r1[h] + c.b2 * r2[h], err);
                    r2[h] = r1[h];
                    r1[h] = nv;
                    buf[u][h] = nv;
                }
#pragma unroll
            for (int u = kRC - 1; u >= 0; --u)
#pragma unroll
                for (int h = 0; h < V; ++h) {
                    const float temp = (buf[u][h] + c.b1 * q3[h] + c.b2 * q4[h]);
                    buf[u][h] = rnd_it<IT>(temp * c.norm, err);
                    q4[h] = q3[h];
                    q3[h] = temp;
                }
            IT *w = P;
#pragma unroll
            for (int u = 0; u < kRC; ++u, w += stride) VecL<IT, V>::put(w, buf[u]);
        } else {
            const int i1 = min(n, i0 + kRC);
            float buf[kRC][V];
#pragma unroll
            for (int u = 0; u < kRC; ++u) {
                const int i = i0 + u;
                if (i >= i1) break;
                float a[V] = {};
                if (i >= 2) VecL<IT, V>::get(P + (uint64_t)u * stride, a);
#pragma unroll
                for (int h = 0; h < V; ++h) {
                    float f;
                    if (i == 0) {
                        f = rnd_it<IT>(v2[h], err);
                    } else if (i == 1) {
                        f = rnd_it<IT>(v1[h], err);
                    } else {
                        f = rnd_it<IT>(a[h] + c.b1 * r1[h] + c.b2 * r2[h], err);
                        r2[h] = r1[h];
                        r1[h] = f;
                    }
                    buf[u][h] = f;
                }
            }
#pragma unroll
            for (int u = kRC - 1; u >= 0; --u) {
                const int i = i0 + u;
                if (i >= i1) continue;
#pragma unroll
                for (int h = 0; h < V; ++h) {
                    float out;
                    if (i == n - 1) {
                        out = rnd_it<IT>(v4[h] * c.norm, err);
                    } else if (i == n - 2) {
                        out = rnd_it<IT>(v3[h] * c.norm, err);
                    } else {
                        const float temp = (buf[u][h] + c.b1 * q3[h] + c.b2 * q4[h]);
                        out = rnd_it<IT>(temp * c.norm, err);
                        q4[h] = q3[h];
                        q3[h] = temp;
                    }
                    buf[u][h] = out;
                }
            }
#pragma unroll
            for (int u = 0; u < kRC; ++u)
                if (i0 + u < i1) VecL<IT, V>::put(P + (uint64_t)u * stride, buf[u]);
        }
    }
    if (err) atomicAdd(err_out, err);
}

// The x / z pass over nlines lines of n samples: four or two lines per thread
// where y_num and the alignment allow, else one.
template <typename IT>
static void launch_strided_iir(IT *work, int yn, int n, uint64_t stride, uint64_t outer_stride, uint64_t nlines,
                               const IIRDev &c, unsigned *d_err, float2 *ck, cudaStream_t s) {
    const uintptr_t a = (uintptr_t)work;
    if (yn % 4 == 0 && a % (4 * sizeof(IT)) == 0)
        iir_strided_rcv_kernel<IT, 4><<<blocks_for(nlines / 4, 128), 128, 0, s>>>(work, yn, n, stride, outer_stride,
                                                                                 nlines, c, d_err, ck);
    else if (yn % 2 == 0 && a % (2 * sizeof(IT)) == 0)
        iir_strided_rcv_kernel<IT, 2><<<blocks_for(nlines / 2, 128), 128, 0, s>>>(work, yn, n, stride, outer_stride,
                                                                                 nlines, c, d_err, ck);
    else
        iir_strided_rc_kernel<IT><<<blocks_for(nlines, 128), 128, 0, s>>>(work, yn, n, stride, outer_stride, nlines,
                                                                        c, d_err, ck);
}

// Copy of the offset input when no smoothing runs (lambda <= 0 or y too short).
template <typename IT>
__global__ void offset_copy_kernel(const uint16_t *__restrict__ src, IT *__restrict__ dst, uint64_t n,
                                   const float *__restrict__ d_offset) {
    const float off = d_offset ? *d_offset : 0.0f;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] = to_it<IT>(raw_to_it<IT>(src[i], off));
}

// ---------------------------------------------------------------------------
// a3 + a4: calc_bspline_fd_ds_mag (ComputeGradient.hpp:976-1051) fused with
// downsample(sum, /8) (PixelData.hpp:916-967).  A CTA owns 8 x 64 ds cells in
// (x, y) and streams 8 ds slices in z through a 4-slice shared-memory ring of
// the full-resolution tile plus a one-sample halo, stored with the index
// clamping both reference functions use (replicate boundary).
// ---------------------------------------------------------------------------
// 4-byte asynchronous global -> shared copy (cp.async, sm_80+) and the wait
// for all of a thread's outstanding copies
__device__ __forceinline__ void cp_async4(float *smem, const float *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// waits until at most the most recently committed group is still in flight
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// ---------------------------------------------------------------------------
// a2 (y), recomputing form: the same recurrences as iir_y_kernel without the
// round trip of the causal values through memory.  The causal sweep keeps
// only the recurrence state at the start of every 64-sample tile (ckpt,
// [tile][line] pairs); the anti-causal sweep then walks the tiles from the
// end, recomputes each tile's causal values from its saved state and the
// input -- the same operations on the same values, so the same bits -- and
// runs the anti-causal recurrence over them.  Traffic per sample: the input
// read twice and the result written once (2 + 2 + 4 bytes for uint16 input
// and float ImageType) instead of 2 + 4 + 4 + 4.
// A warp (one per block) owns 32 lines; tiles arrive by cp.async one tile
// ahead of the arithmetic, every copy one aligned 32-bit word (two uint16
// samples) and a warp's copies one 128-byte run of a line: rows must start
// on 4 bytes, i.e. yn even.  The 64-sample tiles give 128-byte input and
// 256-byte output runs per line (the DRAM efficiency of the pass rises with
// the run length).
// ---------------------------------------------------------------------------
constexpr int kAY = 64;                         // samples per tile
constexpr int kAWords = 2 * 32 * 33 + 32 * 65;  // shared words per warp: two raw stages, the tile values
constexpr int kAWarps = 1;                       // warps per block
__device__ __forceinline__ void cp_async4w(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}

template <typename IT>
__global__ void __launch_bounds__(32 * kAWarps) iir_y_rc_kernel(const uint16_t *__restrict__ src, IT *__restrict__ dst, int yn,
                                                       uint64_t nlines, IIRDev c, const float *__restrict__ d_offset,
                                                       unsigned *err_out, float2 *__restrict__ ckpt) {
    __shared__ uint32_t smem_all[kAWarps][kAWords];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t line0 = ((uint64_t)blockIdx.x * kAWarps + w) * 32;
    if (line0 >= nlines) return;
    const uint64_t myline = line0 + lane;
    const bool valid = myline < nlines;
    const int nl = (int)min((uint64_t)32, nlines - line0);
    const float off = d_offset ? *d_offset : 0.0f;
    uint32_t *S = smem_all[w];
    uint32_t *U0 = S, *U1 = S + 32 * 33;                      // raw stages [2][32][33] words
    float *F = reinterpret_cast<float *>(S + 2 * 32 * 33);  // tile values [32][65]
    unsigned err = 0;

    float t1 = 0, t2 = 0, t3 = 0, t4 = 0;
    if (valid) {
        const uint16_t *L = src + myline * (uint64_t)yn;
        for (int k = 0; k < c.minLen; ++k) {
            float v = raw_to_it<IT>(L[k], off);
            t1 = t1 + __ldg(c.bc + k) * v;
            t2 = t2 + __ldg(c.bc + c.minLen + k) * v;
        }
        for (int k = 0; k < c.minLen; ++k) {
            float v = raw_to_it<IT>(L[yn - 1 - k], off);
            t3 = t3 + __ldg(c.bc + 2 * c.minLen + k) * v;
            t4 = t4 + __ldg(c.bc + 3 * c.minLen + k) * v;
        }
    }
    const int ntile = (yn + kAY - 1) / kAY;
    const uint16_t *src_w = src + line0 * (uint64_t)yn;
    auto issue = [&](int t, uint32_t *buf) {
#pragma unroll
        for (int h = 0; h < kAY / 64; ++h) {
            const int cw = lane + 32 * h;  // word of the line
            const int y = t * kAY + 2 * cw;
            if (y < yn) {
                const uint16_t *p = src_w + y;
                uint32_t *d = buf + cw;
#pragma unroll 4
                for (int jj = 0; jj < 32; ++jj, p += yn, d += 33)
                    if (jj < nl) cp_async4w(d, p);
            }
        }
        cp_async_commit();
    };
    auto sample = [&](const uint32_t *U, int k) -> float {
        const uint32_t wd = U[lane * 33 + (k >> 1)];
        return raw_to_it<IT>((uint16_t)((k & 1) ? (wd >> 16) : (wd & 0xffffu)), off);
    };

    // ---- causal sweep: the state at every tile start
    issue(0, U0);
    for (int t = 0; t < ntile; ++t) {
        const uint32_t *U = (t & 1) ? U1 : U0;
        if (t + 1 < ntile)
            issue(t + 1, (t & 1) ? U0 : U1);
        else
            cp_async_commit();
        cp_async_wait_one();
        __syncwarp();
        const int y0 = t * kAY;
        if (valid) {
            ckpt[(uint64_t)t * nlines + myline] = make_float2(t1, t2);
            if (y0 >= 2 && y0 + kAY <= yn) {
#pragma unroll
                for (int k = 0; k < kAY; ++k) {
                    const float temp = t1 * c.b1 + t2 * c.b2 + sample(U, k);
                    t2 = t1;
                    t1 = temp;
                }
            } else {
                const int kend = min(kAY, yn - y0);
                for (int k = 0; k < kend; ++k) {
                    if (y0 + k < 2) continue;
                    const float temp = t1 * c.b1 + t2 * c.b2 + sample(U, k);
                    t2 = t1;
                    t1 = temp;
                }
            }
        }
        __syncwarp();
    }

    // ---- anti-causal sweep, recomputing each tile's causal values
    float b2v = 0, b1v = 0;
    if (valid) {
        unsigned e0 = 0;
        b2v = rnd_it<IT>(t4 * c.norm, e0) / c.norm;
        b1v = rnd_it<IT>(t3 * c.norm, e0) / c.norm;
    }
    const int last = ntile - 1;
    issue(last, (last & 1) ? U1 : U0);
    for (int t = last; t >= 0; --t) {
        const uint32_t *U = (t & 1) ? U1 : U0;
        if (t > 0)
            issue(t - 1, (t & 1) ? U0 : U1);
        else
            cp_async_commit();
        cp_async_wait_one();
        __syncwarp();
        const int y0 = t * kAY;
        if (valid) {
            const float2 st = ckpt[(uint64_t)t * nlines + myline];
            float r1 = st.x, r2 = st.y;
            if (y0 >= 2 && y0 + kAY <= yn - 2) {
#pragma unroll
                for (int k = 0; k < kAY; ++k) {
                    const float temp = r1 * c.b1 + r2 * c.b2 + sample(U, k);
                    F[lane * 65 + k] = rnd_it<IT>(temp, err);
                    r2 = r1;
                    r1 = temp;
                }
#pragma unroll
                for (int k = kAY - 1; k >= 0; --k) {
                    const float temp = b1v * c.b1 + b2v * c.b2 + F[lane * 65 + k];
                    F[lane * 65 + k] = rnd_it<IT>(temp * c.norm, err);
                    b2v = b1v;
                    b1v = temp;
                }
            } else {
                const int kend = min(kAY, yn - y0);
                for (int k = 0; k < kend; ++k) {
                    const int y = y0 + k;
                    float out;
                    if (y == 0) {
                        out = store_cvt<IT>(r2);
                    } else if (y == 1) {
                        out = store_cvt<IT>(r1);
                    } else {
                        const float temp = r1 * c.b1 + r2 * c.b2 + sample(U, k);
                        out = rnd_it<IT>(temp, err);
                        r2 = r1;
                        r1 = temp;
                    }
                    if (y == yn - 2) out = rnd_it<IT>(t3 * c.norm, err);
                    if (y == yn - 1) out = rnd_it<IT>(t4 * c.norm, err);
                    F[lane * 65 + k] = out;
                }
                for (int k = kend - 1; k >= 0; --k) {
                    if (y0 + k > yn - 3) continue;
                    const float temp = b1v * c.b1 + b2v * c.b2 + F[lane * 65 + k];
                    F[lane * 65 + k] = rnd_it<IT>(temp * c.norm, err);
                    b2v = b1v;
                    b1v = temp;
                }
            }
        }
        __syncwarp();
#pragma unroll
        for (int h = 0; h < kAY / 32; ++h) {
            if (y0 + lane + 32 * h < yn) {
                IT *q = dst + line0 * (uint64_t)yn + y0 + lane + 32 * h;
#pragma unroll 4
                for (int j = 0; j < nl; ++j, q += yn) *q = to_it<IT>(F[j * 65 + lane + 32 * h]);
            }
        }
        __syncwarp();
    }
    if (err) atomicAdd(err_out, err);
}

// 8 x 60 ds cells per plane step: tile columns start four samples before
// 2 * yd0 so that rows split into aligned 16-byte pieces, and six slots of
// 18 x 128 floats let four blocks share an SM
constexpr int kGX = 8, kGY = 60, kGZ = 8, kGThreads = 256, kGSlots = 6;
constexpr int kTX = 2 * kGX + 2, kTY = 2 * kGY + 8;
constexpr size_t kGradSmem = sizeof(float) * kGSlots * kTX * kTY;

__device__ __forceinline__ void cp_async16(float *smem, const float *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

// PW2: every 2h is a power of two, so dividing by it is the exact multiply by
// its reciprocal (both round the same real number once).  VEC (float
// ImageType, yn a multiple of 4, 16-byte aligned image): tile rows arrive in
// 16-byte copies.
template <typename IT, bool PW2, bool VEC>
__global__ void __launch_bounds__(kGThreads, 4) grad_ds_kernel(const IT *__restrict__ im, int yn, int xn, int zn,
                                                            IT *__restrict__ grad, float *__restrict__ ids, int yd,
                                                            int xd, int zd, float hx, float hy, float hz) {
    // six plane slots: the four planes a step reads and the two the next
    // step needs, which (ImageType float) arrive by cp.async during the step
    extern __shared__ float grad_smem[];
    float(*ring)[kTX][kTY] = reinterpret_cast<float(*)[kTX][kTY]>(grad_smem);
    const int yd0 = blockIdx.x * kGY, xd0 = blockIdx.y * kGX, zd0 = blockIdx.z * kGZ;
    const int zd1 = min(zd0 + kGZ, zd);
    const int xf0 = 2 * xd0 - 1, yf0 = 2 * yd0 - 4;
    const float hx2 = 2 * hx, hy2 = 2 * hy, hz2 = 2 * hz;
    const float ihx2 = 1.0f / hx2, ihy2 = 1.0f / hy2, ihz2 = 1.0f / hz2;
    constexpr bool kAsync = std::is_same<IT, float>::value;  // 4-byte elements copy asynchronously

    // a thread fills the same (clamped) tile positions t = threadIdx.x + k *
    // kGThreads of every plane: their in-plane source offsets once
    constexpr int kLoads = VEC ? 1 : (kTX * kTY + kGThreads - 1) / kGThreads;
    uint64_t src_off[kLoads];
    if (!VEC) {
#pragma unroll
        for (int k = 0; k < kLoads; ++k) {
            const int t = threadIdx.x + k * kGThreads;
            const int r = t / kTY, cc = t % kTY;
            const int xg = min(max(xf0 + r, 0), xn - 1), yg = min(max(yf0 + cc, 0), yn - 1);
            src_off[k] = (uint64_t)xg * (uint64_t)yn + (uint64_t)yg;
        }
    }
    auto load = [&](int zf) {  // zf >= -1
        float *S = &ring[(zf + kGSlots) % kGSlots][0][0];
        const int zc = min(max(zf, 0), zn - 1);
        const IT *plane = im + (uint64_t)zc * (uint64_t)xn * (uint64_t)yn;
        if (VEC) {
            constexpr int kQ = kTY / 4;  // 16-byte pieces per row
            for (int ci = threadIdx.x; ci < kTX * kQ; ci += kGThreads) {
                const int r = ci / kQ, q = ci % kQ;
                const int xg = min(max(xf0 + r, 0), xn - 1), yg = yf0 + 4 * q;
                const float *row = reinterpret_cast<const float *>(plane) + (uint64_t)xg * (uint64_t)yn;
                float *d = S + r * kTY + 4 * q;
                if (yg >= 0 && yg + 3 < yn) {
                    cp_async16(d, row + yg);
                } else {
#pragma unroll
                    for (int e = 0; e < 4; ++e) cp_async4(d + e, row + min(max(yg + e, 0), yn - 1));
                }
            }
        } else {
#pragma unroll
            for (int k = 0; k < kLoads; ++k) {
                const int t = threadIdx.x + k * kGThreads;
                if (t < kTX * kTY) {
                    if (kAsync)
                        cp_async4(S + t, reinterpret_cast<const float *>(plane) + src_off[k]);
                    else
                        S[t] = (float)plane[src_off[k]];
                }
            }
        }
    };
    // squared gradient magnitude at full-res (zf, xf, yf) of plane C with
    // neighbour planes U, D: the reference's double sum of the squared float
    // differences, gx^2 + gz^2 then + gy^2.  Each square of a float is exact
    // in double, so the fused forms round exactly where the sums do.
    auto gsq = [&](float cxm, float cxp, float cym, float cyp, float u, float d) -> double {
        float gx, gz, gy;
        if (PW2) {
            gx = (cxp - cxm) * ihx2;
            gz = (d - u) * ihz2;
            gy = (cyp - cym) * ihy2;
        } else {
            gx = (cxp - cxm) / hx2;
            gz = (d - u) / hz2;
            gy = (cyp - cym) / hy2;
        }
        const double s = fma((double)gx, (double)gx, (double)gz * (double)gz);
        return fma((double)gy, (double)gy, s);
    };

    // the (at most two) ds cells of this thread in every plane step: tile row
    // and column of their full-res corner (x0, y0 = 2k), whether y0 + 1 and
    // x0 + 1 lie inside the volume (else the child is clamped onto y0 / x0),
    // and their output offset in plane 0
    constexpr int kCells = (kGX * kGY + kGThreads - 1) / kGThreads;
    bool cell_in[kCells];
    int cell_rx[kCells], cell_cy[kCells], cell_flags[kCells];
    uint64_t cell_o[kCells];
#pragma unroll
    for (int q = 0; q < kCells; ++q) {
        const int t = threadIdx.x + q * kGThreads;
        const int xl = t / kGY, yl = t % kGY;
        const int xk = xd0 + xl, k = yd0 + yl;
        cell_in[q] = t < kGX * kGY && xk < xd && k < yd;
        cell_rx[q] = 2 * xk - xf0;
        cell_cy[q] = 2 * k - yf0;
        cell_flags[q] = (2 * k + 1 < yn ? 1 : 0) | (2 * xk + 1 < xn ? 2 : 0);
        cell_o[q] = idx3(k, xk, 0, yd, xd);
    }
    load(2 * zd0 - 1);
    load(2 * zd0);
    if (kAsync) {
        load(2 * zd0 + 1);
        load(2 * zd0 + 2);
        cp_async_wait_all();
    }
    for (int z = zd0; z < zd1; ++z) {
        if (kAsync) {
            __syncthreads();
            if (z + 1 < zd1) {  // the next step's planes arrive while this step computes
                load(2 * z + 3);
                load(2 * z + 4);
            }
        } else {
            load(2 * z + 1);
            load(2 * z + 2);
            __syncthreads();
        }
        const int z0 = 2 * z;
        const bool z1in = z0 + 1 < zn;
        const float(*P0)[kTY] = ring[(z0 - 1 + kGSlots) % kGSlots];
        const float(*P1)[kTY] = ring[(z0 + kGSlots) % kGSlots];
        const float(*P2)[kTY] = ring[(z0 + 1 + kGSlots) % kGSlots];
        const float(*P3)[kTY] = ring[(z0 + 2 + kGSlots) % kGSlots];
#pragma unroll
        for (int q = 0; q < kCells; ++q) {
            if (!cell_in[q]) continue;
            const int rx = cell_rx[q], cy = cell_cy[q];
            const bool y1in = (cell_flags[q] & 1) != 0, x1in = (cell_flags[q] & 2) != 0;
            // cy is even: the samples come in aligned pairs (y, y + 1)
            auto ld2 = [](const float *q) { return *reinterpret_cast<const float2 *>(q); };
            struct Nb {
                float2 m, p;          // rows rx - 1 and rx + 2 at (cy, cy + 1)
                float2 a0, a1, a2;    // row rx at cy - 2, cy, cy + 2
                float2 b0, b1, b2;    // row rx + 1
            };
            auto nb = [&](const float(*P)[kTY]) {
                Nb q;
                q.m = ld2(&P[rx - 1][cy]);
                q.p = ld2(&P[rx + 2][cy]);
                q.a0 = ld2(&P[rx][cy - 2]);
                q.a1 = ld2(&P[rx][cy]);
                q.a2 = ld2(&P[rx][cy + 2]);
                q.b0 = ld2(&P[rx + 1][cy - 2]);
                q.b1 = ld2(&P[rx + 1][cy]);
                q.b2 = ld2(&P[rx + 1][cy + 2]);
                return q;
            };
            const Nb n1 = nb(P1), n2 = nb(P2);
            float gmax = 0.0f;
            if (yn >= 2) {
                // the gradient magnitude is max over the 2 x 2 x 2 children; the
                // conversion sqrt -> ImageType is monotone (below 2^16 for
                // uint16), so the max is taken over the squares and rooted once
                const float2 u0a = ld2(&P0[rx][cy]), u0b = ld2(&P0[rx + 1][cy]);
                const float2 d3a = ld2(&P3[rx][cy]), d3b = ld2(&P3[rx + 1][cy]);
                // children of plane C with neighbour planes U (rows rx, rx + 1)
                // and D: (x, y) = (rx, cy) (rx, cy+1) (rx+1, cy) (rx+1, cy+1)
                auto children = [&](const Nb &C, float2 ua, float2 ub, float2 da, float2 db, auto &&f) {
                    f(gsq(C.m.x, C.b1.x, C.a0.y, C.a1.y, ua.x, da.x));
                    if (y1in) f(gsq(C.m.y, C.b1.y, C.a1.x, C.a2.x, ua.y, da.y));
                    if (x1in) {
                        f(gsq(C.a1.x, C.p.x, C.b0.y, C.b1.y, ub.x, db.x));
                        if (y1in) f(gsq(C.a1.y, C.p.y, C.b1.x, C.b2.x, ub.y, db.y));
                    }
                };
                auto all = [&](auto &&f) {
                    children(n1, u0a, u0b, n2.a1, n2.b1, f);
                    if (z1in) children(n2, n1.a1, n1.b1, d3a, d3b, f);
                };
                double smax = 0.0;  // every square is >= 0
                auto upd = [&](double q) { smax = q > smax ? q : smax; };
                if (y1in && x1in) {
                    // away from the volume's y / x end every child exists:
                    // straight-line code (the maximum is order-independent)
                    auto four = [&](const Nb &C, float2 ua, float2 ub, float2 da, float2 db) {
                        upd(gsq(C.m.x, C.b1.x, C.a0.y, C.a1.y, ua.x, da.x));
                        upd(gsq(C.m.y, C.b1.y, C.a1.x, C.a2.x, ua.y, da.y));
                        upd(gsq(C.a1.x, C.p.x, C.b0.y, C.b1.y, ub.x, db.x));
                        upd(gsq(C.a1.y, C.p.y, C.b1.x, C.b2.x, ub.y, db.y));
                    };
                    four(n1, u0a, u0b, n2.a1, n2.b1);
                    if (z1in) four(n2, n1.a1, n1.b1, d3a, d3b);
                } else {
                    all(upd);
                }
                if (sizeof(IT) == 4 || smax < 4294967296.0) {
                    const double root = sqrt(smax);
                    gmax = sizeof(IT) == 2 ? cvt_u16d(root) : (float)root;
                } else {
                    // roots of 2^16 and above wrap in the uint16 conversion
                    all([&](double q) {
                        const float v = cvt_u16d(sqrt(q));
                        gmax = v > gmax ? v : gmax;
                    });
                }
            }
            const uint64_t o = cell_o[q] + (uint64_t)z * (uint64_t)xd * (uint64_t)yd;
            grad[o] = to_it<IT>(gmax);
            // mean with the clamped indices of downsample (held by the tile)
            float s = n1.a1.x;
            s = s + n1.a1.y;
            s = s + n1.b1.x;
            s = s + n1.b1.y;
            s = s + n2.a1.x;
            s = s + n2.a1.y;
            s = s + n2.b1.x;
            s = s + n2.b1.y;
            ids[o] = s * 0.125f;  // == s / 8 exactly
        }
        if (kAsync) cp_async_wait_all();
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// a5: calc_inv_bspline_y/x/z (ComputeGradient.hpp:785-964).  A block owns an
// 8 (x) x 256 (y) column of the ds image and a run of up to 32 planes, and
// streams along z; a thread owns one y of the column.  Each input plane (with
// a one-sample x / y halo) arrives by cp.async two planes ahead; the thread
// runs the y pass of its y on the ten rows, the x pass of the eight outputs
// from those, and the z pass from the last three planes it holds in
// registers, so a plane costs one block barrier.  Each value is the
// reference's expression with its operand order, so the columns reproduce
// the whole-volume passes exactly.
// ---------------------------------------------------------------------------
constexpr int kJX = 8, kJY = 256, kJZ = 32;
constexpr int kJXH = kJX + 2, kJYH = kJY + 2;

__global__ void __launch_bounds__(kJY) inv_bspline_kernel(const float *__restrict__ in, float *__restrict__ O, int yd,
                                                          int xd, int zd, int ony, int onx, int onz, InvB c) {
    __shared__ float S[3][kJXH][kJYH];  // input planes with halo, two ahead
    const int y0 = blockIdx.x * kJY, x0 = blockIdx.y * kJX, zs = blockIdx.z * kJZ;
    const int ze = min(zs + kJZ, zd);
    const int zb = zs == 0 ? 0 : zs - 1;            // first plane read
    const int zl = onz ? min(ze, zd - 1) : ze - 1;  // last plane read
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    auto issue = [&](int zi) {
        if (zi <= zl) {
            float(*B)[kJYH] = S[(zi - zb) % 3];
            for (int r = 0; r < kJXH; ++r) {
                const int xg = x0 - 1 + r;
                if (xg < 0 || xg >= xd) continue;
                const float *row = in + idx3(0, xg, zi, yd, xd);
                for (int yy = threadIdx.x; yy < kJYH; yy += kJY) {
                    const int yg = y0 - 1 + yy;
                    if (yg >= 0 && yg < yd) cp_async4(&B[r][yy], row + yg);
                }
            }
        }
        cp_async_commit();
    };
    (void)warp;
    (void)lane;
    const int y = y0 + threadIdx.x;
    const bool yin = y < yd;
    // the thread's x-pass values of planes zi - 2, zi - 1, zi
    float p2[kJX], p1[kJX], p0[kJX];
#pragma unroll
    for (int i = 0; i < kJX; ++i) p2[i] = p1[i] = p0[i] = 0.0f;
    issue(zb);
    issue(zb + 1);
    for (int zi = zb; zi <= zl; ++zi) {
        cp_async_wait_one();
        __syncthreads();
        issue(zi + 2);  // into the buffer of plane zi - 1, read before the barrier
        const float(*B)[kJYH] = S[(zi - zb) % 3];
#pragma unroll
        for (int i = 0; i < kJX; ++i) {
            p2[i] = p1[i];
            p1[i] = p0[i];
        }
        if (yin) {
            // y pass of the ten rows at this y
            float yb[kJXH];
#pragma unroll
            for (int r = 0; r < kJXH; ++r) {
                const int xg = x0 - 1 + r;
                const float *Sr = &B[r][0] + 1 - y0;  // [global y]
                float v = 0.0f;
                if (xg >= 0 && xg < xd) {
                    if (!ony)
                        v = Sr[y];
                    else if (y == 0)
                        v = c.a2 * Sr[0] + c.a13 * Sr[1];
                    else if (y == yd - 1)
                        v = c.a13 * Sr[yd - 2] + c.a2 * Sr[yd - 1];
                    else
                        v = c.a1 * Sr[y - 1] + c.a2 * Sr[y] + c.a3 * Sr[y + 1];
                }
                yb[r] = v;
            }
            // x pass of the eight outputs
#pragma unroll
            for (int i = 0; i < kJX; ++i) {
                const int x = x0 + i;
                float v = 0.0f;
                if (x < xd) {
                    if (!onx) {
                        v = yb[i + 1];
                    } else if (x == xd - 1) {
                        v = c.a13 * yb[i] + c.a2 * yb[i + 1];
                    } else if (x == 0) {
                        v = c.a1 * yb[2] + c.a2 * yb[1] + c.a3 * yb[2];
                    } else {
                        v = c.a1 * yb[i] + c.a2 * yb[i + 1] + c.a3 * yb[i + 2];
                    }
                }
                p0[i] = v;
            }
            // z pass of the planes now complete
            auto emit = [&](int z, const float *xm, const float *xc, const float *xp, bool last) {
#pragma unroll
                for (int i = 0; i < kJX; ++i) {
                    const int x = x0 + i;
                    if (x >= xd) continue;
                    float r;
                    if (!onz)
                        r = xc[i];
                    else if (last)
                        r = c.a13 * xm[i] + c.a2 * xc[i];
                    else
                        r = c.a1 * xm[i] + c.a2 * xc[i] + c.a3 * xp[i];
                    O[idx3(y, x, z, yd, xd)] = r;
                }
            };
            if (!onz) {
                if (zi >= zs) emit(zi, p0, p0, p0, false);
            } else {
                const int z = zi - 1;
                if (z >= zs) {
                    if (z == zd - 1)
                        emit(z, p2, p1, p0, true);
                    else if (z == 0)
                        emit(z, p0, p1, p0, false);  // zm = 1 = zi
                    else
                        emit(z, p2, p1, p0, false);
                }
                if (zi == zd - 1 && zi >= zs) emit(zi, p1, p0, p0, true);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// a6: local intensity scale (LocalIntensityScale.hpp:26-150) on the
// reflect-padded ds image (paddPixels, PixelData.hpp:1071-1178).
// ---------------------------------------------------------------------------
__global__ void pad_reflect_kernel(const float *__restrict__ in, int yn, int xn, int zn, float *__restrict__ out,
                                   int sy, int sx, int sz, int py, int px, int pz) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (uint64_t)py * px * pz) return;
    int y = (int)(g % py), x = (int)((g / py) % px), z = (int)(g / ((uint64_t)py * px));
    int ry = y - sy, rx = x - sx, rz = z - sz;
    ry = ry < 0 ? -ry : (ry > yn - 1 ? 2 * (yn - 1) - ry : ry);
    rx = rx < 0 ? -rx : (rx > xn - 1 ? 2 * (xn - 1) - rx : rx);
    rz = rz < 0 ? -rz : (rz > zn - 1 ? 2 * (zn - 1) - rz : rz);
    out[g] = in[idx3(ry, rx, rz, yn, xn)];
}

// Output i of the y box mean (calc_sat_mean_y, LocalIntensityScale.hpp:
// 311-362) from the quotients qm = C[i-off-1] / d and qp = C[i+off] / d of the
// cumulative sums (each the correctly rounded quotient, and -cm / d ==
// -(cm / d) exactly) and the last sum C[n-1]: the edge windows rescaled as
// the reference does.
template <int OFF>
__device__ __forceinline__ float sat_y_value_q(int i, int n, float d, float qm, float qp, float clast) {
    float v = (i <= OFF) ? 0.0f : -qm;
    if (i < n - OFF) v = v + qp;
    if (i >= n - OFF) {
        float cnt = (float)(i - (n - OFF) + 1);
        v = v * d;
        v = v + clast;
        v = (float)((double)v * (1.0 / (double)(d - cnt)));
    }
    if (i >= 1 && i <= OFF) v = (float)((double)v * ((double)d / ((double)i + (double)OFF + 1.0)));
    if (i == 0) v = (float)((double)v * ((double)d / ((double)OFF + 1.0)));
    return v;
}

// Reads of the padded image folded into the first y pass: padded (y, x, z)
// maps to the unpadded image by reflection about the edge sample (paddPixels,
// PixelData.hpp:1071-1178).  on_in maps the input, on_ref the |in - ref| operand.
struct PadMap {
    int on_in, on_ref;
    int sy, sx, sz, yd, xd, zd, px;
};

__device__ __forceinline__ int reflect101(int i, int n) { return i < 0 ? -i : (i > n - 1 ? 2 * (n - 1) - i : i); }

// y box mean: one thread per y-line, the cumulative sum carried in a register
// and the quotients of the last 2*OFF+2 sums in a register shift window; REF
// makes the input |in - ref| (calc_abs_diff, :188-196) on the fly.  The
// samples are staged by cp.async one tile ahead of the recurrence: a warp
// owns 32 lines and walks them in tiles of kSY samples, so no registers hold
// the prefetch and more warps stay resident.
// 32-sample tiles (a warp's copies and stores are 128-byte runs of a line),
// one warp per block.
// In tiles that touch neither end of the line the recurrence runs fully
// unrolled (the window shift becomes register renaming).  REF: the input is
// |in - ref| (the second pass of each window).
constexpr int kSY = 32;
constexpr int kSW = 1;                         // warps per block
constexpr int kSH = kSY >= 32 ? kSY / 32 : 1;   // y samples per lane and line in a copy
constexpr int kLPI = kSY >= 32 ? 1 : 32 / kSY;  // lines per warp copy instruction

template <int OFF, bool REF>
__global__ void __launch_bounds__(32 * kSW) sat_y_async_kernel(const float *__restrict__ in,
                                                               const float *__restrict__ ref, float *__restrict__ out,
                                                               int n, uint64_t nlines, PadMap pm) {
    constexpr int W = 2 * OFF + 2;
    constexpr int NB = REF ? 2 : 1;
    __shared__ float sm[kSW][2][NB][32][kSY + 1];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t line0 = ((uint64_t)blockIdx.x * kSW + w) * 32;
    if (line0 >= nlines) return;
    const bool valid = line0 + lane < nlines;
    const float d = (float)(2 * OFF + 1);
    const bool refl = pm.on_in | pm.on_ref;
    uint64_t mbase = 0;
    if (refl && valid) {
        const uint64_t ln = line0 + lane;
        const int xp = (int)(ln % (uint64_t)pm.px), zp = (int)(ln / (uint64_t)pm.px);
        mbase = idx3(0, reflect101(xp - pm.sx, pm.xd), reflect101(zp - pm.sz, pm.zd), pm.yd, pm.xd);
    }
    // copy / store mapping: a warp instruction moves kLPI lines of
    // min(kSY, 32) samples
    const int cy0 = kSY < 32 ? (lane & (kSY - 1)) : lane, cj = kSY < 32 ? lane / kSY : 0;
    const int ntile = (n + kSY - 1) / kSY;
    const float rd = __frcp_rn(d);
    auto issue = [&](int t, int b) {
#pragma unroll
        for (int h = 0; h < kSH; ++h) {
            const int cy = cy0 + 32 * h;
            const int y = t * kSY + cy;
            const int my = (refl && y < n) ? reflect101(y - pm.sy, pm.yd) : 0;
            const float *pa = in + (line0 + cj) * (uint64_t)n + y;  // unreflected source of line cj
            const float *ra = REF ? ref + (line0 + cj) * (uint64_t)n + y : nullptr;
            const uint64_t step = kLPI * (uint64_t)n;
#pragma unroll 2
            for (int jj = 0; jj < 32 / kLPI; ++jj, pa += step, ra += REF ? step : 0) {
                const int j = kLPI * jj + cj;
                const uint64_t bj = __shfl_sync(0xffffffffu, mbase, j);
                if (line0 + j < nlines && y < n) {
                    const uint64_t am = bj + (uint64_t)my;
                    cp_async4(&sm[w][b][0][j][cy], pm.on_in ? in + am : pa);
                    if (REF) cp_async4(&sm[w][b][NB - 1][j][cy], pm.on_ref ? ref + am : ra);
                }
            }
        }
        cp_async_commit();
    };
    // quotients C / d of the last W cumulative sums: the window's older end
    // divided once, when it was the newest
    float qr[W];
#pragma unroll
    for (int q = 0; q < W; ++q) qr[q] = 0.0f;
    float C = 0.0f;
    issue(0, 0);
    for (int t = 0; t < ntile; ++t) {
        const int b = t & 1;
        if (t + 1 < ntile)
            issue(t + 1, b ^ 1);
        else
            cp_async_commit();
        cp_async_wait_one();
        __syncwarp();
        float(*T)[kSY + 1] = sm[w][b][0];
        float(*R)[kSY + 1] = sm[w][b][NB - 1];
        const int y0 = t * kSY;
        if (valid) {
            if (y0 > 2 * OFF && y0 + kSY <= n) {
#pragma unroll
                for (int k = 0; k < kSY; ++k) {
                    float v = T[lane][k];
                    if (REF) v = fabsf(v - R[lane][k]);
                    C = C + v;
                    const float qn = div_const(C, d, rd);
#pragma unroll
                    for (int q = 0; q < W - 1; ++q) qr[q] = qr[q + 1];
                    qr[W - 1] = qn;
                    T[lane][k] = -qr[0] + qn;
                }
            } else {
                const int kend = min(kSY, n - y0);
                for (int k = 0; k < kend; ++k) {
                    float v = T[lane][k];
                    if (REF) v = fabsf(v - R[lane][k]);
                    C = C + v;
                    const float qn = div_const(C, d, rd);
#pragma unroll
                    for (int q = 0; q < W - 1; ++q) qr[q] = qr[q + 1];
                    qr[W - 1] = qn;
                    const int i = y0 + k - OFF;
                    if (i >= 0 && i < n - OFF) T[lane][k] = sat_y_value_q<OFF>(i, n, d, qr[0], qn, 0.0f);
                }
            }
        }
        __syncwarp();
#pragma unroll
        for (int h = 0; h < kSH; ++h) {
            const int cy = cy0 + 32 * h;
            const int yy = y0 + cy, i = yy - OFF;
            if (yy < n && i >= 0 && i < n - OFF) {
                float *q = out + (line0 + cj) * (uint64_t)n + i;
                const uint64_t step = kLPI * (uint64_t)n;
#pragma unroll 4
                for (int jj = 0; jj < 32 / kLPI; ++jj, q += step)
                    if (line0 + kLPI * jj + cj < nlines) *q = T[kLPI * jj + cj][cy];
            }
        }
        __syncwarp();
    }
    if (valid) {
        for (int i = n - OFF; i < n; ++i) {
            if (i < 0) continue;
            const int back = (n - 1) - (i - OFF - 1);
            float qm = 0.0f;
#pragma unroll
            for (int q = 0; q < W; ++q)
                if (q == W - 1 - back) qm = qr[q];
            out[(line0 + lane) * (uint64_t)n + i] = sat_y_value_q<OFF>(i, n, d, qm, 0.0f, C);
        }
    }
}

// Final pass writing the unpadded window times the rescale factor
// (unpaddPixels + rescale_var, LocalIntensityScale.hpp:174-184) directly.
struct LisOut {
    float *out;
    int sy, sx, sz, yd, xd, zd, axis;
    float rescale;
};

// x / z box mean (:364-494): one thread per strided line, a warp takes 32
// lines of adjacent y.  The samples come through shared memory in chunks of
// 32 (32 coalesced loads in flight per warp); each lane then runs its line's
// recurrence over the chunk in order.
template <int OFF, bool FINAL>
__global__ void __launch_bounds__(128) sat_strided_kernel(const float *__restrict__ in,
                                                          const float *__restrict__ absdiff_ref,
                                                          float *__restrict__ out, int yn, int n, uint64_t stride,
                                                          uint64_t outer_stride, uint64_t nlines, LisOut fo) {
    constexpr int W = 2 * OFF + 2;
    __shared__ float tile[4][32][33];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t g0 = g - lane;  // first line of the warp
    if (g0 >= nlines) return;
    const bool valid = g < nlines;
    const uint64_t y = valid ? g % (uint64_t)yn : 0, o = valid ? g / (uint64_t)yn : 0;
    const uint64_t base = o * outer_stride + y;
    auto emit = [&](int i, float v) {
        if (!FINAL) {
            out[base + (uint64_t)i * stride] = v;
            return;
        }
        const int xpad = fo.axis == 1 ? i : (int)o, zpad = fo.axis == 1 ? (int)o : i;
        const int uy = (int)y - fo.sy, ux = xpad - fo.sx, uz = zpad - fo.sz;
        if (uy >= 0 && uy < fo.yd && ux >= 0 && ux < fo.xd && uz >= 0 && uz < fo.zd)
            fo.out[idx3(uy, ux, uz, fo.yd, fo.xd)] = v * fo.rescale;
    };
    float c[W];
#pragma unroll
    for (int q = 0; q < W; ++q) c[q] = 0.0f;
    float C = 0.0f;
    const float dd = (float)(2 * OFF + 1), rdd = __frcp_rn(dd);
    for (int j0 = 0; j0 < n; j0 += 32) {
        const int m = min(32, n - j0);
        // lane l loads sample j0 + k of its own line for k < m (coalesced over
        // the warp's lines), stored transposed: tile[k][lane]; whole chunks
        // keep eight loads in flight per thread
        if (valid && m == 32) {
            const float *p = in + base + (uint64_t)j0 * stride;
            const float *q = absdiff_ref ? absdiff_ref + base + (uint64_t)j0 * stride : nullptr;
#pragma unroll 1
            for (int k0 = 0; k0 < 32; k0 += 8) {
                float v[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) v[u] = p[(uint64_t)(k0 + u) * stride];
                if (q) {
#pragma unroll
                    for (int u = 0; u < 8; ++u) v[u] = fabsf(v[u] - q[(uint64_t)(k0 + u) * stride]);
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) tile[w][k0 + u][lane] = v[u];
            }
        } else if (valid) {
            for (int k = 0; k < m; ++k) {
                const uint64_t a = base + (uint64_t)(j0 + k) * stride;
                float v = in[a];
                if (absdiff_ref) v = fabsf(v - absdiff_ref[a]);
                tile[w][k][lane] = v;
            }
        }
        __syncwarp();
        if (valid) {
            for (int k = 0; k < m; ++k) {
                const int j = j0 + k;
                const float v = tile[w][k][lane];
                C = (j == 0) ? v : v + C;
#pragma unroll
                for (int q = 0; q < W - 1; ++q) c[q] = c[q + 1];
                c[W - 1] = C;
                const int i = j - OFF;
                if (i >= 0) {
                    if (i < OFF + 1)
                        emit(i, C / (float)(i + OFF + 1));
                    else if (i < n - OFF)
                        emit(i, div_const(C - c[0], dd, rdd));
                }
            }
        }
        __syncwarp();
    }
    if (!valid) return;
    for (int i = n - OFF; i < n; ++i) {
        if (i < 0) continue;
        const int back = (n - 1) - (i - OFF - 1);
        float cm = 0.0f;
#pragma unroll
        for (int q = 0; q < W; ++q)
            if (q == W - 1 - back) cm = c[q];
        emit(i, (C - cm) / (float)(n - i + OFF));
    }
}

// The x / z box mean with V neighbouring lines (y .. y + V - 1) per thread:
// each line's recurrence and divisions exactly as in sat_strided_kernel, the
// V samples of a step moved as one access (longer runs per plane), eight
// steps of loads in flight.  Needs yn a multiple of V (used with V = 2: the
// padded y extent is even whenever the image's is).
template <int OFF, bool FINAL, int V>
__global__ void __launch_bounds__(128) sat_stridedv_kernel(const float *__restrict__ in,
                                                           const float *__restrict__ absdiff_ref,
                                                           float *__restrict__ out, int yn, int n, uint64_t stride,
                                                           uint64_t outer_stride, uint64_t nlines, LisOut fo) {
    constexpr int W = 2 * OFF + 2;
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t hy = (uint64_t)(yn / V);
    if (g >= nlines / V) return;
    const uint64_t y = V * (g % hy), o = g / hy;
    const uint64_t base = o * outer_stride + y;
    auto emit = [&](int i, const float *v) {
        if (!FINAL) {
            VecL<float, V>::put(out + base + (uint64_t)i * stride, v);
            return;
        }
        const int xpad = fo.axis == 1 ? i : (int)o, zpad = fo.axis == 1 ? (int)o : i;
        const int ux = xpad - fo.sx, uz = zpad - fo.sz;
        if (ux < 0 || ux >= fo.xd || uz < 0 || uz >= fo.zd) return;
#pragma unroll
        for (int h = 0; h < V; ++h) {
            const int uy = (int)y + h - fo.sy;
            if (uy >= 0 && uy < fo.yd) fo.out[idx3(uy, ux, uz, fo.yd, fo.xd)] = v[h] * fo.rescale;
        }
    };
    float c[V][W], C[V];
#pragma unroll
    for (int h = 0; h < V; ++h) {
        C[h] = 0.0f;
#pragma unroll
        for (int q = 0; q < W; ++q) c[h][q] = 0.0f;
    }
    const float dd = (float)(2 * OFF + 1), rdd = __frcp_rn(dd);
    for (int j0 = 0; j0 < n; j0 += 8) {
        const int m = min(8, n - j0);
        float v[8][V];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            if (u < m) {
                const uint64_t a = base + (uint64_t)(j0 + u) * stride;
                VecL<float, V>::get(in + a, v[u]);
                if (absdiff_ref) {
                    float r[V];
                    VecL<float, V>::get(absdiff_ref + a, r);
#pragma unroll
                    for (int h = 0; h < V; ++h) v[u][h] = fabsf(v[u][h] - r[h]);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            if (u >= m) break;
            const int j = j0 + u;
#pragma unroll
            for (int h = 0; h < V; ++h) {
                C[h] = (j == 0) ? v[u][h] : v[u][h] + C[h];
#pragma unroll
                for (int q = 0; q < W - 1; ++q) c[h][q] = c[h][q + 1];
                c[h][W - 1] = C[h];
            }
            const int i = j - OFF;
            if (i >= 0) {
                float e[V];
                if (i < OFF + 1) {
#pragma unroll
                    for (int h = 0; h < V; ++h) e[h] = C[h] / (float)(i + OFF + 1);
                    emit(i, e);
                } else if (i < n - OFF) {
#pragma unroll
                    for (int h = 0; h < V; ++h) e[h] = div_const(C[h] - c[h][0], dd, rdd);
                    emit(i, e);
                }
            }
        }
    }
    for (int i = n - OFF; i < n; ++i) {
        if (i < 0) continue;
        const int back = (n - 1) - (i - OFF - 1);
        float e[V];
#pragma unroll
        for (int h = 0; h < V; ++h) {
            float cm = 0.0f;
#pragma unroll
            for (int q = 0; q < W; ++q)
                if (q == W - 1 - back) cm = c[h][q];
            e[h] = (C[h] - cm) / (float)(n - i + OFF);
        }
        emit(i, e);
    }
}

__global__ void unpad_rescale_kernel(const float *__restrict__ in, int py, int px, float *__restrict__ out, int yn,
                                     int xn, int zn, int oy, int ox, int oz, float rescale) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (uint64_t)yn * xn * zn) return;
    int y = (int)(g % yn), x = (int)((g / yn) % xn), z = (int)(g / ((uint64_t)yn * xn));
    out[g] = in[idx3(y + oy, x + ox, z + oz, py, px)] * rescale;
}

// constant-scale fallback (:126-148): sum in double, min in float
__global__ void sum_min_kernel(const float *__restrict__ in, uint64_t n, double *sum, unsigned *minbits) {
    double s = 0;
    float mn = 660000.0f;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        float t = in[i];
        s += t;
        mn = t < mn ? t : mn;
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        mn = fminf(mn, __shfl_down_sync(0xffffffffu, mn, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(sum, s);
        // order-preserving float bits for non-negative and negative values
        unsigned b = __float_as_uint(mn);
        b = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
        atomicMin(minbits, b);
    }
}

__global__ void const_scale_fill_kernel(float *out, uint64_t n, const double *sum, const unsigned *minbits,
                                        float numel) {
    unsigned b = *minbits;
    b = (b & 0x80000000u) ? (b & 0x7fffffffu) : ~b;
    const float mn = __uint_as_float(b);
    const float sv = (float)(*sum / (double)numel - (double)mn);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = sv;
}

// ---------------------------------------------------------------------------
// a7 + a8 + first fill of a9: applyParameters (APRConverter.hpp:250-297),
// computeLevels / compute_level_for_array (LocalParticleCellSet.hpp:129-171)
// and PullingScheme::fill at the top pct level (PullingScheme.hpp:137-149).
// ---------------------------------------------------------------------------
template <typename IT>
__device__ __forceinline__ void level_of(IT &gv, float &sv, float idv, float th, float sigma_th, float sigma_th_max,
                                         float grad_th, float mult, int top_level, uint8_t &lev8, uint8_t &st8) {
    float g = (float)gv;
    float s = sv;
    if (idv <= th) g = 0.0f;
    if (s < sigma_th) s = (s < sigma_th_max) ? 60000.0f : sigma_th;
    if (g < grad_th) g = 0.0f;
    gv = to_it<IT>(g);
    sv = s;
    const float q = g / s;
    const uint32_t u = cvt_u32(q * mult);
    const int lev = u == 0 ? 0 : 31 - __clz(u);
    lev8 = (uint8_t)lev;
    st8 = ((float)lev >= (float)top_level) ? kSeed : kEmpty;
}

// Four cells per thread with vector loads and stores when the arrays allow it
// (VEC), else one.
template <typename IT, bool VEC>
__global__ void levels_kernel(IT *__restrict__ grad, float *__restrict__ lis, const float *__restrict__ ids,
                              uint64_t nd, const float *__restrict__ d_offset, float Ip_th, float sigma_th,
                              float sigma_th_max, float grad_th, float mult, int top_level, uint8_t *__restrict__ level,
                              uint8_t *__restrict__ status, int keep) {
    const float th = Ip_th + (d_offset ? *d_offset : 0.0f);
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (VEC) {
        const uint64_t i = 4 * t;
        if (i >= nd) return;
        if (i + 4 <= nd) {
            IT g[4];
            float s[4], d[4];
            if (sizeof(IT) == 4) {
                const float4 v = *reinterpret_cast<const float4 *>(grad + i);
                g[0] = (IT)v.x, g[1] = (IT)v.y, g[2] = (IT)v.z, g[3] = (IT)v.w;
            } else {
                const ushort4 v = *reinterpret_cast<const ushort4 *>(grad + i);
                g[0] = (IT)v.x, g[1] = (IT)v.y, g[2] = (IT)v.z, g[3] = (IT)v.w;
            }
            const float4 sv = *reinterpret_cast<const float4 *>(lis + i);
            const float4 dv = *reinterpret_cast<const float4 *>(ids + i);
            s[0] = sv.x, s[1] = sv.y, s[2] = sv.z, s[3] = sv.w;
            d[0] = dv.x, d[1] = dv.y, d[2] = dv.z, d[3] = dv.w;
            uint8_t lv[4], st[4];
#pragma unroll
            for (int k = 0; k < 4; ++k)
                level_of<IT>(g[k], s[k], d[k], th, sigma_th, sigma_th_max, grad_th, mult, top_level, lv[k], st[k]);
            *reinterpret_cast<uchar4 *>(level + i) = make_uchar4(lv[0], lv[1], lv[2], lv[3]);
            if (status) *reinterpret_cast<uchar4 *>(status + i) = make_uchar4(st[0], st[1], st[2], st[3]);
            if (keep) {
                if (sizeof(IT) == 4)
                    *reinterpret_cast<float4 *>(grad + i) = make_float4((float)g[0], (float)g[1], (float)g[2],
                                                                        (float)g[3]);
                else
                    *reinterpret_cast<ushort4 *>(grad + i) = make_ushort4((uint16_t)g[0], (uint16_t)g[1],
                                                                          (uint16_t)g[2], (uint16_t)g[3]);
                *reinterpret_cast<float4 *>(lis + i) = make_float4(s[0], s[1], s[2], s[3]);
            }
            return;
        }
        for (uint64_t j = i; j < nd; ++j) {
            IT g = grad[j];
            float s = lis[j];
            uint8_t lv, st;
            level_of<IT>(g, s, ids[j], th, sigma_th, sigma_th_max, grad_th, mult, top_level, lv, st);
            level[j] = lv;
            if (status) status[j] = st;
            if (keep) {
                grad[j] = g;
                lis[j] = s;
            }
        }
        return;
    }
    const uint64_t i = t;
    if (i >= nd) return;
    IT g = grad[i];
    float s = lis[i];
    uint8_t lv, st;
    level_of<IT>(g, s, ids[i], th, sigma_th, sigma_th_max, grad_th, mult, top_level, lv, st);
    level[i] = lv;
    if (status) status[i] = st;
    if (keep) {
        grad[i] = g;
        lis[i] = s;
    }
}

// ---------------------------------------------------------------------------
// host drivers
// ---------------------------------------------------------------------------
// Folded boundary vectors ([4][minLen] floats) of one filter, uploaded once
// per device and content and then kept: converters on other host threads and
// streams may use other filters at the same time, so no launch's vectors are
// ever overwritten.
static const float *bc_table(const IIRCoef &c) {
    if (c.minLen > kMaxK0) {
        set_error("recursive filter support exceeds the supported maximum (lambda too large)");
        throw Error{APRB_ERR_UNSUPPORTED};
    }
    int dev = 0;
    APRB_CUDA(cudaGetDevice(&dev));
    std::vector<float> h;
    h.reserve(4 * c.minLen + 1);
    h.push_back((float)dev);
    for (const auto *v : {&c.bc1, &c.bc2, &c.bc3, &c.bc4}) h.insert(h.end(), v->begin(), v->begin() + c.minLen);
    static std::mutex mu;
    static std::map<std::vector<float>, float *> *tab = new std::map<std::vector<float>, float *>();
    std::lock_guard<std::mutex> lock(mu);
    auto it = tab->find(h);
    if (it != tab->end()) return it->second;
    float *d = nullptr;
    APRB_CUDA(cudaMalloc(&d, std::max<size_t>(4 * c.minLen, 1) * sizeof(float)));
    if (c.minLen) APRB_CUDA(cudaMemcpy(d, h.data() + 1, 4 * c.minLen * sizeof(float), cudaMemcpyHostToDevice));
    tab->emplace(std::move(h), d);
    return d;
}

static IIRDev dev_coef(const IIRCoef &c) {
    IIRDev d;
    d.b1 = c.b1;
    d.b2 = c.b2;
    d.norm = c.norm;
    d.minLen = c.minLen;
    d.bc = bc_table(c);
    return d;
}

void launch_minmax_offset(const uint16_t *img, uint64_t n, unsigned *mm, float *offset, int apply, cudaStream_t s) {
    APRB_PROF("offset", s);
    if (apply) {
        unsigned init[2] = {0xffffu, 0u};
        APRB_CUDA(cudaMemcpyAsync(mm, init, sizeof(init), cudaMemcpyHostToDevice, s));
        unsigned blocks = (unsigned)std::min<uint64_t>(blocks_for(n, 256), 148u * 16u);
        minmax_u16_kernel<<<blocks, 256, 0, s>>>(img, n, mm);
        count_launch();
        APRB_CHECK_LAUNCH();
    }
    offset_kernel<<<1, 32, 0, s>>>(mm, offset, apply);
    count_launch();
    APRB_CHECK_LAUNCH();
}

// y pass (or the plain offset copy) then x pass of planes that the caller
// chose: both only read lines that lie inside the planes.
template <typename IT>
static void launch_smooth_yx(const uint16_t *img, IT *work, int yn, int xn, int zn, float lambda,
                             const float *d_offset, unsigned *d_err, DevBuf &ckpt, cudaStream_t s) {
    const uint64_t n = (uint64_t)yn * xn * zn;
    if (lambda > 0 && yn > 2) {
        APRB_PROF("bspline_y", s);
        const IIRDev c = dev_coef(iir_coefficients(lambda, yn));
        const uint64_t nlines = (uint64_t)xn * zn;
        const uint64_t nck = nlines * (uint64_t)((yn + kAY - 1) / kAY);
        if (std::is_same<IT, float>::value &&
            launch_iir_y_tma(img, (float *)work, yn, nlines, c, d_err + 1, ckpt.as_on<float2>(nck, s), nck, s)) {
            // TMA-staged tiles (iir_y_tma.cu); the launch is counted there
        } else if (yn % 2 == 0 && ((uintptr_t)img & 3) == 0) {
            float2 *ck = ckpt.as_on<float2>(nck, s);
            iir_y_rc_kernel<IT><<<blocks_for(nlines, 32 * kAWarps), 32 * kAWarps, 0, s>>>(img, work, yn, nlines, c, d_offset, d_err, ck);
            count_launch();
        } else {
            const unsigned blocks = blocks_for(nlines, kYWarps * kTile);
            iir_y_kernel<IT><<<blocks, kYWarps * 32, 0, s>>>(img, work, yn, nlines, c, d_offset, d_err);
            count_launch();
        }
        APRB_CHECK_LAUNCH();
    } else {
        APRB_PROF("offset_copy", s);
        unsigned blocks = (unsigned)std::min<uint64_t>(blocks_for(n, 256), 148u * 32u);
        offset_copy_kernel<IT><<<blocks, 256, 0, s>>>(img, work, n, d_offset);
        count_launch();
        APRB_CHECK_LAUNCH();
    }
    if (lambda > 0 && xn > 2) {
        APRB_PROF("bspline_x", s);
        const IIRDev c = dev_coef(iir_coefficients(lambda, xn));
        const uint64_t nlines = (uint64_t)yn * zn;
        const uint64_t nck = nlines * (uint64_t)((xn + kRC - 1) / kRC);
        float2 *ck = ckpt.as_on<float2>(nck, s);
        if (!(std::is_same<IT, float>::value &&
              launch_strided_iir_tma((float *)work, yn, xn, zn, false, c, d_err + 1, ck, nck, s))) {
            launch_strided_iir<IT>(work, yn, xn, (uint64_t)yn, (uint64_t)xn * yn, nlines, c, d_err, ck, s);
            count_launch();
            APRB_CHECK_LAUNCH();
        }
    }
}

template <typename IT>
static void launch_smooth_z(IT *work, int yn, int xn, int zn, float lambda, unsigned *d_err, DevBuf &ckpt,
                            cudaStream_t s) {
    if (lambda > 0 && zn > 2) {
        APRB_PROF("bspline_z", s);
        const IIRDev c = dev_coef(iir_coefficients(lambda, zn));
        const uint64_t nlines = (uint64_t)yn * xn;
        const uint64_t nck = nlines * (uint64_t)((zn + kRC - 1) / kRC);
        float2 *ck = ckpt.as_on<float2>(nck, s);
        if (!(std::is_same<IT, float>::value &&
              launch_strided_iir_tma((float *)work, yn, xn, zn, true, c, d_err + 1, ck, nck, s))) {
            launch_strided_iir<IT>(work, yn, zn, (uint64_t)xn * yn, (uint64_t)yn, nlines, c, d_err, ck, s);
            count_launch();
            APRB_CHECK_LAUNCH();
        }
    }
}

template <typename IT>
void launch_smooth(const uint16_t *img, IT *work, int yn, int xn, int zn, float lambda, const float *d_offset,
                   unsigned *d_err, DevBuf &ckpt, cudaStream_t s) {
    launch_smooth_yx<IT>(img, work, yn, xn, zn, lambda, d_offset, d_err, ckpt, s);
    launch_smooth_z<IT>(work, yn, xn, zn, lambda, d_err, ckpt, s);
}

// Offset and smoothing of a volume that is still in host memory: it is copied
// to `img` in z-chunks on stream `up`, and each chunk's work starts on s as
// soon as its copy has landed, while the later chunks are still on the bus.
// With an offset that needs the whole volume's min/max (uint16 ImageType with
// smoothing) the chunks overlap the min/max reduction only; otherwise they
// overlap the y and x passes.  The z pass needs every plane and runs last.
template <typename IT>
void launch_upload_smooth(const uint16_t *host, uint16_t *img, IT *work, int yn, int xn, int zn, float lambda,
                          unsigned *mm, float *d_offset, int apply, unsigned *d_err, DevBuf &ckpt,
                          cudaStream_t s, cudaStream_t up) {
    const uint64_t plane = (uint64_t)yn * xn;
    const int chunk = (int)std::max<uint64_t>(4, (uint64_t(1) << 27) / std::max<uint64_t>(plane, 1));
    const int nch = (zn + chunk - 1) / chunk;
    std::vector<cudaEvent_t> ev(nch, nullptr);
    for (auto &e : ev) APRB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    struct Release {
        std::vector<cudaEvent_t> &ev;
        ~Release() {
            for (auto e : ev)
                if (e) cudaEventDestroy(e);
        }
    } release{ev};
    if (apply) {
        const unsigned init[2] = {0xffffu, 0u};
        APRB_CUDA(cudaMemcpyAsync(mm, init, sizeof(init), cudaMemcpyHostToDevice, s));
    }
    // the copies start after all of s's earlier work, which includes the
    // stream-ordered allocation of img
    cudaEvent_t ready = nullptr;
    APRB_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    ev.push_back(ready);
    APRB_CUDA(cudaEventRecord(ready, s));
    APRB_CUDA(cudaStreamWaitEvent(up, ready, 0));
    for (int k = 0; k < nch; ++k) {
        const int z0 = k * chunk, z1 = std::min(zn, z0 + chunk);
        const uint64_t o = (uint64_t)z0 * plane, cnt = (uint64_t)(z1 - z0) * plane;
        APRB_CUDA(cudaMemcpyAsync(img + o, host + o, cnt * sizeof(uint16_t), cudaMemcpyHostToDevice, up));
        APRB_CUDA(cudaEventRecord(ev[k], up));
        APRB_CUDA(cudaStreamWaitEvent(s, ev[k], 0));
        if (apply) {
            APRB_PROF("offset", s);
            unsigned blocks = (unsigned)std::min<uint64_t>(blocks_for(cnt, 256), 148u * 16u);
            minmax_u16_kernel<<<blocks, 256, 0, s>>>(img + o, cnt, mm);
            count_launch();
            APRB_CHECK_LAUNCH();
        } else {
            if (k == 0) {
                offset_kernel<<<1, 32, 0, s>>>(mm, d_offset, 0);
                count_launch();
                APRB_CHECK_LAUNCH();
            }
            launch_smooth_yx<IT>(img + o, work + o, yn, xn, z1 - z0, lambda, d_offset, d_err, ckpt, s);
        }
    }
    if (apply) {
        offset_kernel<<<1, 32, 0, s>>>(mm, d_offset, 1);
        count_launch();
        APRB_CHECK_LAUNCH();
        launch_smooth_yx<IT>(img, work, yn, xn, zn, lambda, d_offset, d_err, ckpt, s);
    }
    launch_smooth_z<IT>(work, yn, xn, zn, lambda, d_err, ckpt, s);
}

template <typename IT>
void launch_gradient(const IT *work, int yn, int xn, int zn, IT *grad, float *ids_raw, float *ids, int yd, int xd,
                     int zd, const aprb_params &p, unsigned *d_timeout, cudaStream_t s) {
    {
        APRB_PROF("gradient_ds", s);
        dim3 grid((yd + kGY - 1) / kGY, (xd + kGX - 1) / kGX, (zd + kGZ - 1) / kGZ);
        auto pow2 = [](float h) {
            int e = 0;
            const float m = std::frexp(2.0f * h, &e);
            return m == 0.5f && e > -120 && e < 120;
        };
        auto run = [&](auto kern) {
            APRB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGradSmem));
            kern<<<grid, kGThreads, kGradSmem, s>>>(work, yn, xn, zn, grad, ids_raw, yd, xd, zd, p.dx, p.dy, p.dz);
        };
        const bool vec = sizeof(IT) == 4 && yn % 4 == 0 && ((uintptr_t)work & 15) == 0;
        if (pow2(p.dx) && pow2(p.dy) && pow2(p.dz)) {
            if (vec)
                run(grad_ds_kernel<IT, true, true>);
            else
                run(grad_ds_kernel<IT, true, false>);
        } else {
            if (vec)
                run(grad_ds_kernel<IT, false, true>);
            else
                run(grad_ds_kernel<IT, false, false>);
        }
        count_launch();
        APRB_CHECK_LAUNCH();
    }
    APRB_PROF("inv_bspline", s);
    const bool on = p.lambda > 0;
    InvB c;
    c.a1 = (float)(1.0 / 6.0);
    c.a2 = (float)(4.0 / 6.0);
    c.a3 = (float)(1.0 / 6.0);
    c.a13 = c.a1 + c.a3;
    dim3 grid((yd + kJY - 1) / kJY, (xd + kJX - 1) / kJX, (zd + kJZ - 1) / kJZ);
    const int ony = on && yn > 2, onx = on && xn > 2, onz = on && zn > 2;
    if (!launch_inv_bspline_tma(ids_raw, ids, yd, xd, zd, ony, onx, onz, c, d_timeout, s)) {
        inv_bspline_kernel<<<grid, kJY, 0, s>>>(ids_raw, ids, yd, xd, zd, ony, onx, onz, c);
        count_launch();
        APRB_CHECK_LAUNCH();
    }
}

template <int OFF>
static void sat_axis_t(const float *in, const float *absref, float *out, int py, int px, int pz, int axis,
                       const PadMap &pm, const LisOut *fo, cudaStream_t s) {
    if (axis == 0) {
        const uint64_t nlines = (uint64_t)px * pz;
        if (absref)
            sat_y_async_kernel<OFF, true><<<blocks_for(nlines, 32 * kSW), 32 * kSW, 0, s>>>(in, absref, out, py, nlines, pm);
        else
            sat_y_async_kernel<OFF, false><<<blocks_for(nlines, 32 * kSW), 32 * kSW, 0, s>>>(in, absref, out, py, nlines, pm);
    } else {
        const uint64_t nlines = axis == 1 ? (uint64_t)py * pz : (uint64_t)py * px;
        const int n = axis == 1 ? px : pz;
        const uint64_t stride = axis == 1 ? (uint64_t)py : (uint64_t)px * py;
        const uint64_t outer = axis == 1 ? (uint64_t)px * py : (uint64_t)py;
        if (py % 2 == 0 && fo)
            sat_stridedv_kernel<OFF, true, 2><<<blocks_for(nlines / 2, 128), 128, 0, s>>>(in, absref, nullptr, py, n,
                                                                                      stride, outer, nlines, *fo);
        else if (py % 2 == 0)
            sat_stridedv_kernel<OFF, false, 2><<<blocks_for(nlines / 2, 128), 128, 0, s>>>(in, absref, out, py, n,
                                                                                       stride, outer, nlines, LisOut{});
        else if (fo)
            sat_strided_kernel<OFF, true><<<blocks_for(nlines, 128), 128, 0, s>>>(in, absref, nullptr, py, n, stride,
                                                                                  outer, nlines, *fo);
        else
            sat_strided_kernel<OFF, false><<<blocks_for(nlines, 128), 128, 0, s>>>(in, absref, out, py, n, stride,
                                                                                   outer, nlines, LisOut{});
    }
    count_launch();
    APRB_CHECK_LAUNCH();
}

static void sat_axis(const float *in, const float *absref, float *out, int py, int px, int pz, int axis, int off,
                     const PadMap &pm, const LisOut *fo, cudaStream_t s) {
    switch (off) {
        case 1: sat_axis_t<1>(in, absref, out, py, px, pz, axis, pm, fo, s); break;
        case 2: sat_axis_t<2>(in, absref, out, py, px, pz, axis, pm, fo, s); break;
        case 3: sat_axis_t<3>(in, absref, out, py, px, pz, axis, pm, fo, s); break;
        case 4: sat_axis_t<4>(in, absref, out, py, px, pz, axis, pm, fo, s); break;
        case 5: sat_axis_t<5>(in, absref, out, py, px, pz, axis, pm, fo, s); break;
        case 6: sat_axis_t<6>(in, absref, out, py, px, pz, axis, pm, fo, s); break;
        default: set_error("unsupported local intensity scale window"); throw Error{APRB_ERR_UNSUPPORTED};
    }
}

void launch_local_intensity_scale(const float *ids, float *lis, int yd, int xd, int zd, const aprb_params &p,
                                  LisBuffers &b, cudaStream_t s) {
    APRB_PROF("local_intensity_scale", s);
    const LisWindow w = lis_window(p, yd, xd, zd);
    const uint64_t nd = (uint64_t)yd * xd * zd;
    if (p.constant_intensity_scale || w.n_active == 0) {
        double *sum = b.scalars.as_on<double>(2, s);
        unsigned *mb = (unsigned *)(sum + 1);
        unsigned init_min = 0xffffffffu;
        APRB_CUDA(cudaMemsetAsync(sum, 0, sizeof(double), s));
        APRB_CUDA(cudaMemcpyAsync(mb, &init_min, sizeof(unsigned), cudaMemcpyHostToDevice, s));
        unsigned blocks = (unsigned)std::min<uint64_t>(blocks_for(nd, 256), 148u * 8u);
        sum_min_kernel<<<blocks, 256, 0, s>>>(ids, nd, sum, mb);
        const_scale_fill_kernel<<<blocks, 256, 0, s>>>(lis, nd, sum, mb, (float)(yd * xd * zd));
        count_launch(2);
        APRB_CHECK_LAUNCH();
        return;
    }
    int sy = std::max(w.win1[0], w.win2[0]), sx = std::max(w.win1[1], w.win2[1]), sz = std::max(w.win1[2], w.win2[2]);
    if (p.reflect_bc_lis) {
        sy = yd > 1 ? std::min(sy, yd - 1) : 0;
        sx = xd > 1 ? std::min(sx, xd - 1) : 0;
        sz = zd > 1 ? std::min(sz, zd - 1) : 0;
    } else {
        sy = sx = sz = 0;
    }
    const int py = yd + 2 * sy, px = xd + 2 * sx, pz = zd + 2 * sz;
    const int pd[3] = {py, px, pz};
    int last = -1;
    for (int a = 0; a < 3; ++a) {
        if (w.active[a] && pd[a] < 2 * std::max(w.win1[a], w.win2[a]) + 2) {
            set_error("local intensity scale window longer than the (padded) image axis");
            throw Error{APRB_ERR_UNSUPPORTED};
        }
        if (w.active[a]) last = a;
    }
    // The padded copy is read only by the first pass of each window; when y is
    // active that pass is a y pass, which reads the unpadded image through the
    // reflection instead.  A final x or z pass writes the unpadded, rescaled
    // window itself.
    const bool fold_pad = w.active[0], fold_unpad = last >= 1;
    const uint64_t pn = (uint64_t)py * px * pz;
    float *A = b.a.as_on<float>(pn, s);
    float *C2 = b.c.as_on<float>(pn, s);
    const float *padded = ids;
    if (!fold_pad) {
        float *B = b.padded.as_on<float>(pn, s);
        pad_reflect_kernel<<<blocks_for(pn, 256), 256, 0, s>>>(ids, yd, xd, zd, B, sy, sx, sz, py, px, pz);
        count_launch();
        APRB_CHECK_LAUNCH();
        padded = B;
    }
    const PadMap none{0, 0, 0, 0, 0, 1, 1, 1, 1};
    const PadMap map_in{1, 0, sy, sx, sz, yd, xd, zd, px}, map_ref{0, 1, sy, sx, sz, yd, xd, zd, px};
    const LisOut fo{lis, sy, sx, sz, yd, xd, zd, last, w.rescale};
    const float *src = padded;
    float *bufs[2] = {A, C2};
    int nb = 0;
    bool first = true;
    for (int a = 0; a < 3; ++a)
        if (w.active[a]) {
            sat_axis(src, nullptr, bufs[nb], py, px, pz, a, w.win1[a], (first && fold_pad) ? map_in : none, nullptr,
                     s);
            first = false;
            src = bufs[nb];
            nb ^= 1;
        }
    first = true;
    for (int a = 0; a < 3; ++a)
        if (w.active[a]) {
            const bool fin = fold_unpad && a == last;
            sat_axis(src, first ? padded : nullptr, fin ? nullptr : bufs[nb], py, px, pz, a, w.win2[a],
                     (first && fold_pad) ? map_ref : none, fin ? &fo : nullptr, s);
            first = false;
            src = bufs[nb];
            nb ^= 1;
        }
    if (!fold_unpad) {
        unpad_rescale_kernel<<<blocks_for(nd, 256), 256, 0, s>>>(src, py, px, lis, yd, xd, zd, (py - yd) / 2,
                                                                (px - xd) / 2, (pz - zd) / 2, w.rescale);
        count_launch();
        APRB_CHECK_LAUNCH();
    }
}

template <typename IT>
void launch_levels(IT *grad, float *lis, const float *ids, uint64_t nd, const float *d_offset, const aprb_params &p,
                   int apr_l_max, int top_level, uint8_t *level, uint8_t *status, int keep, cudaStream_t s) {
    APRB_PROF("levels", s);
    const float mxz = p.dz < p.dx ? p.dz : p.dx;
    const float min_dim = mxz < p.dy ? mxz : p.dy;
    const float level_factor = (float)(std::pow(2.0, (double)apr_l_max) * (double)min_dim);
    const float mult = level_factor / p.rel_error;
    auto al = [](const void *q, int a) { return ((uintptr_t)q % a) == 0; };
    if (al(grad, 4 * sizeof(IT)) && al(lis, 16) && al(ids, 16) && al(level, 4) && (!status || al(status, 4)))
        levels_kernel<IT, true><<<blocks_for((nd + 3) / 4, 256), 256, 0, s>>>(
            grad, lis, ids, nd, d_offset, p.Ip_th, p.sigma_th, p.sigma_th_max, p.grad_th, mult, top_level, level,
            status, keep);
    else
        levels_kernel<IT, false><<<blocks_for(nd, 256), 256, 0, s>>>(grad, lis, ids, nd, d_offset, p.Ip_th,
                                                                    p.sigma_th, p.sigma_th_max, p.grad_th, mult,
                                                                    top_level, level, status, keep);
    count_launch();
    APRB_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------
// Level-decision margins (diagnostic, outside get_apr): the level of a ds cell
// is floor(log2(v)) for v = (grad / scale) * mult >= 1 (level_of above,
// LocalParticleCellSet.hpp:129-171), so a computation of v that is off by a
// relative r can decide another level only where v lies within r of a power
// of two 2^k, k >= 1.  Counts those cells and the cells with v >= 1, from the
// gradient and scale after applyParameters.
template <typename IT>
__global__ void level_margin_kernel(const IT *__restrict__ grad, const float *__restrict__ lis, uint64_t nd,
                                    float mult, double rel, unsigned long long *counts) {
    unsigned long long near = 0, active = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nd;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float q = (float)grad[i] / lis[i];
        const double v = (double)(q * mult);
        if (!(v >= 1.0)) continue;
        ++active;
        int e;
        frexp(v, &e);  // v = m 2^e, m in [0.5, 1): the nearest powers are 2^(e-1) and 2^e
        const double lo = ldexp(1.0, e - 1), hi = ldexp(1.0, e);
        if ((e - 1 >= 1 && v - lo <= rel * lo) || hi - v <= rel * hi) ++near;
    }
    for (int o = 16; o; o >>= 1) {
        near += __shfl_down_sync(0xffffffffu, near, o);
        active += __shfl_down_sync(0xffffffffu, active, o);
    }
    if ((threadIdx.x & 31) == 0 && (near | active)) {
        atomicAdd(&counts[0], near);
        atomicAdd(&counts[1], active);
    }
}

template <typename IT>
void launch_level_margins(const IT *grad, const float *lis, uint64_t nd, const aprb_params &p, int apr_l_max,
                          double rel, unsigned long long *counts, cudaStream_t s) {
    const float mxz = p.dz < p.dx ? p.dz : p.dx;
    const float min_dim = mxz < p.dy ? mxz : p.dy;
    const float level_factor = (float)(std::pow(2.0, (double)apr_l_max) * (double)min_dim);
    const float mult = level_factor / p.rel_error;
    APRB_CUDA(cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned long long), s));
    const unsigned blocks = (unsigned)std::min<uint64_t>(blocks_for(nd, 256), 148 * 8);
    level_margin_kernel<IT><<<blocks, 256, 0, s>>>(grad, lis, nd, mult, rel, counts);
    count_launch();
    APRB_CHECK_LAUNCH();
}
template void launch_level_margins<uint16_t>(const uint16_t *, const float *, uint64_t, const aprb_params &, int,
                                             double, unsigned long long *, cudaStream_t);
template void launch_level_margins<float>(const float *, const float *, uint64_t, const aprb_params &, int, double,
                                          unsigned long long *, cudaStream_t);

template void launch_upload_smooth<uint16_t>(const uint16_t *, uint16_t *, uint16_t *, int, int, int, float,
                                             unsigned *, float *, int, unsigned *, DevBuf &, cudaStream_t,
                                             cudaStream_t);
template void launch_upload_smooth<float>(const uint16_t *, uint16_t *, float *, int, int, int, float, unsigned *,
                                          float *, int, unsigned *, DevBuf &, cudaStream_t, cudaStream_t);
template void launch_smooth<uint16_t>(const uint16_t *, uint16_t *, int, int, int, float, const float *, unsigned *,
                                      DevBuf &, cudaStream_t);
template void launch_smooth<float>(const uint16_t *, float *, int, int, int, float, const float *, unsigned *,
                                   DevBuf &, cudaStream_t);
template void launch_gradient<uint16_t>(const uint16_t *, int, int, int, uint16_t *, float *, float *, int, int, int,
                                        const aprb_params &, unsigned *, cudaStream_t);
template void launch_gradient<float>(const float *, int, int, int, float *, float *, float *, int, int, int,
                                     const aprb_params &, unsigned *, cudaStream_t);
template void launch_levels<uint16_t>(uint16_t *, float *, const float *, uint64_t, const float *, const aprb_params &,
                                      int, int, uint8_t *, uint8_t *, int, cudaStream_t);
template void launch_levels<float>(float *, float *, const float *, uint64_t, const float *, const aprb_params &, int,
                                   int, uint8_t *, uint8_t *, int, cudaStream_t);

// ---------------------------------------------------------------------------
// exhaustive comparison of div_const with the IEEE division
// ---------------------------------------------------------------------------
__global__ void check_div_const_kernel(float d, unsigned long long *out) {
    const float r = __frcp_rn(d);
    unsigned long long bad = 0, first = ~0ull;
    for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; b < (1ull << 32);
         b += (uint64_t)gridDim.x * blockDim.x) {
        const float x = __uint_as_float((uint32_t)b);
        const float a = div_const(x, d, r), e = __fdiv_rn(x, d);
        if (__float_as_uint(a) != __float_as_uint(e) && !(a != a && e != e)) {
            ++bad;
            first = b < first ? b : first;
        }
    }
    if (bad) {
        atomicAdd(&out[0], bad);
        atomicMin(&out[1], first);
    }
}

void launch_check_div_const(float d, unsigned long long *out, cudaStream_t s) {
    check_div_const_kernel<<<148 * 16, 256, 0, s>>>(d, out);
    count_launch();
    APRB_CHECK_LAUNCH();
}

}  // namespace aprb
