// Automatic parameters: autoParametersLiEntropy
// (src/algorithm/AutoParameters.hpp:103-153) on the converter's device arrays.
//
//  1. The foreground cells (ds image > Ip_th + bspline_offset) are counted
//     per chunk of kFgChunk cells, the counts scanned, and the gradient and
//     local intensity scale of every delta-th foreground cell (in index order)
//     gathered into two arrays of at most 32*512*512 values, as the reference
//     compacts and then strides (:117-147).
//  2. threshold_li (:50-100) on each array: min, max and mean, then Li's
//     one-point iteration, whose means come from li_stats_kernel and whose
//     scalar steps run on the host with the reference's float arithmetic and
//     std::log.  The sums are FP64 in a fixed order (deterministic; the
//     reference's FP32 sums depend on its OpenMP thread count), each mean is
//     rounded to float once.
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "kernels.cuh"

namespace aprb {
namespace {

constexpr int kFgThreads = 256;
constexpr int kFgIter = 16;
constexpr uint64_t kFgChunk = (uint64_t)kFgThreads * kFgIter;  // cells per block
constexpr uint64_t kSubsampleCap = (uint64_t)32 * 512 * 512;   // AutoParameters.hpp:140
constexpr int kScanThreads = 1024;
constexpr int kStatsThreads = 256;
constexpr int kStatsBlocks = 1184;  // 8 per SM; fixed, so the reduction order is too
constexpr int kLiMaxSteps = 1000;  // bound on Li steps (the reference has none)

__device__ __forceinline__ float fg_threshold(const float *d_off, float Ip_th) {
    return Ip_th + (d_off ? *d_off : 0.0f);
}

// Foreground cells of each kFgChunk-cell chunk.
__global__ void __launch_bounds__(kFgThreads) fg_count_kernel(const float *__restrict__ ids, uint64_t nd,
                                                              const float *__restrict__ d_off, float Ip_th,
                                                              unsigned *__restrict__ counts) {
    const float th = fg_threshold(d_off, Ip_th);
    const uint64_t base = (uint64_t)blockIdx.x * kFgChunk;
    unsigned c = 0;
#pragma unroll 4
    for (int k = 0; k < kFgIter; ++k) {
        const uint64_t i = base + (uint64_t)k * kFgThreads + threadIdx.x;
        if (i < nd && ids[i] > th) ++c;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    __shared__ unsigned ws[kFgThreads / 32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned t = 0;
        for (int w = 0; w < kFgThreads / 32; ++w) t += ws[w];
        counts[blockIdx.x] = t;
    }
}

// Exclusive scan of the chunk counts in one block; offs[nblk] = total.
__global__ void __launch_bounds__(kScanThreads) fg_scan_kernel(const unsigned *__restrict__ counts, uint64_t nblk,
                                                               unsigned long long *__restrict__ offs) {
    __shared__ unsigned long long sh[kScanThreads];
    const uint64_t per = (nblk + kScanThreads - 1) / kScanThreads;
    const uint64_t b0 = min(nblk, (uint64_t)threadIdx.x * per), b1 = min(nblk, b0 + per);
    unsigned long long s = 0;
    for (uint64_t b = b0; b < b1; ++b) s += counts[b];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < kScanThreads; o <<= 1) {
        const unsigned long long v = threadIdx.x >= (unsigned)o ? sh[threadIdx.x - o] : 0ull;
        __syncthreads();
        sh[threadIdx.x] += v;
        __syncthreads();
    }
    unsigned long long run = sh[threadIdx.x] - s;
    for (uint64_t b = b0; b < b1; ++b) {
        offs[b] = run;
        run += counts[b];
    }
    if (threadIdx.x == kScanThreads - 1) offs[nblk] = sh[threadIdx.x];
}

// Gathers the gradient and scale of the foreground cells whose rank r (in
// index order) is a multiple of delta, to position r / delta < m.  Warp w of
// a block owns the 32 * kFgIter consecutive cells from base + w * 32 *
// kFgIter: it counts them, the block adds the counts of the warps before it
// to the chunk's offset (the only barrier), and the warp ranks its cells
// with ballots in a second read (from L1).
template <typename IT>
__global__ void __launch_bounds__(kFgThreads) fg_subsample_kernel(
    const float *__restrict__ ids, const IT *__restrict__ grad, const float *__restrict__ lis, uint64_t nd,
    const float *__restrict__ d_off, float Ip_th, const unsigned long long *__restrict__ offs, uint64_t m,
    uint64_t delta, float *__restrict__ sub_g, float *__restrict__ sub_l) {
    __shared__ unsigned wc[kFgThreads / 32];
    const float th = fg_threshold(d_off, Ip_th);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint64_t base = (uint64_t)blockIdx.x * kFgChunk + (uint64_t)w * (32 * kFgIter);
    const uint64_t end = m * delta;
    uint64_t run = offs[blockIdx.x];
    if (run >= end) return;  // uniform over the block
    unsigned c = 0;
#pragma unroll 4
    for (int k = 0; k < kFgIter; ++k) {
        const uint64_t i = base + (uint64_t)(32 * k + lane);
        if (i < nd && ids[i] > th) ++c;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    if (lane == 0) wc[w] = c;
    __syncthreads();
    for (int q = 0; q < w; ++q) run += wc[q];
    if (run >= end) return;  // uniform over the warp
    const unsigned below = (1u << lane) - 1u;
    for (int k = 0; k < kFgIter; ++k) {
        const uint64_t i = base + (uint64_t)(32 * k + lane);
        const bool f = i < nd && ids[i] > th;
        const unsigned bal = __ballot_sync(0xffffffffu, f);
        if (f) {
            const uint64_t r = run + __popc(bal & below);
            const uint64_t j = delta == 1 ? r : r / delta;
            if (j < m && j * delta == r) {
                sub_g[j] = (float)grad[i];
                sub_l[j] = lis[i];
            }
        }
        run += __popc(bal);
    }
}

// Per array: mode 0 -> a = sum, mn, mx; mode 1 -> a = sum above t, b = sum
// at or below t, c = count above t (compute_means, AutoParameters.hpp:17-36).
struct LiStats {
    double a, b;
    unsigned long long c;
    float mn, mx;
};

struct LiArgs {
    const float *v[2];
    float t[2];
    int active[2];
};

__device__ __forceinline__ LiStats li_combine(LiStats x, const LiStats &y) {
    x.a += y.a;
    x.b += y.b;
    x.c += y.c;
    x.mn = fminf(x.mn, y.mn);
    x.mx = fmaxf(x.mx, y.mx);
    return x;
}

__device__ __forceinline__ LiStats li_shfl_down(const LiStats &s, int o) {
    LiStats r;
    r.a = __shfl_down_sync(0xffffffffu, s.a, o);
    r.b = __shfl_down_sync(0xffffffffu, s.b, o);
    r.c = __shfl_down_sync(0xffffffffu, s.c, o);
    r.mn = __shfl_down_sync(0xffffffffu, s.mn, o);
    r.mx = __shfl_down_sync(0xffffffffu, s.mx, o);
    return r;
}

// Fixed-shape block reduction; the result is in thread 0.
__device__ LiStats li_block_reduce(LiStats s) {
    __shared__ LiStats ws[kStatsThreads / 32];
    for (int o = 16; o > 0; o >>= 1) s = li_combine(s, li_shfl_down(s, o));
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int w = 1; w < kStatsThreads / 32; ++w) s = li_combine(s, ws[w]);
    __syncthreads();
    return s;
}

__device__ __forceinline__ LiStats li_zero() {
    LiStats s;
    s.a = 0;
    s.b = 0;
    s.c = 0;
    s.mn = INFINITY;
    s.mx = -INFINITY;
    return s;
}

// One pass over both arrays; every block writes its partials, the last block
// to finish (ticket) sums them in block order into res[2] and rearms the
// ticket.  No block waits on another.
__global__ void __launch_bounds__(kStatsThreads) li_stats_kernel(LiArgs args, uint64_t m, int mode,
                                                                 LiStats *__restrict__ part,
                                                                 LiStats *__restrict__ res,
                                                                 unsigned *__restrict__ ticket) {
    __shared__ bool last;
    const uint64_t stride = (uint64_t)gridDim.x * kStatsThreads;
    for (int q = 0; q < 2; ++q) {
        LiStats s = li_zero();
        if (args.active[q]) {
            const float *v = args.v[q];
            const float t = args.t[q];
            auto take = [&](float x) {
                if (mode == 0) {
                    s.a += (double)x;
                    s.mn = fminf(s.mn, x);
                    s.mx = fmaxf(s.mx, x);
                } else if (x > t) {
                    s.a += (double)x;
                    s.c += 1;
                } else {
                    s.b += (double)x;
                }
            };
            // four values per load (the arrays start 16-byte aligned), the
            // last m % 4 by the first threads
            const uint64_t m4 = m / 4;
            const float4 *v4 = reinterpret_cast<const float4 *>(v);
            for (uint64_t i = (uint64_t)blockIdx.x * kStatsThreads + threadIdx.x; i < m4; i += stride) {
                const float4 x = __ldg(v4 + i);
                take(x.x);
                take(x.y);
                take(x.z);
                take(x.w);
            }
            const uint64_t g = (uint64_t)blockIdx.x * kStatsThreads + threadIdx.x;
            if (g < m - 4 * m4) take(v[4 * m4 + g]);
        }
        s = li_block_reduce(s);
        if (threadIdx.x == 0) part[(size_t)blockIdx.x * 2 + q] = s;
    }
    __threadfence();
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int q = 0; q < 2; ++q) {
        LiStats s = li_zero();
        for (unsigned b = threadIdx.x; b < gridDim.x; b += kStatsThreads) {
            const LiStats *p = part + (size_t)b * 2 + q;
            LiStats y;
            y.a = __ldcg(&p->a);
            y.b = __ldcg(&p->b);
            y.c = __ldcg(&p->c);
            y.mn = __ldcg(&p->mn);
            y.mx = __ldcg(&p->mx);
            s = li_combine(s, y);
        }
        s = li_block_reduce(s);
        if (threadIdx.x == 0) res[q] = s;
    }
    if (threadIdx.x == 0) *ticket = 0;
}

// Host side of threshold_li for one array.
struct LiState {
    bool integer = false, done = false;
    float tol = 0, t_curr = 0, t_next = 0, result = 0;
    int steps = 0;
};

void li_init(LiState &st, const LiStats &r, uint64_t m) {
    if (m == 0) {  // AutoParameters.hpp:52
        st.done = true;
        st.result = 0.f;
        return;
    }
    if (r.mn == r.mx) {  // :57
        st.done = true;
        st.result = r.mn;
        return;
    }
    st.tol = 0.5f;
    if (!st.integer) {
        const float range = r.mx - r.mn;
        st.tol = std::min(0.01f, range * 1e-4f);
    }
    st.t_next = (float)(r.a / (double)m);
    st.t_curr = -2.f * st.tol;
    if (st.integer && st.t_next < 1.f) st.t_next = std::min(1.5f, (r.mn + r.mx) / 2.f);
}

// Checks the loop condition of :81; true while another step is due.
bool li_wants_step(LiState &st) {
    if (st.done) return false;
    if (!(std::abs(st.t_next - st.t_curr) > st.tol) || st.steps >= kLiMaxSteps) {
        st.done = true;
        st.result = st.t_next;
        return false;
    }
    st.t_curr = st.t_next;
    st.steps++;
    return true;
}

void li_step(LiState &st, const LiStats &r, uint64_t m) {
    const float mean_fore = (float)(r.a / (double)r.c);
    const float mean_back = (float)(r.b / (double)(m - r.c));
    if (mean_back == 0) {  // :89-92
        st.done = true;
        st.result = st.t_curr;
        return;
    }
    st.t_next = (mean_fore - mean_back) / (std::log(mean_fore) - std::log(mean_back));
}

}  // namespace

void threshold_li_pair(const float *const v[2], uint64_t m, const int integer[2], const int active[2],
                       AutoParBuffers &b, cudaStream_t s, float out[2]) {
    LiState st[2];
    for (int q = 0; q < 2; ++q) {
        st[q].integer = integer[q] != 0;
        st[q].done = !active[q];
    }
    if (m == 0) {  // AutoParameters.hpp:52
        out[0] = out[1] = 0.f;
        return;
    }
    LiStats *part = b.part.as_on<LiStats>((size_t)kStatsBlocks * 2, s);
    LiStats *res = b.res.as_on<LiStats>(2, s);
    if (!b.ticket_ready) {
        APRB_CUDA(cudaMemsetAsync(b.ticket.as_on<unsigned>(1, s), 0, sizeof(unsigned), s));
        b.ticket_ready = true;
    }
    unsigned *ticket = (unsigned *)b.ticket.p;
    LiStats hres[2];
    const unsigned grid =
        (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(kStatsBlocks, (m / 4 + kStatsThreads - 1) / kStatsThreads));
    auto stats = [&](const LiArgs &args, int mode) {
        li_stats_kernel<<<grid, kStatsThreads, 0, s>>>(args, m, mode, part, res, ticket);
        APRB_CHECK_LAUNCH();
        count_launch();
        APRB_CUDA(cudaMemcpyAsync(hres, res, sizeof(LiStats) * 2, cudaMemcpyDeviceToHost, s));
        APRB_CUDA(cudaStreamSynchronize(s));
    };
    LiArgs args{{v[0], v[1]}, {0.f, 0.f}, {!st[0].done, !st[1].done}};
    stats(args, 0);
    for (int q = 0; q < 2; ++q)
        if (!st[q].done) li_init(st[q], hres[q], m);
    for (;;) {
        bool any = false;
        for (int q = 0; q < 2; ++q) {
            args.active[q] = li_wants_step(st[q]);
            args.t[q] = st[q].t_curr;
            any = any || args.active[q];
        }
        if (!any) break;
        stats(args, 1);
        for (int q = 0; q < 2; ++q)
            if (args.active[q]) li_step(st[q], hres[q], m);
    }
    for (int q = 0; q < 2; ++q) out[q] = st[q].result;
}

template <typename IT>
void auto_parameters(const float *ids, const IT *grad, const float *lis, uint64_t nd, const float *d_off,
                     float Ip_th, int grad_integer, AutoParBuffers &b, cudaStream_t s, float *grad_th,
                     float *sigma_th, uint64_t *n_subsample) {
    APRB_PROF("auto_parameters", s);
    const uint64_t nblk = (nd + kFgChunk - 1) / kFgChunk;
    uint64_t n_fg = 0;
    if (nblk) {
        unsigned *counts = b.counts.as_on<unsigned>(nblk, s);
        unsigned long long *offs = b.offs.as_on<unsigned long long>(nblk + 1, s);
        fg_count_kernel<<<(unsigned)nblk, kFgThreads, 0, s>>>(ids, nd, d_off, Ip_th, counts);
        APRB_CHECK_LAUNCH();
        fg_scan_kernel<<<1, kScanThreads, 0, s>>>(counts, nblk, offs);
        APRB_CHECK_LAUNCH();
        count_launch(2);
        unsigned long long h = 0;
        APRB_CUDA(cudaMemcpyAsync(&h, offs + nblk, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
        APRB_CUDA(cudaStreamSynchronize(s));
        n_fg = h;
    }
    const uint64_t m = std::min(kSubsampleCap, n_fg);
    if (n_subsample) *n_subsample = m;
    if (m == 0) {  // the reference divides by m here (:141); an empty input's thresholds
        *grad_th = 0.f;
        *sigma_th = 0.f;
        return;
    }
    const uint64_t delta = n_fg / m;
    float *sub_g = b.sub_g.as_on<float>(m, s), *sub_l = b.sub_l.as_on<float>(m, s);
    fg_subsample_kernel<IT><<<(unsigned)nblk, kFgThreads, 0, s>>>(ids, grad, lis, nd, d_off, Ip_th,
                                                                 (const unsigned long long *)b.offs.p, m, delta,
                                                                 sub_g, sub_l);
    APRB_CHECK_LAUNCH();
    count_launch();
    const float *v[2] = {sub_g, sub_l};
    const int integer[2] = {grad_integer != 0, 0};  // local_scale_temp is float
    const int active[2] = {1, 1};
    float out[2];
    threshold_li_pair(v, m, integer, active, b, s, out);
    *grad_th = out[0];
    *sigma_th = out[1];
}

template void auto_parameters<uint16_t>(const float *, const uint16_t *, const float *, uint64_t, const float *,
                                        float, int, AutoParBuffers &, cudaStream_t, float *, float *, uint64_t *);
template void auto_parameters<float>(const float *, const float *, const float *, uint64_t, const float *, float,
                                     int, AutoParBuffers &, cudaStream_t, float *, float *, uint64_t *);

}  // namespace aprb
