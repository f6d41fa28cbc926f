// a2 (x, z) for float ImageType: bspline_filt_rec_x (ComputeGradient.hpp:602-779)
// and bspline_filt_rec_z (:416-599) with TMA-staged segments.
//
// A CTA owns a run of consecutive y (one or more boxes of 256) of one plane of
// the other axis (one x row for the z pass, one z plane for the x pass): one
// line along the filtered axis per y, a few neighbouring lines per thread.
// The lines move through shared memory in segments of 16 samples, each
// segment one cp.async.bulk.tensor box of 256 y x 16 samples per 256 y, in a
// ring of stages whose mbarriers the copy engine completes; a CTA keeps
// several segments in flight without spending registers on them.
//
// The recurrences are those of the register-staged kernels in pipeline.cu,
// operation for operation: the causal sweep walks the segments forward and
// keeps only the recurrence state at each segment start (ckpt); the
// anti-causal sweep walks them backward, recomputes each segment's causal
// values from its saved state and the untouched input, runs the anti-causal
// recurrence, writes the results over the segment in shared memory and hands
// it to a TMA store (in place: a segment's samples are no longer read once it
// has been stored).  Every mbarrier wait is bounded; a wait that runs out sets
// the timeout word and the CTA returns.
#include "kernels.cuh"
#include "tma.cuh"

// Shapes of the TMA-staged x / z passes (boxes of 256 y per CTA, lines per
// thread, stages in flight), chosen at run time per axis and line length by
// the smoothing schedule (set_smoothing_variant; libapr_b200.autotune times
// them and persists the choice).  Measured on 2048x2048x512 (B200): 1 box,
// 2 lines, 4 stages (three 64 KB CTAs per SM) x 4.27 / z 4.03 ms; 2 boxes,
// 4 lines, 3 stages 4.29 / 4.20; one CTA per SM with 8 stages 5.5 - 7.3 ms
// (too few warps for the recurrences' latency).

namespace aprb {

namespace {

constexpr int kTS = 16;     // samples per segment (one stage)
constexpr int kTBox = 256;  // y extent of one TMA box

template <int V>
struct LdV;
template <>
struct LdV<4> {
    __device__ __forceinline__ static void ld(const float *p, float *a) {
        const float4 v = *reinterpret_cast<const float4 *>(p);
        a[0] = v.x, a[1] = v.y, a[2] = v.z, a[3] = v.w;
    }
    __device__ __forceinline__ static void st(float *p, const float *a) {
        *reinterpret_cast<float4 *>(p) = make_float4(a[0], a[1], a[2], a[3]);
    }
};
template <>
struct LdV<2> {
    __device__ __forceinline__ static void ld(const float *p, float *a) {
        const float2 v = *reinterpret_cast<const float2 *>(p);
        a[0] = v.x, a[1] = v.y;
    }
    __device__ __forceinline__ static void st(float *p, const float *a) {
        *reinterpret_cast<float2 *>(p) = make_float2(a[0], a[1]);
    }
};
template <>
struct LdV<1> {
    __device__ __forceinline__ static void ld(const float *p, float *a) { a[0] = *p; }
    __device__ __forceinline__ static void st(float *p, const float *a) { *p = a[0]; }
};

template <int BOXES, int V, int STAGES>
struct TmaShape {
    static constexpr int kY = BOXES * kTBox;          // y columns (lines) of a CTA
    static constexpr int kThreads = kY / V;           // V neighbouring lines per thread
    static constexpr int kStageFloats = kTS * kY;
    // the stages, then the stages' mbarriers
    static constexpr size_t kSmem = sizeof(float) * STAGES * kStageFloats + 8 * STAGES;
};

// ZAXIS: lines along z (box 256 y x 1 x x 16 z, coordinates (y, o = x, i = z));
// else lines along x (box 256 y x 16 x x 1 z, coordinates (y, i = x, o = z)).
// A CTA owns BOXES * 256 consecutive y of plane o; thread t the V lines
// y0 + V t .. y0 + V t + V - 1.
template <bool ZAXIS, int BOXES, int V, int STAGES>
__global__ void __launch_bounds__(TmaShape<BOXES, V, STAGES>::kThreads)
    iir_strided_tma_kernel(const __grid_constant__ CUtensorMap tm, const float *__restrict__ im, int yn, int n,
                           uint64_t s1, uint64_t s2, IIRDev c, float2 *__restrict__ ckpt, uint64_t nlines,
                           unsigned *timeout) {
    using Sh = TmaShape<BOXES, V, STAGES>;
    constexpr int kY = Sh::kY, kSF = Sh::kStageFloats;
    extern __shared__ __align__(128) float tsm[];
    uint64_t *full = reinterpret_cast<uint64_t *>(tsm + (size_t)STAGES * kSF);
    const int ytiles = (yn + kY - 1) / kY;
    const int y0 = (int)(blockIdx.x % ytiles) * kY;
    const int o = (int)(blockIdx.x / ytiles);
    const int t = threadIdx.x;
    const int box = (V * t) / kTBox, col = (V * t) % kTBox;
    const int y = y0 + box * kTBox + col;
    const bool valid = y < yn;
    int nbox = 0;  // boxes of the CTA that start inside the image
    for (int b = 0; b < BOXES; ++b) nbox += (y0 + b * kTBox < yn) ? 1 : 0;
    const uint32_t stage_bytes = (uint32_t)nbox * (uint32_t)(kTS * kTBox * sizeof(float));
    const int nseg = (n + kTS - 1) / kTS;
    const int njobs = 2 * nseg;
    const uint64_t line = (uint64_t)o * (uint64_t)yn + (uint64_t)y;

    if (t == 0) {
        for (int i = 0; i < STAGES; ++i) mbar_init(&full[i], 1);
        mbar_fence_init();
    }
    __syncthreads();
    // job j < nseg: causal sweep over segment j; else anti-causal over segment 2 nseg - 1 - j
    auto issue = [&](int j) {
        if (j >= njobs) return;
        const int st = j % STAGES;
        float *S = tsm + (size_t)st * kSF;
        const int i0 = (j < nseg ? j : njobs - 1 - j) * kTS;
        mbar_arrive_expect_tx(&full[st], stage_bytes);
        for (int b = 0; b < nbox; ++b) {
            if (ZAXIS)
                tma_load_3d(S + b * kTS * kTBox, &tm, &full[st], y0 + b * kTBox, o, i0);
            else
                tma_load_3d(S + b * kTS * kTBox, &tm, &full[st], y0 + b * kTBox, i0, o);
        }
    };
    if (t == 0)
        for (int j = 0; j < STAGES; ++j) issue(j);

    // boundary sums over the first and last minLen samples (ComputeGradient.hpp:434-470)
    float v1[V] = {}, v2[V] = {}, v3[V] = {}, v4[V] = {};
    if (valid) {
        const float *L = im + (uint64_t)o * s2 + (uint64_t)y;
        for (int i = 0; i < c.minLen; ++i) {
            float a[V], b[V];
            LdV<V>::ld(L + (uint64_t)i * s1, a);
            LdV<V>::ld(L + (uint64_t)(n - 1 - i) * s1, b);
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
    }
    float p1[V], p2[V], q3[V], q4[V];
#pragma unroll
    for (int h = 0; h < V; ++h) p1[h] = v1[h], p2[h] = v2[h], q3[h] = v3[h], q4[h] = v4[h];

    for (int j = 0; j < njobs; ++j) {
        const int st = j % STAGES;
        const bool ok = mbar_wait_bounded(&full[st], (uint32_t)((j / STAGES) & 1));
        if (__syncthreads_or(!ok)) {
            if (t == 0) {
                atomicOr(timeout, 1u);
                // the loads issued for jobs j .. j + STAGES - 1 may still land: wait for them (bounded)
                for (int k = j; k < j + STAGES && k < njobs; ++k)
                    mbar_wait_bounded(&full[k % STAGES], (uint32_t)((k / STAGES) & 1));
                bulk_wait_all();
            }
            return;
        }
        float *S = tsm + (size_t)st * kSF + box * (kTS * kTBox) + col;
        const bool causal = j < nseg;
        const int sgm = causal ? j : njobs - 1 - j;
        const int i0 = sgm * kTS;
        float2 *ck = ckpt + (uint64_t)sgm * nlines + line;
        if (valid && causal) {
            // ---- causal sweep: the state at the segment start, then the segment
#pragma unroll
            for (int h = 0; h < V; ++h) ck[h] = make_float2(p1[h], p2[h]);
            if (i0 >= 2 && i0 + kTS <= n) {
#pragma unroll
                for (int u = 0; u < kTS; ++u) {
                    float a[V];
                    LdV<V>::ld(S + u * kTBox, a);
#pragma unroll
                    for (int h = 0; h < V; ++h) {
                        const float nv = a[h] + c.b1 * p1[h] + c.b2 * p2[h];
                        p2[h] = p1[h];
                        p1[h] = nv;
                    }
                }
            } else {
                const int i1 = min(n, i0 + kTS);
                for (int i = max(i0, 2); i < i1; ++i) {
                    float a[V];
                    LdV<V>::ld(S + (i - i0) * kTBox, a);
#pragma unroll
                    for (int h = 0; h < V; ++h) {
                        const float nv = a[h] + c.b1 * p1[h] + c.b2 * p2[h];
                        p2[h] = p1[h];
                        p1[h] = nv;
                    }
                }
            }
        } else if (valid) {
            // ---- anti-causal sweep, recomputing the segment's causal values
            float r1[V], r2[V];
#pragma unroll
            for (int h = 0; h < V; ++h) {
                const float2 q = ck[h];
                r1[h] = q.x;
                r2[h] = q.y;
            }
            float buf[kTS][V];
            if (i0 >= 2 && i0 + kTS <= n - 2) {
#pragma unroll
                for (int u = 0; u < kTS; ++u) {
                    float a[V];
                    LdV<V>::ld(S + u * kTBox, a);
#pragma unroll
                    for (int h = 0; h < V; ++h) {
                        const float nv = a[h] + c.b1 * r1[h] + c.b2 * r2[h];
                        r2[h] = r1[h];
                        r1[h] = nv;
                        buf[u][h] = nv;
                    }
                }
#pragma unroll
                for (int u = kTS - 1; u >= 0; --u) {
#pragma unroll
                    for (int h = 0; h < V; ++h) {
                        const float temp = buf[u][h] + c.b1 * q3[h] + c.b2 * q4[h];
                        buf[u][h] = temp * c.norm;
                        q4[h] = q3[h];
                        q3[h] = temp;
                    }
                    LdV<V>::st(S + u * kTBox, buf[u]);
                }
            } else {
                const int i1 = min(n, i0 + kTS);
#pragma unroll
                for (int u = 0; u < kTS; ++u) {
                    const int i = i0 + u;
                    if (i >= i1) break;
                    float a[V] = {};
                    if (i >= 2) LdV<V>::ld(S + u * kTBox, a);
#pragma unroll
                    for (int h = 0; h < V; ++h) {
                        float f;
                        if (i == 0) {
                            f = v2[h];
                        } else if (i == 1) {
                            f = v1[h];
                        } else {
                            f = a[h] + c.b1 * r1[h] + c.b2 * r2[h];
                            r2[h] = r1[h];
                            r1[h] = f;
                        }
                        buf[u][h] = f;
                    }
                }
#pragma unroll
                for (int u = kTS - 1; u >= 0; --u) {
                    const int i = i0 + u;
                    if (i >= i1) continue;
#pragma unroll
                    for (int h = 0; h < V; ++h) {
                        float out;
                        if (i == n - 1) {
                            out = v4[h] * c.norm;
                        } else if (i == n - 2) {
                            out = v3[h] * c.norm;
                        } else {
                            const float temp = buf[u][h] + c.b1 * q3[h] + c.b2 * q4[h];
                            out = temp * c.norm;
                            q4[h] = q3[h];
                            q3[h] = temp;
                        }
                        buf[u][h] = out;
                    }
                    LdV<V>::st(S + u * kTBox, buf[u]);
                }
            }
        }
        if (!causal) fence_proxy_async_smem();
        __syncthreads();
        if (t == 0) {
            if (!causal) {
                float *SS = tsm + (size_t)st * kSF;
                for (int b = 0; b < nbox; ++b) {
                    if (ZAXIS)
                        tma_store_3d(&tm, SS + b * kTS * kTBox, y0 + b * kTBox, o, i0);
                    else
                        tma_store_3d(&tm, SS + b * kTS * kTBox, y0 + b * kTBox, i0, o);
                }
                bulk_commit();
                bulk_wait_read_all();  // the stage is loaded again below
            }
            issue(j + STAGES);
        }
    }
    if (t == 0) bulk_wait_all();
}

template <bool ZAXIS, int BOXES, int V, int STAGES>
void launch_tma_variant(const CUtensorMap &tm, float *work, int yn, int n, int m, uint64_t s1, uint64_t s2,
                        const IIRDev &c, float2 *ckpt, unsigned *d_timeout, cudaStream_t s) {
    using Sh = TmaShape<BOXES, V, STAGES>;
    auto kern = iir_strided_tma_kernel<ZAXIS, BOXES, V, STAGES>;
    set_smem_once<iir_strided_tma_kernel<ZAXIS, BOXES, V, STAGES>>((int)Sh::kSmem);
    const unsigned blocks = (unsigned)((uint64_t)((yn + Sh::kY - 1) / Sh::kY) * (uint64_t)m);
    kern<<<blocks, Sh::kThreads, Sh::kSmem, s>>>(tm, work, yn, n, s1, s2, c, ckpt, (uint64_t)yn * (uint64_t)m,
                                                 d_timeout);
    count_launch();
    APRB_CHECK_LAUNCH();
}

}  // namespace

// ---------------------------------------------------------------------------
// smoothing schedule: the kernel variant per axis and line-length bucket
namespace {
int g_sched[3][kSchedBuckets] = {{1, 1, 1, 1, 1, 1}, {1, 1, 1, 1, 1, 1}, {1, 1, 1, 1, 1, 1}};
constexpr int kVariants[3] = {3, 5, 5};
}  // namespace

int sched_bucket(int n) {
    int b = 0;
    for (int lim = 128; b < kSchedBuckets - 1 && n > lim; lim *= 2) ++b;
    return b;
}
int smoothing_variants(int axis) { return axis >= 0 && axis < 3 ? kVariants[axis] : 0; }
int smoothing_variant(int axis, int n) {
    return __atomic_load_n(&g_sched[axis][sched_bucket(n)], __ATOMIC_RELAXED);
}
bool set_smoothing_variant(int axis, int bucket, int v) {
    if (axis < 0 || axis > 2 || bucket < 0 || bucket >= kSchedBuckets || v < 0 || v >= kVariants[axis]) return false;
    __atomic_store_n(&g_sched[axis][bucket], v, __ATOMIC_RELAXED);
    return true;
}

bool launch_strided_iir_tma(float *work, int yn, int xn, int zn, bool zaxis, const IIRDev &c, unsigned *d_timeout,
                            float2 *ckpt, uint64_t ckpt_elems, cudaStream_t s) {
    const int n = zaxis ? zn : xn, m = zaxis ? xn : zn;
    const int variant = smoothing_variant(zaxis ? 2 : 1, n);
    if (variant == 0) return false;  // the register-staged kernel
    if (yn % 4 != 0 || yn < kTBox || n < kTS || ((uintptr_t)work & 15) != 0 || ((uintptr_t)ckpt & 15) != 0)
        return false;
    if ((uint64_t)yn * (uint64_t)m * (uint64_t)((n + kTS - 1) / kTS) > ckpt_elems) return false;
    CUtensorMap tm;
    const uint64_t d[3] = {(uint64_t)yn, (uint64_t)xn, (uint64_t)zn};
    const uint32_t box[3] = {(uint32_t)kTBox, zaxis ? 1u : (uint32_t)kTS, zaxis ? (uint32_t)kTS : 1u};
    if (!make_tensor_map_3d_f32(&tm, work, d, (uint64_t)yn * 4, (uint64_t)xn * yn * 4, box)) return false;
    const uint64_t s1 = zaxis ? (uint64_t)xn * yn : (uint64_t)yn, s2 = zaxis ? (uint64_t)yn : (uint64_t)xn * yn;
    // variants: 1 = (1 box, 2 lines, 4 stages), 2 = (2, 4, 3), 3 = (1, 1, 4), 4 = (2, 2, 3)
#define APRB_TMA_LAUNCH(Z, B, V, S) launch_tma_variant<Z, B, V, S>(tm, work, yn, n, m, s1, s2, c, ckpt, d_timeout, s)
    if (zaxis) {
        switch (variant) {
            case 2: APRB_TMA_LAUNCH(true, 2, 4, 3); break;
            case 3: APRB_TMA_LAUNCH(true, 1, 1, 4); break;
            case 4: APRB_TMA_LAUNCH(true, 2, 2, 3); break;
            default: APRB_TMA_LAUNCH(true, 1, 2, 4); break;
        }
    } else {
        switch (variant) {
            case 2: APRB_TMA_LAUNCH(false, 2, 4, 3); break;
            case 3: APRB_TMA_LAUNCH(false, 1, 1, 4); break;
            case 4: APRB_TMA_LAUNCH(false, 2, 2, 3); break;
            default: APRB_TMA_LAUNCH(false, 1, 2, 4); break;
        }
    }
#undef APRB_TMA_LAUNCH
    return true;
}

}  // namespace aprb

// ---------------------------------------------------------------------------
// host: tiled tensor maps through the driver entry point
#include <cudaTypedefs.h>

#include <mutex>

namespace aprb {

namespace {
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;
}  // namespace

// (map == nullptr: only looks the driver's encoder up)
bool make_tensor_map_3d_f32(CUtensorMap *map, const void *base, const uint64_t d[3], uint64_t s1, uint64_t s2,
                            const uint32_t b[3]) {
    std::call_once(g_encode_once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_encode = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    auto encode = g_encode;
    if (!map) return encode != nullptr;
    if (!encode || ((uintptr_t)base & 15) != 0 || (s1 & 15) != 0 || (s2 & 15) != 0) return false;
    cuuint64_t gdim[3] = {d[0], d[1], d[2]};
    cuuint64_t gstride[2] = {s1, s2};
    cuuint32_t box[3] = {b[0], b[1], b[2]};
    cuuint32_t estride[3] = {1, 1, 1};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void *>(base), gdim, gstride, box,
                              estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

bool make_tensor_map_2d_sw128(CUtensorMap *map, const void *base, bool f32, const uint64_t d[2], uint64_t s1,
                              const uint32_t b[2]) {
    make_tensor_map_3d_f32(nullptr, nullptr, nullptr, 0, 0, nullptr);  // looks the encoder up
    if (!g_encode || ((uintptr_t)base & 15) != 0 || (s1 & 15) != 0) return false;
    cuuint64_t gdim[2] = {d[0], d[1]};
    cuuint64_t gstride[1] = {s1};
    cuuint32_t box[2] = {b[0], b[1]};
    cuuint32_t estride[2] = {1, 1};
    const CUresult r =
        g_encode(map, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, const_cast<void *>(base),
                 gdim, gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace aprb
