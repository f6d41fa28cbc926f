// a2 (x, z) for float ImageType: bspline_filt_rec_x (ComputeGradient.hpp:602-779)
// and bspline_filt_rec_z (:416-599) with TMA-staged segments.
//
// A CTA owns 512 consecutive y of one plane of the other axis (one x row for
// the z pass, one z plane for the x pass): 512 lines along the filtered axis,
// four neighbouring lines per thread.  The lines move through shared memory in
// segments of 16 samples, each segment two cp.async.bulk.tensor boxes of
// 256 y x 16 samples (2 KB contiguous per sample), in a ring of three stages
// whose mbarriers the copy engine completes; a CTA keeps up to three segments
// (96 KB) in flight without spending registers on them.
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

namespace aprb {

namespace {

constexpr int kTS = 16;                // samples per segment (one stage)
constexpr int kTBox = 256;             // y extent of one TMA box
constexpr int kTY = 2 * kTBox;         // y columns (lines) of a CTA
constexpr int kTThreads = kTY / 4;     // four lines per thread
constexpr int kTStages = 3;            // segments in flight per CTA
constexpr int kStageFloats = kTS * kTY;
// the stages, then the stages' mbarriers
constexpr size_t kTSmem = sizeof(float) * kTStages * kStageFloats + 8 * kTStages;

__device__ __forceinline__ void ld4(const float *p, float *a) {
    const float4 v = *reinterpret_cast<const float4 *>(p);
    a[0] = v.x, a[1] = v.y, a[2] = v.z, a[3] = v.w;
}
__device__ __forceinline__ void st4(float *p, const float *a) {
    *reinterpret_cast<float4 *>(p) = make_float4(a[0], a[1], a[2], a[3]);
}

// ZAXIS: lines along z (box 256 y x 1 x x 16 z, coordinates (y, o = x, i = z));
// else lines along x (box 256 y x 16 x x 1 z, coordinates (y, i = x, o = z)).
template <bool ZAXIS>
__global__ void __launch_bounds__(kTThreads, 2)
    iir_strided_tma_kernel(const __grid_constant__ CUtensorMap tm, const float *__restrict__ im, int yn, int n,
                           uint64_t s1, uint64_t s2, IIRDev c, float2 *__restrict__ ckpt, uint64_t nlines,
                           unsigned *timeout) {
    extern __shared__ __align__(128) float tsm[];
    uint64_t *full = reinterpret_cast<uint64_t *>(tsm + (size_t)kTStages * kStageFloats);
    const int ytiles = (yn + kTY - 1) / kTY;
    const int y0 = (int)(blockIdx.x % ytiles) * kTY;
    const int o = (int)(blockIdx.x / ytiles);
    const int t = threadIdx.x;
    const int half = t / (kTBox / 4), col = 4 * (t % (kTBox / 4));
    const int y = y0 + half * kTBox + col;
    const bool valid = y < yn;
    const bool second = y0 + kTBox < yn;
    const uint32_t stage_bytes = (second ? 2u : 1u) * (uint32_t)(kTS * kTBox * sizeof(float));
    const int nseg = (n + kTS - 1) / kTS;
    const int njobs = 2 * nseg;
    const uint64_t line = (uint64_t)o * (uint64_t)yn + (uint64_t)y;

    if (t == 0) {
        for (int i = 0; i < kTStages; ++i) mbar_init(&full[i], 1);
        mbar_fence_init();
    }
    __syncthreads();
    // job j < nseg: causal sweep over segment j; else anti-causal over segment 2 nseg - 1 - j
    auto issue = [&](int j) {
        if (j >= njobs) return;
        const int st = j % kTStages;
        float *S = tsm + (size_t)st * kStageFloats;
        const int i0 = (j < nseg ? j : njobs - 1 - j) * kTS;
        mbar_arrive_expect_tx(&full[st], stage_bytes);
        if (ZAXIS) {
            tma_load_3d(S, &tm, &full[st], y0, o, i0);
            if (second) tma_load_3d(S + kTS * kTBox, &tm, &full[st], y0 + kTBox, o, i0);
        } else {
            tma_load_3d(S, &tm, &full[st], y0, i0, o);
            if (second) tma_load_3d(S + kTS * kTBox, &tm, &full[st], y0 + kTBox, i0, o);
        }
    };
    if (t == 0)
        for (int j = 0; j < kTStages; ++j) issue(j);

    // boundary sums over the first and last minLen samples (ComputeGradient.hpp:434-470)
    float v1[4] = {}, v2[4] = {}, v3[4] = {}, v4[4] = {};
    if (valid) {
        const float *L = im + (uint64_t)o * s2 + (uint64_t)y;
        for (int i = 0; i < c.minLen; ++i) {
            float a[4], b[4];
            ld4(L + (uint64_t)i * s1, a);
            ld4(L + (uint64_t)(n - 1 - i) * s1, b);
            const float k1 = __ldg(c.bc + i), k2 = __ldg(c.bc + c.minLen + i);
            const float k3 = __ldg(c.bc + 2 * c.minLen + i), k4 = __ldg(c.bc + 3 * c.minLen + i);
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                v1[h] = v1[h] + k1 * a[h];
                v2[h] = v2[h] + k2 * a[h];
                v3[h] = v3[h] + k3 * b[h];
                v4[h] = v4[h] + k4 * b[h];
            }
        }
    }
    float p1[4], p2[4], q3[4], q4[4];
#pragma unroll
    for (int h = 0; h < 4; ++h) p1[h] = v1[h], p2[h] = v2[h], q3[h] = v3[h], q4[h] = v4[h];

    for (int j = 0; j < njobs; ++j) {
        const int st = j % kTStages;
        const bool ok = mbar_wait_bounded(&full[st], (uint32_t)((j / kTStages) & 1));
        if (__syncthreads_or(!ok)) {
            if (t == 0) {
                atomicOr(timeout, 1u);
                // the loads issued for jobs j .. j + kTStages - 1 may still land: wait for them (bounded)
                for (int k = j; k < j + kTStages && k < njobs; ++k)
                    mbar_wait_bounded(&full[k % kTStages], (uint32_t)((k / kTStages) & 1));
                bulk_wait_all();
            }
            return;
        }
        float *S = tsm + (size_t)st * kStageFloats + half * (kTS * kTBox) + col;
        const bool causal = j < nseg;
        const int sgm = causal ? j : njobs - 1 - j;
        const int i0 = sgm * kTS;
        float2 *ck = ckpt + (uint64_t)sgm * nlines + line;
        if (valid && causal) {
            // ---- causal sweep: the state at the segment start, then the segment
            reinterpret_cast<float4 *>(ck)[0] = make_float4(p1[0], p2[0], p1[1], p2[1]);
            reinterpret_cast<float4 *>(ck)[1] = make_float4(p1[2], p2[2], p1[3], p2[3]);
            if (i0 >= 2 && i0 + kTS <= n) {
#pragma unroll
                for (int u = 0; u < kTS; ++u) {
                    float a[4];
                    ld4(S + u * kTBox, a);
#pragma unroll
                    for (int h = 0; h < 4; ++h) {
                        const float nv = a[h] + c.b1 * p1[h] + c.b2 * p2[h];
                        p2[h] = p1[h];
                        p1[h] = nv;
                    }
                }
            } else {
                const int i1 = min(n, i0 + kTS);
                for (int i = max(i0, 2); i < i1; ++i) {
                    float a[4];
                    ld4(S + (i - i0) * kTBox, a);
#pragma unroll
                    for (int h = 0; h < 4; ++h) {
                        const float nv = a[h] + c.b1 * p1[h] + c.b2 * p2[h];
                        p2[h] = p1[h];
                        p1[h] = nv;
                    }
                }
            }
        } else if (valid) {
            // ---- anti-causal sweep, recomputing the segment's causal values
            const float4 c0 = reinterpret_cast<const float4 *>(ck)[0];
            const float4 c1 = reinterpret_cast<const float4 *>(ck)[1];
            float r1[4] = {c0.x, c0.z, c1.x, c1.z}, r2[4] = {c0.y, c0.w, c1.y, c1.w};
            float buf[kTS][4];
            if (i0 >= 2 && i0 + kTS <= n - 2) {
#pragma unroll
                for (int u = 0; u < kTS; ++u) {
                    float a[4];
                    ld4(S + u * kTBox, a);
#pragma unroll
                    for (int h = 0; h < 4; ++h) {
                        const float nv = a[h] + c.b1 * r1[h] + c.b2 * r2[h];
                        r2[h] = r1[h];
                        r1[h] = nv;
                        buf[u][h] = nv;
                    }
                }
#pragma unroll
                for (int u = kTS - 1; u >= 0; --u) {
#pragma unroll
                    for (int h = 0; h < 4; ++h) {
                        const float temp = buf[u][h] + c.b1 * q3[h] + c.b2 * q4[h];
                        buf[u][h] = temp * c.norm;
                        q4[h] = q3[h];
                        q3[h] = temp;
                    }
                    st4(S + u * kTBox, buf[u]);
                }
            } else {
                const int i1 = min(n, i0 + kTS);
#pragma unroll
                for (int u = 0; u < kTS; ++u) {
                    const int i = i0 + u;
                    if (i >= i1) break;
                    float a[4] = {};
                    if (i >= 2) ld4(S + u * kTBox, a);
#pragma unroll
                    for (int h = 0; h < 4; ++h) {
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
                    for (int h = 0; h < 4; ++h) {
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
                    st4(S + u * kTBox, buf[u]);
                }
            }
        }
        if (!causal) fence_proxy_async_smem();
        __syncthreads();
        if (t == 0) {
            if (!causal) {
                float *SS = tsm + (size_t)st * kStageFloats;
                if (ZAXIS) {
                    tma_store_3d(&tm, SS, y0, o, i0);
                    if (second) tma_store_3d(&tm, SS + kTS * kTBox, y0 + kTBox, o, i0);
                } else {
                    tma_store_3d(&tm, SS, y0, i0, o);
                    if (second) tma_store_3d(&tm, SS + kTS * kTBox, y0 + kTBox, i0, o);
                }
                bulk_commit();
                bulk_wait_read_all();  // the stage is loaded again below
            }
            issue(j + kTStages);
        }
    }
    if (t == 0) bulk_wait_all();
}

}  // namespace

bool launch_strided_iir_tma(float *work, int yn, int xn, int zn, bool zaxis, const IIRDev &c, unsigned *d_timeout,
                            float2 *ckpt, uint64_t ckpt_elems, cudaStream_t s) {
    const int n = zaxis ? zn : xn, m = zaxis ? xn : zn;
    if (yn % 4 != 0 || yn < kTBox || n < kTS || ((uintptr_t)work & 15) != 0 || ((uintptr_t)ckpt & 15) != 0)
        return false;
    if ((uint64_t)yn * (uint64_t)m * (uint64_t)((n + kTS - 1) / kTS) > ckpt_elems) return false;
    CUtensorMap tm;
    const uint64_t d[3] = {(uint64_t)yn, (uint64_t)xn, (uint64_t)zn};
    const uint32_t box[3] = {(uint32_t)kTBox, zaxis ? 1u : (uint32_t)kTS, zaxis ? (uint32_t)kTS : 1u};
    if (!make_tensor_map_3d_f32(&tm, work, d, (uint64_t)yn * 4, (uint64_t)xn * yn * 4, box)) return false;
    auto kern = zaxis ? iir_strided_tma_kernel<true> : iir_strided_tma_kernel<false>;
    APRB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTSmem));
    const uint64_t nlines = (uint64_t)yn * (uint64_t)m;
    const uint64_t s1 = zaxis ? (uint64_t)xn * yn : (uint64_t)yn, s2 = zaxis ? (uint64_t)yn : (uint64_t)xn * yn;
    const unsigned blocks = (unsigned)((uint64_t)((yn + kTY - 1) / kTY) * (uint64_t)m);
    kern<<<blocks, kTThreads, kTSmem, s>>>(tm, work, yn, n, s1, s2, c, ckpt, nlines, d_timeout);
    count_launch();
    APRB_CHECK_LAUNCH();
    return true;
}

}  // namespace aprb

// ---------------------------------------------------------------------------
// host: tiled tensor maps through the driver entry point
#include <cudaTypedefs.h>

#include <mutex>

namespace aprb {

bool make_tensor_map_3d_f32(CUtensorMap *map, const void *base, const uint64_t d[3], uint64_t s1, uint64_t s2,
                            const uint32_t b[3]) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
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

}  // namespace aprb
