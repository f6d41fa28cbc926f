// a2 (y) for float ImageType: bspline_filt_rec_y (ComputeGradient.hpp:249-413)
// with TMA-staged tiles.
//
// A CTA is one warp and owns 32 consecutive y-lines (rows of the (y, line)
// view of the volume); lane r runs line r's recurrences.  The uint16 input
// moves in tiles of 64 samples x 32 lines (one cp.async.bulk.tensor box of
// 4 KB) through a ring of stages with mbarriers, swizzled by the copy engine
// (128-byte rows, 16-byte chunk j of row r at j ^ (r % 8)) so that a lane
// reads eight samples of its own line in one conflict-free 16-byte load.
// The recurrences are those of iir_y_rc_kernel (pipeline.cu) operation for
// operation: the causal sweep keeps the state at every tile start (ckpt);
// the anti-causal sweep recomputes each tile's causal values from it and
// writes the results into a swizzled float tile that two TMA stores (32 y x
// 32 lines each) put back in place.  Every mbarrier wait is bounded; a wait
// that runs out sets the timeout word and the CTA returns.
#include "kernels.cuh"
#include "tma.cuh"

// Input stages in flight per warp: 2 (variant 1) or 3 (variant 2) of the
// smoothing schedule.  Measured on 2048x2048x512 (B200): 2 stages (17 KB per
// CTA, 13 warps per SM) 2.97 ms, 3 stages 3.00, 4 stages 3.31, 6 stages 3.94
// (fewer resident warps); the cp.async-staged kernel (variant 0) 4.30 ms.

namespace aprb {

namespace {

constexpr int kYT = 64;                            // samples per tile
constexpr uint32_t kYInBytes = 32u * kYT * 2u;     // 32 lines x 64 uint16
constexpr uint32_t kYOutBytes = 32u * kYT * 4u;    // 2 boxes of 32 lines x 32 floats

template <int STAGES>
struct YShape {
    // 1024-byte alignment slack, the input stages, the output tile, the mbarriers
    static constexpr size_t kSmem = 1024 + STAGES * kYInBytes + kYOutBytes + 8 * STAGES;
};

// 16-byte chunk j (samples 8j .. 8j+7) of row r of a swizzled input tile
__device__ __forceinline__ uint4 in_chunk(const uint8_t *st, int r, int j) {
    return *reinterpret_cast<const uint4 *>(st + r * 128 + ((j ^ (r & 7)) << 4));
}
__device__ __forceinline__ float in_sample(const uint8_t *st, int r, int k) {
    return (float)*reinterpret_cast<const uint16_t *>(st + r * 128 + (((k >> 3) ^ (r & 7)) << 4) + ((k & 7) << 1));
}
// sample k (0 .. 63) of row r of the swizzled output tile (two 32-float boxes)
__device__ __forceinline__ float *out_at(uint8_t *ot, int r, int k) {
    const int h = k >> 5, kk = k & 31;
    return reinterpret_cast<float *>(ot + h * 4096 + r * 128 + (((kk >> 2) ^ (r & 7)) << 4) + ((kk & 3) << 2));
}

template <int STAGES>
__global__ void __launch_bounds__(32)
    iir_y_tma_kernel(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tout,
                     const uint16_t *__restrict__ src, int yn, uint64_t nlines, IIRDev c, float2 *__restrict__ ckpt,
                     unsigned *timeout) {
    extern __shared__ uint8_t ysm_raw[];
    uint8_t *sm = ysm_raw + ((1024u - (smem_addr(ysm_raw) & 1023u)) & 1023u);
    uint8_t *in = sm;
    uint8_t *ot = sm + STAGES * kYInBytes;
    uint64_t *full = reinterpret_cast<uint64_t *>(ot + kYOutBytes);
    const int lane = threadIdx.x;
    const uint64_t line0 = (uint64_t)blockIdx.x * 32;
    const uint64_t myline = line0 + lane;
    const bool valid = myline < nlines;
    const int ntile = (yn + kYT - 1) / kYT;
    const int njobs = 2 * ntile;
    if (lane == 0) {
        for (int i = 0; i < STAGES; ++i) mbar_init(&full[i], 1);
        mbar_fence_init();
    }
    __syncwarp();
    // job j < ntile: causal sweep over tile j; else anti-causal over tile 2 ntile - 1 - j
    auto issue = [&](int j) {
        if (j >= njobs) return;
        const int st = j % STAGES;
        const int t = j < ntile ? j : njobs - 1 - j;
        mbar_arrive_expect_tx(&full[st], kYInBytes);
        tma_load_2d(in + st * kYInBytes, &tin, &full[st], t * kYT, (int)line0);
    };
    if (lane == 0)
        for (int j = 0; j < STAGES; ++j) issue(j);

    float t1 = 0, t2 = 0, t3 = 0, t4 = 0;
    if (valid) {
        const uint16_t *L = src + myline * (uint64_t)yn;
        for (int k = 0; k < c.minLen; ++k) {
            const float v = (float)L[k];
            t1 = t1 + __ldg(c.bc + k) * v;
            t2 = t2 + __ldg(c.bc + c.minLen + k) * v;
        }
        for (int k = 0; k < c.minLen; ++k) {
            const float v = (float)L[yn - 1 - k];
            t3 = t3 + __ldg(c.bc + 2 * c.minLen + k) * v;
            t4 = t4 + __ldg(c.bc + 3 * c.minLen + k) * v;
        }
    }
    float b2v = 0, b1v = 0;
    if (valid) {
        b2v = (t4 * c.norm) / c.norm;
        b1v = (t3 * c.norm) / c.norm;
    }

    for (int j = 0; j < njobs; ++j) {
        const int st = j % STAGES;
        const bool ok = mbar_wait_bounded(&full[st], (uint32_t)((j / STAGES) & 1));
        if (__any_sync(0xffffffffu, !ok)) {
            if (lane == 0) {
                atomicOr(timeout, 1u);
                for (int k = j; k < j + STAGES && k < njobs; ++k)
                    mbar_wait_bounded(&full[k % STAGES], (uint32_t)((k / STAGES) & 1));
                bulk_wait_all();
            }
            return;
        }
        const uint8_t *S = in + st * kYInBytes;
        const bool causal = j < ntile;
        const int t = causal ? j : njobs - 1 - j;
        const int y0 = t * kYT;
        if (causal) {
            // ---- causal sweep: the state at every tile start
            if (valid) {
                ckpt[(uint64_t)t * nlines + myline] = make_float2(t1, t2);
                if (y0 >= 2 && y0 + kYT <= yn) {
#pragma unroll
                    for (int q = 0; q < kYT / 8; ++q) {
                        const uint4 w = in_chunk(S, lane, q);
                        const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
                        for (int e = 0; e < 8; ++e) {
                            const float v = (float)((e & 1) ? (ws[e >> 1] >> 16) : (ws[e >> 1] & 0xffffu));
                            const float temp = t1 * c.b1 + t2 * c.b2 + v;
                            t2 = t1;
                            t1 = temp;
                        }
                    }
                } else {
                    const int kend = min(kYT, yn - y0);
                    for (int k = 0; k < kend; ++k) {
                        if (y0 + k < 2) continue;
                        const float temp = t1 * c.b1 + t2 * c.b2 + in_sample(S, lane, k);
                        t2 = t1;
                        t1 = temp;
                    }
                }
            }
            __syncwarp();
            if (lane == 0) issue(j + STAGES);
            continue;
        }
        // ---- anti-causal sweep, recomputing the tile's causal values
        if (lane == 0) bulk_wait_read_all();  // the previous tile's stores have read the output tile
        __syncwarp();
        if (valid) {
            const float2 stt = ckpt[(uint64_t)t * nlines + myline];
            float r1 = stt.x, r2 = stt.y;
            if (y0 >= 2 && y0 + kYT <= yn - 2) {
                float F[kYT];
#pragma unroll
                for (int q = 0; q < kYT / 8; ++q) {
                    const uint4 w = in_chunk(S, lane, q);
                    const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        const float v = (float)((e & 1) ? (ws[e >> 1] >> 16) : (ws[e >> 1] & 0xffffu));
                        const float temp = r1 * c.b1 + r2 * c.b2 + v;
                        F[8 * q + e] = temp;
                        r2 = r1;
                        r1 = temp;
                    }
                }
#pragma unroll
                for (int k = kYT - 1; k >= 0; --k) {
                    const float temp = b1v * c.b1 + b2v * c.b2 + F[k];
                    F[k] = temp * c.norm;
                    b2v = b1v;
                    b1v = temp;
                }
#pragma unroll
                for (int q = 0; q < kYT / 4; ++q)
                    *reinterpret_cast<float4 *>(out_at(ot, lane, 4 * q)) =
                        make_float4(F[4 * q], F[4 * q + 1], F[4 * q + 2], F[4 * q + 3]);
            } else {
                const int kend = min(kYT, yn - y0);
                for (int k = 0; k < kend; ++k) {
                    const int y = y0 + k;
                    float out;
                    if (y == 0) {
                        out = r2;
                    } else if (y == 1) {
                        out = r1;
                    } else {
                        const float temp = r1 * c.b1 + r2 * c.b2 + in_sample(S, lane, k);
                        out = temp;
                        r2 = r1;
                        r1 = temp;
                    }
                    if (y == yn - 2) out = t3 * c.norm;
                    if (y == yn - 1) out = t4 * c.norm;
                    *out_at(ot, lane, k) = out;
                }
                for (int k = kend - 1; k >= 0; --k) {
                    if (y0 + k > yn - 3) continue;
                    float *f = out_at(ot, lane, k);
                    const float temp = b1v * c.b1 + b2v * c.b2 + *f;
                    *f = temp * c.norm;
                    b2v = b1v;
                    b1v = temp;
                }
            }
        }
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
            tma_store_2d(&tout, ot, y0, (int)line0);
            if (y0 + 32 < yn) tma_store_2d(&tout, ot + 4096, y0 + 32, (int)line0);
            bulk_commit();
            issue(j + STAGES);
        }
    }
    if (lane == 0) bulk_wait_all();
}

}  // namespace

bool launch_iir_y_tma(const uint16_t *img, float *work, int yn, uint64_t nlines, const IIRDev &c, unsigned *d_timeout,
                      float2 *ckpt, uint64_t ckpt_elems, cudaStream_t s) {
    const int variant = smoothing_variant(0, yn);
    if (variant == 0) return false;  // the cp.async-staged kernel
    if (yn % 8 != 0 || yn < kYT || nlines < 32 || nlines > (uint64_t)INT32_MAX || ((uintptr_t)img & 15) != 0 ||
        ((uintptr_t)work & 15) != 0 || ((uintptr_t)ckpt & 7) != 0)
        return false;
    const uint64_t ntile = (uint64_t)((yn + kYT - 1) / kYT);
    if (ntile * nlines > ckpt_elems) return false;
    CUtensorMap tin, tout;
    const uint64_t d[2] = {(uint64_t)yn, nlines};
    const uint32_t bin[2] = {(uint32_t)kYT, 32u}, bout[2] = {32u, 32u};
    if (!make_tensor_map_2d_sw128(&tin, img, false, d, (uint64_t)yn * 2, bin)) return false;
    if (!make_tensor_map_2d_sw128(&tout, work, true, d, (uint64_t)yn * 4, bout)) return false;
    if (variant == 2) {
        set_smem_once<iir_y_tma_kernel<3>>((int)YShape<3>::kSmem);
        iir_y_tma_kernel<3><<<(unsigned)((nlines + 31) / 32), 32, YShape<3>::kSmem, s>>>(tin, tout, img, yn, nlines, c,
                                                                                        ckpt, d_timeout);
    } else {
        set_smem_once<iir_y_tma_kernel<2>>((int)YShape<2>::kSmem);
        iir_y_tma_kernel<2><<<(unsigned)((nlines + 31) / 32), 32, YShape<2>::kSmem, s>>>(tin, tout, img, yn, nlines, c,
                                                                                        ckpt, d_timeout);
    }
    count_launch();
    APRB_CHECK_LAUNCH();
    return true;
}

}  // namespace aprb
