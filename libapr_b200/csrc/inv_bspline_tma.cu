// a5: calc_inv_bspline_y/x/z (ComputeGradient.hpp:785-964) with TMA-staged
// planes.  A CTA owns 248 (y) x 16 (x) columns of the ds image and a run of
// up to 32 planes, and streams along z; thread t owns y = y0 + t.  Each input
// plane arrives as one cp.async.bulk.tensor box of 256 y x 18 x (from y0 - 4,
// so the box starts on a 16-byte boundary, and x0 - 1: the one-sample halo;
// samples outside the image read as zero and are not used) into a ring of
// three stages; the thread runs the y pass of its y on the 18 rows, the x pass
// of its 16 outputs and the z pass from the last three planes it holds in
// registers.  The arithmetic is inv_bspline_kernel's (pipeline.cu), operand
// for operand, so the result is the same bits.  Every mbarrier wait is
// bounded; a wait that runs out sets the timeout word and the CTA returns.
#include "kernels.cuh"
#include "tma.cuh"

namespace aprb {

namespace {

constexpr int kVY = 248, kVX = 16, kVZ = 32;  // outputs per CTA: y, x, planes per run
constexpr int kVBoxY = 256, kVBoxX = kVX + 2;  // the loaded box: y from y0 - 4, x from x0 - 1
constexpr int kVStages = 3;  // 0.79 ms on the 1024x1024x256 ds image (4 stages: 0.90, 2: 0.80)
constexpr int kVThreads = 256;
constexpr uint32_t kVPlaneBytes = kVBoxY * kVBoxX * 4;
constexpr size_t kVSmem = (size_t)kVStages * kVPlaneBytes + 8 * kVStages;

__global__ void __launch_bounds__(kVThreads)
    inv_bspline_tma_kernel(const __grid_constant__ CUtensorMap tm, float *__restrict__ O, int yd, int xd, int zd,
                           int ony, int onx, int onz, InvB c, unsigned *timeout) {
    extern __shared__ __align__(128) float vsm[];
    uint64_t *full = reinterpret_cast<uint64_t *>(vsm + (size_t)kVStages * kVBoxY * kVBoxX);
    const int y0 = blockIdx.x * kVY, x0 = blockIdx.y * kVX, zs = blockIdx.z * kVZ;
    const int ze = min(zs + kVZ, zd);
    const int zb = zs == 0 ? 0 : zs - 1;            // first plane read
    const int zl = onz ? min(ze, zd - 1) : ze - 1;  // last plane read
    const int nplanes = zl - zb + 1;
    const int t = threadIdx.x;
    if (t == 0) {
        for (int i = 0; i < kVStages; ++i) mbar_init(&full[i], 1);
        mbar_fence_init();
    }
    __syncthreads();
    auto issue = [&](int k) {  // k-th plane of the run into stage k % kVStages
        if (k >= nplanes) return;
        const int st = k % kVStages;
        mbar_arrive_expect_tx(&full[st], kVPlaneBytes);
        tma_load_3d(vsm + (size_t)st * kVBoxY * kVBoxX, &tm, &full[st], y0 - 4, x0 - 1, zb + k);
    };
    if (t == 0)
        for (int k = 0; k < kVStages; ++k) issue(k);
    const int y = y0 + t;
    const bool yin = t < kVY && y < yd;
    float p2[kVX], p1[kVX], p0[kVX];
#pragma unroll
    for (int i = 0; i < kVX; ++i) p2[i] = p1[i] = p0[i] = 0.0f;
    for (int k = 0; k < nplanes; ++k) {
        const int zi = zb + k;
        const int st = k % kVStages;
        const bool ok = mbar_wait_bounded(&full[st], (uint32_t)((k / kVStages) & 1));
        if (__syncthreads_or(!ok)) {
            if (t == 0) {
                atomicOr(timeout, 1u);
                for (int q = k; q < k + kVStages && q < nplanes; ++q)
                    mbar_wait_bounded(&full[q % kVStages], (uint32_t)((q / kVStages) & 1));
            }
            return;
        }
        const float *B = vsm + (size_t)st * kVBoxY * kVBoxX;  // [row r: x0 - 1 + r][y - (y0 - 4)]
#pragma unroll
        for (int i = 0; i < kVX; ++i) {
            p2[i] = p1[i];
            p1[i] = p0[i];
        }
        if (yin) {
            // y pass of the 18 rows at this y
            float yb[kVBoxX];
#pragma unroll
            for (int r = 0; r < kVBoxX; ++r) {
                const int xg = x0 - 1 + r;
                const float *Sr = B + r * kVBoxY + 4 - y0;  // [global y]
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
            // x pass of the 16 outputs
#pragma unroll
            for (int i = 0; i < kVX; ++i) {
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
                for (int i = 0; i < kVX; ++i) {
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
        __syncthreads();  // every thread is done with the stage
        if (t == 0) issue(k + kVStages);
    }
}

}  // namespace

bool launch_inv_bspline_tma(const float *in, float *O, int yd, int xd, int zd, int ony, int onx, int onz,
                            const InvB &c, unsigned *d_timeout, cudaStream_t s) {
    if (yd % 4 != 0 || yd < kVBoxY || xd < kVBoxX || ((uintptr_t)in & 15) != 0) return false;
    CUtensorMap tm;
    const uint64_t d[3] = {(uint64_t)yd, (uint64_t)xd, (uint64_t)zd};
    const uint32_t box[3] = {(uint32_t)kVBoxY, (uint32_t)kVBoxX, 1u};
    if (!make_tensor_map_3d_f32(&tm, in, d, (uint64_t)yd * 4, (uint64_t)xd * yd * 4, box)) return false;
    set_smem_once<inv_bspline_tma_kernel>((int)kVSmem);
    dim3 grid((yd + kVY - 1) / kVY, (xd + kVX - 1) / kVX, (zd + kVZ - 1) / kVZ);
    inv_bspline_tma_kernel<<<grid, kVThreads, kVSmem, s>>>(tm, O, yd, xd, zd, ony, onx, onz, c, d_timeout);
    count_launch();
    APRB_CHECK_LAUNCH();
    return true;
}

}  // namespace aprb
