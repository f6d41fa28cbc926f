// Learned Richardson-Lucy proposal: a small sparse CNN on APR particles.
// There is no counterpart in the reference; it builds on its neighbourhood
// definition.  A layer applies one 3x3x3 multi-channel stencil on every level
// of the APR: the neighbourhood of a particle at level l is the level's
// isotropic image of APRFilter::convolve_pencil (same-level particles, parents
// one level coarser, tree means of the level), with a zero boundary and zero
// for cells no particle covers.  Activations are 16 channels, channels-last
// (row-major P x 16 float); the operands of the products are rounded to
// bfloat16 and multiplied on the tensor cores (mma.sync m16n8k16, fp32
// accumulation): a warp computes 16 targets x 16 output channels, one k-step
// per stencil tap (16 input channels).
//
// Backward: weight gradients by the same tiles with the roles of particles and
// channels exchanged; input gradients by the transposed convolution over every
// cell of the level (the flipped, transposed stencil), routed to the cell's
// owner: the particle itself, the parent (sum over the cells it covers) or the
// tree node, whose gradient flows to its children through the transpose of
// the tree mean (scale factor / 8, coarse to fine).
//
// Tree means here are unordered sums (atomics): the network needs no bit
// parity with anything, its oracle checks it within a tolerance.
#include <cuda_bf16.h>

#include "kernels.cuh"

namespace aprb {

namespace {

constexpr int kC = 16;   // channels
constexpr int kTaps = 27;

struct LDc {
    int yn, xn, zn;
};
LDc ldc(const Geom &g, int l) { return LDc{g.y_num[l], g.x_num[l], g.z_num[l]}; }
__host__ __device__ __forceinline__ uint64_t ncells(const LDc &d) { return (uint64_t)d.yn * d.xn * d.zn; }

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// ---------------------------------------------------------------------------
// particle rows: prow[i] = z * x_num + x of particle i within its level
// ---------------------------------------------------------------------------
__global__ void rows_kernel(const uint64_t *__restrict__ xz_end, uint64_t row_base, uint64_t rows,
                            uint32_t *__restrict__ prow) {
    const uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= rows) return;
    const uint64_t b = xz_end[row_base + r - 1], e = xz_end[row_base + r];
    for (uint64_t i = b + lane; i < e; i += 32) prow[i] = (uint32_t)r;
}

// ---------------------------------------------------------------------------
// tree means of 16 channels (APRTreeNumerics::fill_tree_mean,
// APRTreeNumerics.hpp:63-203, with unordered sums): children of tree level t
// are the particles and tree nodes of level t+1.
// ---------------------------------------------------------------------------
struct TreeMap {
    LDc dt, dc;              // parent (tree level t) and child level dims
    uint64_t t_row_base;     // tree level_xz[t]
    const uint16_t *t_cidx;  // row chunk index of tree level t
    int nct;                 // chunks per tree row
};

// parent index of the child at (zc, xc, yc) and its scale factor / 8
__device__ __forceinline__ uint64_t tree_parent(const TreeMap &m, const uint64_t *__restrict__ t_xz_end,
                                                const uint16_t *__restrict__ t_y_vec, int zc, int xc, int yc,
                                                float &w) {
    const int zp = zc / 2, xp = xc / 2, yp = yc / 2;
    const uint64_t prow = (uint64_t)zp * m.dt.xn + xp;
    const uint64_t b = t_xz_end[m.t_row_base + prow - 1], e = t_xz_end[m.t_row_base + prow];
    uint64_t i = b + m.t_cidx[prow * (uint64_t)(m.nct + 1) + yp / 64];
    while (i + 1 < e && t_y_vec[i] < yp) ++i;
    float sxz = (float)((((2 * m.dt.xn != m.dc.xn) && (xp == m.dt.xn - 1)) +
                         ((2 * m.dt.zn != m.dc.zn) && (zp == m.dt.zn - 1))) * 2);
    if (sxz == 0) sxz = 1;
    const float syxz = (2 * m.dt.yn != m.dc.yn) ? sxz * 2 : sxz;
    w = ((yp == m.dt.yn - 1) ? syxz : sxz) / 8.0f;
    return i;
}

// forward: tree[parent] += w * child (one warp per child row)
// (cval and tree may be the same array: children of level t+1, parents of t)
__global__ void tree_up_kernel(TreeMap m, const uint64_t *__restrict__ c_xz_end, uint64_t c_row_base,
                               const uint16_t *__restrict__ c_y_vec, const float *cval,
                               const uint64_t *__restrict__ t_xz_end, const uint16_t *__restrict__ t_y_vec,
                               float *tree) {
    const uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= (uint64_t)m.dc.xn * m.dc.zn) return;
    const int zc = (int)(r / (uint64_t)m.dc.xn), xc = (int)(r % (uint64_t)m.dc.xn);
    const uint64_t b = c_xz_end[c_row_base + r - 1], e = c_xz_end[c_row_base + r];
    for (uint64_t i = b + lane; i < e; i += 32) {
        float w;
        const uint64_t p = tree_parent(m, t_xz_end, t_y_vec, zc, xc, c_y_vec[i], w);
        const float4 *src = reinterpret_cast<const float4 *>(cval + i * kC);
        float4 *dst = reinterpret_cast<float4 *>(tree + p * kC);
#pragma unroll
        for (int q = 0; q < kC / 4; ++q) {
            const float4 v = src[q];
            atomicAdd(dst + q, make_float4(w * v.x, w * v.y, w * v.z, w * v.w));  // vector atomic (sm_90+)
        }
    }
}

// backward: child += w * tree_grad[parent]
// (cgrad and tgrad may be the same array: children of level t+1, parents of t)
__global__ void tree_down_kernel(TreeMap m, const uint64_t *__restrict__ c_xz_end, uint64_t c_row_base,
                                 const uint16_t *__restrict__ c_y_vec, float *cgrad,
                                 const uint64_t *__restrict__ t_xz_end, const uint16_t *__restrict__ t_y_vec,
                                 const float *tgrad) {
    const uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= (uint64_t)m.dc.xn * m.dc.zn) return;
    const int zc = (int)(r / (uint64_t)m.dc.xn), xc = (int)(r % (uint64_t)m.dc.xn);
    const uint64_t b = c_xz_end[c_row_base + r - 1], e = c_xz_end[c_row_base + r];
    for (uint64_t i = b + lane; i < e; i += 32) {
        float w;
        const uint64_t p = tree_parent(m, t_xz_end, t_y_vec, zc, xc, c_y_vec[i], w);
#pragma unroll
        for (int c = 0; c < kC; ++c) cgrad[i * kC + c] += w * tgrad[p * kC + c];
    }
}

// ---------------------------------------------------------------------------
// densify: the level's neighbourhood image, 16 bfloat16 channels per cell
// ---------------------------------------------------------------------------
struct DenseArgs {
    LDc d, dp;
    uint64_t row_base, prow_base, trow_base;  // 0: source absent
};

__global__ void densify16_kernel(DenseArgs a, const uint64_t *__restrict__ xz_end, const uint16_t *__restrict__ y_vec,
                                 const float *__restrict__ part, const uint64_t *__restrict__ t_xz_end,
                                 const uint16_t *__restrict__ t_y_vec, const float *__restrict__ tree,
                                 __nv_bfloat16 *__restrict__ D) {
    const uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= (uint64_t)a.d.xn * a.d.zn) return;
    const int yn = a.d.yn;
    uint4 *row = reinterpret_cast<uint4 *>(D + r * (uint64_t)yn * kC);  // 2 x uint4 per cell
    for (int k = lane; k < 2 * yn; k += 32) row[k] = make_uint4(0, 0, 0, 0);
    __syncwarp();
    auto put = [&](int y, const float *v) {
        const float4 *s = reinterpret_cast<const float4 *>(v);
        const float4 f0 = s[0], f1 = s[1], f2 = s[2], f3 = s[3];
        row[2 * y] = make_uint4(pack_bf16(f0.x, f0.y), pack_bf16(f0.z, f0.w), pack_bf16(f1.x, f1.y),
                                pack_bf16(f1.z, f1.w));
        row[2 * y + 1] = make_uint4(pack_bf16(f2.x, f2.y), pack_bf16(f2.z, f2.w), pack_bf16(f3.x, f3.y),
                                    pack_bf16(f3.z, f3.w));
    };
    if (a.row_base) {
        const uint64_t b = xz_end[a.row_base + r - 1], e = xz_end[a.row_base + r];
        for (uint64_t i = b + lane; i < e; i += 32) put(y_vec[i], part + i * kC);
    }
    if (a.prow_base) {
        const int z = (int)(r / (uint64_t)a.d.xn), x = (int)(r % (uint64_t)a.d.xn);
        const uint64_t pr = (uint64_t)(z / 2) * a.dp.xn + x / 2;
        const uint64_t b = xz_end[a.prow_base + pr - 1], e = xz_end[a.prow_base + pr];
        for (uint64_t i = b + lane; i < e; i += 32) {
            const int c0 = 2 * (int)y_vec[i], c1 = min(c0 + 1, yn - 1);
            put(c0, part + i * kC);
            if (c1 != c0) put(c1, part + i * kC);
        }
    }
    if (a.trow_base) {
        const uint64_t b = t_xz_end[a.trow_base + r - 1], e = t_xz_end[a.trow_base + r];
        for (uint64_t i = b + lane; i < e; i += 32) put(t_y_vec[i], tree + i * kC);
    }
}

// gradient image of one level: the output gradient at the level's particle
// cells (bfloat16), zero elsewhere
__global__ void scatter_grad_kernel(LDc d, const uint64_t *__restrict__ xz_end, uint64_t row_base,
                                    const uint16_t *__restrict__ y_vec, const float *__restrict__ g,
                                    __nv_bfloat16 *__restrict__ D) {
    const uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= (uint64_t)d.xn * d.zn) return;
    uint4 *row = reinterpret_cast<uint4 *>(D + r * (uint64_t)d.yn * kC);
    for (int k = lane; k < 2 * d.yn; k += 32) row[k] = make_uint4(0, 0, 0, 0);
    __syncwarp();
    const uint64_t b = xz_end[row_base + r - 1], e = xz_end[row_base + r];
    for (uint64_t i = b + lane; i < e; i += 32) {
        const float4 *s = reinterpret_cast<const float4 *>(g + i * kC);
        const float4 f0 = s[0], f1 = s[1], f2 = s[2], f3 = s[3];
        const int y = y_vec[i];
        row[2 * y] = make_uint4(pack_bf16(f0.x, f0.y), pack_bf16(f0.z, f0.w), pack_bf16(f1.x, f1.y),
                                pack_bf16(f1.z, f1.w));
        row[2 * y + 1] = make_uint4(pack_bf16(f2.x, f2.y), pack_bf16(f2.z, f2.w), pack_bf16(f3.x, f3.y),
                                    pack_bf16(f3.z, f3.w));
    }
}

// ---------------------------------------------------------------------------
// the 3x3x3 multi-channel stencil on the tensor cores
// ---------------------------------------------------------------------------
// Weights W[t][co][ci] (fp32, t = (iz*3 + ix)*3 + iy, offsets iz-1, ix-1, iy-1)
// become bfloat16 in shared memory.  TARGETS 0: the particles [p0, p1) of the
// level (coordinates from prow / y_vec), output to out[p] with bias and an
// optional ReLU; TARGETS 1: every cell of the level, output to out[cell]
// (no bias) -- with flipped, transposed weights this is the input gradient.
struct ConvArgs {
    LDc d;
    uint64_t p0, p1;  // TARGETS 0: particle range of the level
    const uint32_t *prow;
    const uint16_t *y_vec;
    const __nv_bfloat16 *D;
    const float *W, *bias;
    float *out;
    int relu;
};

constexpr int kTilesPerWarp = 8;

// weights as bfloat16, converted once per call: Wb[t][co][ci]
__global__ void to_bf16_kernel(const float *__restrict__ W, __nv_bfloat16 *__restrict__ Wb, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) Wb[k] = __float2bfloat16_rn(W[k]);
}

template <int TARGETS>
__global__ void __launch_bounds__(128) conv16_kernel(ConvArgs a, const __nv_bfloat16 *__restrict__ Wb) {
    __shared__ __align__(16) __nv_bfloat16 Ws[kTaps * kC * kC];
    __shared__ float bs[kC];
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(Wb);
        uint4 *dst = reinterpret_cast<uint4 *>(Ws);
        for (int k = threadIdx.x; k < kTaps * kC * kC / 8; k += blockDim.x) dst[k] = src[k];
    }
    if (threadIdx.x < kC) bs[threadIdx.x] = a.bias ? a.bias[threadIdx.x] : 0.0f;
    __syncthreads();
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    const uint64_t n = TARGETS == 0 ? a.p1 - a.p0 : ncells(a.d);
    const uint32_t *D32 = reinterpret_cast<const uint32_t *>(a.D);
    const uint32_t *W32 = reinterpret_cast<const uint32_t *>(Ws);
    const uint64_t first = ((uint64_t)blockIdx.x * 4 + (threadIdx.x >> 5)) * kTilesPerWarp;
    for (uint64_t tile = first; tile < first + kTilesPerWarp; ++tile) {
        if (tile * 16 >= n) return;
        // coordinates of targets g and g + 8 of the tile
        int tz[2], tx[2], ty[2];
        bool tv[2];
        uint64_t tid[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint64_t k = tile * 16 + g + 8 * h;
            tv[h] = k < n;
            const uint64_t kk = tv[h] ? k : tile * 16;
            if (TARGETS == 0) {
                tid[h] = a.p0 + kk;
                const uint32_t r = a.prow[tid[h]];
                tz[h] = (int)(r / (uint32_t)a.d.xn);
                tx[h] = (int)(r % (uint32_t)a.d.xn);
                ty[h] = a.y_vec[tid[h]];
            } else {
                tid[h] = kk;
                ty[h] = (int)(kk % (uint64_t)a.d.yn);
                const uint64_t r = kk / (uint64_t)a.d.yn;
                tx[h] = (int)(r % (uint64_t)a.d.xn);
                tz[h] = (int)(r / (uint64_t)a.d.xn);
            }
        }
        float c[2][4];
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
            for (int k = 0; k < 4; ++k) c[nt][k] = 0.0f;
#pragma unroll 1
        for (int t0 = 0; t0 < kTaps; t0 += 3) {  // one (iz, ix) neighbour row, iy = 0..2, loads first
            const int dz = t0 / 9 - 1, dx = (t0 / 3) % 3 - 1;
            uint32_t lo[3][2], hi[3][2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int zz = tz[h] + dz, xx = tx[h] + dx;
                const bool rin = zz >= 0 && zz < a.d.zn && xx >= 0 && xx < a.d.xn;
                const uint64_t rbase = ((uint64_t)(rin ? zz : 0) * a.d.xn + (rin ? xx : 0)) * a.d.yn;
#pragma unroll
                for (int iy = 0; iy < 3; ++iy) {
                    const int yy = ty[h] + iy - 1;
                    if (rin && yy >= 0 && yy < a.d.yn) {
                        const uint64_t base = (rbase + yy) * (kC / 2);  // in uint32
                        lo[iy][h] = D32[base + q];
                        hi[iy][h] = D32[base + 4 + q];
                    } else {
                        lo[iy][h] = 0;
                        hi[iy][h] = 0;
                    }
                }
            }
#pragma unroll
            for (int iy = 0; iy < 3; ++iy) {
                const int t = t0 + iy;
                const uint32_t A[4] = {lo[iy][0], lo[iy][1], hi[iy][0], hi[iy][1]};
#pragma unroll
                for (int nt = 0; nt < 2; ++nt) {
                    const int co = nt * 8 + g;
                    const uint32_t b0 = W32[(t * kC + co) * (kC / 2) + q];
                    const uint32_t b1 = W32[(t * kC + co) * (kC / 2) + 4 + q];
                    mma_bf16(c[nt], A, b0, b1);
                }
            }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (!tv[h]) continue;
            float *o = a.out + tid[h] * kC;
#pragma unroll
            for (int nt = 0; nt < 2; ++nt) {
                const int co = nt * 8 + 2 * q;
                float v0 = c[nt][2 * h] + (TARGETS == 0 ? bs[co] : 0.0f);
                float v1 = c[nt][2 * h + 1] + (TARGETS == 0 ? bs[co + 1] : 0.0f);
                if (a.relu) {
                    v0 = fmaxf(v0, 0.0f);
                    v1 = fmaxf(v1, 0.0f);
                }
                *reinterpret_cast<float2 *>(o + co) = make_float2(v0, v1);
            }
        }
    }
}

unsigned conv16_grid(uint64_t targets) {
    const uint64_t tiles = (targets + 15) / 16;
    return blocks_for((tiles + kTilesPerWarp - 1) / kTilesPerWarp, 4);
}

// ---------------------------------------------------------------------------
// weight and bias gradients: dW[t][co][ci] += sum_p D[cell(p) + off(t)][ci] *
// gp[p][co] over the particles [p0, p1) of one level.  A warp takes kDWTiles
// tiles of 16 particles; a tile is one k-step with rows = input channels and
// columns = output channels.  Partial sums meet in shared memory, then one
// atomic per value and block.
// ---------------------------------------------------------------------------
constexpr int kDWTiles = 8;

__global__ void __launch_bounds__(128) dweight_kernel(ConvArgs a, const float *__restrict__ gp,
                                                      float *__restrict__ dW, float *__restrict__ db) {
    __shared__ float red[kC * kC];
    __shared__ float redb[kC];
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3, w = threadIdx.x >> 5;
    const uint64_t n = a.p1 - a.p0;
    const uint64_t t0 = ((uint64_t)blockIdx.x * 4 + w) * kDWTiles;  // first tile of this warp
    const __nv_bfloat16 *D = a.D;
    // bias gradient
    if (threadIdx.x < kC) redb[threadIdx.x] = 0.0f;
    __syncthreads();
    {
        float s = 0.0f;
        for (int tt = 0; tt < kDWTiles; ++tt)
            for (int r = 0; r < 16; ++r) {
                const uint64_t k = (t0 + tt) * 16 + r;
                if (k < n && lane < kC) s += gp[(a.p0 + k) * kC + lane];
            }
        if (lane < kC) atomicAdd(&redb[lane], s);
    }
    __syncthreads();
    if (threadIdx.x < kC) atomicAdd(&db[threadIdx.x], redb[threadIdx.x]);
#pragma unroll 1
    for (int t = 0; t < kTaps; ++t) {
        const int dz = t / 9 - 1, dx = (t / 3) % 3 - 1, dy = t % 3 - 1;
        for (int k = threadIdx.x; k < kC * kC; k += blockDim.x) red[k] = 0.0f;
        __syncthreads();
        float c[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
        for (int tt = 0; tt < kDWTiles; ++tt) {
            const uint64_t tile = t0 + tt;
            if (tile * 16 >= n) break;
            // particles 2q, 2q+1, 2q+8, 2q+9 of the tile
            float dv[4][2];  // [particle][channel g, g+8]
            float gv[4][2];  // [particle][co g (ntile 0), g+8 (ntile 1)]
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int r = 2 * q + (j & 1) + 8 * (j >> 1);
                const uint64_t k = tile * 16 + r;
                dv[j][0] = dv[j][1] = gv[j][0] = gv[j][1] = 0.0f;
                if (k >= n) continue;
                const uint64_t pi = a.p0 + k;
                const uint32_t row = a.prow[pi];
                const int zz = (int)(row / (uint32_t)a.d.xn) + dz, xx = (int)(row % (uint32_t)a.d.xn) + dx,
                          yy = (int)a.y_vec[pi] + dy;
                if (zz >= 0 && zz < a.d.zn && xx >= 0 && xx < a.d.xn && yy >= 0 && yy < a.d.yn) {
                    const uint64_t cell = ((uint64_t)zz * a.d.xn + xx) * a.d.yn + yy;
                    dv[j][0] = __bfloat162float(D[cell * kC + g]);
                    dv[j][1] = __bfloat162float(D[cell * kC + g + 8]);
                }
                gv[j][0] = gp[pi * kC + g];
                gv[j][1] = gp[pi * kC + g + 8];
            }
            // A rows = channels (g, g+8), columns = particles (2q, 2q+1 | 2q+8, 2q+9)
            const uint32_t A[4] = {pack_bf16(dv[0][0], dv[1][0]), pack_bf16(dv[0][1], dv[1][1]),
                                   pack_bf16(dv[2][0], dv[3][0]), pack_bf16(dv[2][1], dv[3][1])};
#pragma unroll
            for (int nt = 0; nt < 2; ++nt) {
                const uint32_t b0 = pack_bf16(gv[0][nt], gv[1][nt]), b1 = pack_bf16(gv[2][nt], gv[3][nt]);
                mma_bf16(c[nt], A, b0, b1);
            }
        }
        // c[nt]: rows ci = g / g+8, columns co = nt*8 + 2q, 2q+1
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) {
            const int co = nt * 8 + 2 * q;
            atomicAdd(&red[co * kC + g], c[nt][0]);
            atomicAdd(&red[(co + 1) * kC + g], c[nt][1]);
            atomicAdd(&red[co * kC + g + 8], c[nt][2]);
            atomicAdd(&red[(co + 1) * kC + g + 8], c[nt][3]);
        }
        __syncthreads();
        for (int k = threadIdx.x; k < kC * kC; k += blockDim.x) atomicAdd(&dW[t * kC * kC + k], red[k]);
        __syncthreads();
    }
}

// ReLU mask of the output gradient: gp = g * (out > 0)
__global__ void relu_mask_kernel(const float *__restrict__ g, const float *__restrict__ out, float *__restrict__ gp,
                                 uint64_t n, int relu) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    gp[i] = (!relu || out[i] > 0.0f) ? g[i] : 0.0f;
}

// flipped, transposed stencil: Wt[26 - t][ci][co] = W[t][co][ci]
__global__ void flip_transpose_kernel(const float *__restrict__ W, float *__restrict__ Wt) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= kTaps * kC * kC) return;
    const int t = k / (kC * kC), co = (k / kC) % kC, ci = k % kC;
    Wt[((kTaps - 1 - t) * kC + ci) * kC + co] = W[k];
}

// route the level's cell gradients G (float, 16 per cell) to the owners
// mode 0: particles of the level (own cell);  mode 1: tree nodes of the
// level (own cell, written);  mode 2: parents one level coarser (sum over the
// cells each covers)
__global__ void route_kernel(LDc d, const uint64_t *__restrict__ xz_end, uint64_t row_base,
                             const uint16_t *__restrict__ y_vec, const float *__restrict__ G,
                             float *__restrict__ dst, int mode, LDc dchild) {
    const uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= (uint64_t)d.xn * d.zn) return;
    const int z = (int)(r / (uint64_t)d.xn), x = (int)(r % (uint64_t)d.xn);
    const uint64_t b = xz_end[row_base + r - 1], e = xz_end[row_base + r];
    for (uint64_t i = b + lane; i < e; i += 32) {
        const int y = y_vec[i];
        float acc[kC];
        if (mode != 2) {
            const float *s = G + (((uint64_t)z * d.xn + x) * d.yn + y) * kC;
#pragma unroll
            for (int c = 0; c < kC; ++c) acc[c] = s[c];
        } else {
#pragma unroll
            for (int c = 0; c < kC; ++c) acc[c] = 0.0f;
            for (int cz = 2 * z; cz < min(2 * z + 2, dchild.zn); ++cz)
                for (int cx = 2 * x; cx < min(2 * x + 2, dchild.xn); ++cx) {
                    const int c0 = 2 * y, c1 = min(2 * y + 1, dchild.yn - 1);
                    for (int cy = c0; cy <= c1; ++cy) {
                        const float *s = G + (((uint64_t)cz * dchild.xn + cx) * dchild.yn + cy) * kC;
#pragma unroll
                        for (int c = 0; c < kC; ++c) acc[c] += s[c];
                    }
                }
        }
        float *o = dst + i * kC;
        if (mode == 1) {
#pragma unroll
            for (int c = 0; c < kC; ++c) o[c] = acc[c];
        } else {
#pragma unroll
            for (int c = 0; c < kC; ++c) o[c] += acc[c];
        }
    }
}

__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, const float *__restrict__ mask, uint64_t n, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = mask ? g[i] * mask[i] : g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// network inputs: log of the estimate relative to the data, log of the RL
// ratio data / blurred estimate, and the log data scaled to ~[0, 1]
__global__ void features_kernel(const float *__restrict__ u, const float *__restrict__ ratio,
                                const uint16_t *__restrict__ raw, float *__restrict__ f, uint64_t P) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const float lr = log1pf((float)raw[i]);
    float4 *o = reinterpret_cast<float4 *>(f + i * kC);
    o[0] = make_float4(logf(fmaxf(u[i], 1e-6f)) - lr, logf(fmaxf(ratio[i], 1e-6f)), lr * 0.125f, 0.0f);
    o[1] = o[2] = o[3] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// loss = mean over particles of (pred - log(u1 / u0))^2; g = d loss / d pred
__global__ void loss_kernel(const float *__restrict__ pred, const float *__restrict__ u0, const float *__restrict__ u1,
                            float *__restrict__ g, uint64_t P, double *loss) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (i < P) {
        const float tgt = logf(fmaxf(u1[i], 1e-6f)) - logf(fmaxf(u0[i], 1e-6f));
        const float d = pred[i * kC] - tgt;
        float4 *o = reinterpret_cast<float4 *>(g + i * kC);
        o[0] = make_float4(2.0f * d / (float)P, 0.0f, 0.0f, 0.0f);
        o[1] = o[2] = o[3] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        l = (double)d * (double)d / (double)P;
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}

// the proposal: u <- u * exp(clamp(pred, -2, 2))
__global__ void apply_kernel(const float *__restrict__ pred, float *__restrict__ u, uint64_t P) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    u[i] = u[i] * expf(fminf(fmaxf(pred[i * kC], -2.0f), 2.0f));
}

// Poisson data-fit objective of RL: sum (k - d log k), k = blurred estimate
__global__ void objective_kernel(const float *__restrict__ k, const uint16_t *__restrict__ raw, uint64_t P,
                                 double *out) {
    double s = 0.0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P; i += (uint64_t)gridDim.x * blockDim.x) {
        const double kv = fmax((double)k[i], 1e-30);
        s += kv - (double)raw[i] * log(kv);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

TreeMap tree_map(const Geom &g, const Geom &tg, int t, const FilterIndex &fi) {
    TreeMap m;
    m.dt = ldc(tg, t);
    m.dc = ldc(g, t + 1);
    m.t_row_base = tg.level_xz[t];
    m.t_cidx = (const uint16_t *)fi.buf.p + fi.tree_off[t];
    m.nct = (tg.y_num[t] + 63) / 64;
    return m;
}

unsigned row_grid(const LDc &d) { return blocks_for((uint64_t)d.xn * d.zn * 32, 256); }

}  // namespace

void cnn_build_rows(const Geom &g, const uint64_t *xz_end, uint32_t *prow, cudaStream_t s) {
    for (int l = g.l_min; l <= g.l_max; ++l) {
        const uint64_t rows = (uint64_t)g.x_num[l] * g.z_num[l];
        if (!rows) continue;
        rows_kernel<<<blocks_for(rows * 32, 256), 256, 0, s>>>(xz_end, g.level_xz[l], rows, prow);
        count_launch();
    }
    APRB_CHECK_LAUNCH();
}

static void tree_means16(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const Geom &tg,
                         const uint64_t *t_xz_end, const uint16_t *t_y_vec, const FilterIndex &fi, const float *in,
                         float *tree, uint64_t T, cudaStream_t s) {
    APRB_CUDA(cudaMemsetAsync(tree, 0, (T ? T : 1) * kC * sizeof(float), s));
    for (int t = tg.l_max; t >= tg.l_min; --t) {
        const int l = t + 1;
        if (l > g.l_max || l < g.l_min) continue;
        const TreeMap m = tree_map(g, tg, t, fi);
        tree_up_kernel<<<row_grid(m.dc), 256, 0, s>>>(m, xz_end, g.level_xz[l], y_vec, in, t_xz_end, t_y_vec, tree);
        if (l <= tg.l_max)
            tree_up_kernel<<<row_grid(m.dc), 256, 0, s>>>(m, t_xz_end, tg.level_xz[l], t_y_vec, tree, t_xz_end,
                                                          t_y_vec, tree);
        count_launch(l <= tg.l_max ? 2 : 1);
    }
    APRB_CHECK_LAUNCH();
}

static DenseArgs dense_args(const Geom &g, const Geom &tg, int l) {
    DenseArgs a;
    a.d = ldc(g, l);
    a.dp = l > g.l_min ? ldc(g, l - 1) : LDc{1, 1, 1};
    a.row_base = g.level_xz[l];
    a.prow_base = l > g.l_min ? g.level_xz[l - 1] : 0;
    a.trow_base = l <= tg.l_max ? tg.level_xz[l] : 0;
    return a;
}

void cnn_layer_forward(const CnnGeom &cg, const float *in, const float *W, const float *b, int relu, float *out,
                       CnnScratch &sc, cudaStream_t s) {
    APRB_PROF("cnn_forward", s);
    const Geom &g = *cg.g, &tg = *cg.tg;
    float *tree = (float *)sc.tree.get((cg.T ? cg.T : 1) * kC * sizeof(float));
    __nv_bfloat16 *Wb = (__nv_bfloat16 *)sc.wbf.get(kTaps * kC * kC * sizeof(__nv_bfloat16));
    to_bf16_kernel<<<blocks_for(kTaps * kC * kC, 256), 256, 0, s>>>(W, Wb, kTaps * kC * kC);
    count_launch();
    {
        APRB_PROF("cnn_tree", s);
        tree_means16(g, cg.xz_end, cg.y_vec, tg, cg.t_xz_end, cg.t_y_vec, *cg.fi, in, tree, cg.T, s);
    }
    for (int l = g.l_max; l >= g.l_min; --l) {
        const uint64_t p0 = cg.level_begin[l], p1 = cg.level_begin[l + 1];
        if (p1 == p0) continue;
        const DenseArgs da = dense_args(g, tg, l);
        __nv_bfloat16 *D = (__nv_bfloat16 *)sc.dense.get(ncells(da.d) * kC * sizeof(__nv_bfloat16));
        {
            APRB_PROF("cnn_densify", s);
            densify16_kernel<<<row_grid(da.d), 256, 0, s>>>(da, cg.xz_end, cg.y_vec, in, cg.t_xz_end, cg.t_y_vec,
                                                            tree, D);
        }
        ConvArgs ca{da.d, p0, p1, cg.prow, cg.y_vec, D, W, b, out, relu};
        {
            APRB_PROF("cnn_conv", s);
            conv16_kernel<0><<<conv16_grid(p1 - p0), 128, 0, s>>>(ca, Wb);
        }
        count_launch(2);
    }
    APRB_CHECK_LAUNCH();
}

void cnn_layer_backward(const CnnGeom &cg, const float *in, const float *W, const float *out, const float *g_out,
                        int relu, float *g_in, float *dW, float *db, CnnScratch &sc, cudaStream_t s) {
    APRB_PROF("cnn_backward", s);
    const Geom &g = *cg.g, &tg = *cg.tg;
    const uint64_t P = cg.level_begin[g.l_max + 1];
    float *tree = (float *)sc.tree.get((cg.T ? cg.T : 1) * kC * sizeof(float));
    float *gtree = (float *)sc.gtree.get((cg.T ? cg.T : 1) * kC * sizeof(float));
    float *gp = (float *)sc.gp.get((P ? P : 1) * kC * sizeof(float));
    float *Wt = (float *)sc.wt.get(kTaps * kC * kC * sizeof(float));
    tree_means16(g, cg.xz_end, cg.y_vec, tg, cg.t_xz_end, cg.t_y_vec, *cg.fi, in, tree, cg.T, s);
    relu_mask_kernel<<<blocks_for(P * kC, 256), 256, 0, s>>>(g_out, out, gp, P * kC, relu);
    flip_transpose_kernel<<<blocks_for(kTaps * kC * kC, 256), 256, 0, s>>>(W, Wt);
    __nv_bfloat16 *Wtb = (__nv_bfloat16 *)sc.wbf.get(kTaps * kC * kC * sizeof(__nv_bfloat16));
    to_bf16_kernel<<<blocks_for(kTaps * kC * kC, 256), 256, 0, s>>>(Wt, Wtb, kTaps * kC * kC);
    count_launch(3);
    APRB_CUDA(cudaMemsetAsync(g_in, 0, (P ? P : 1) * kC * sizeof(float), s));
    APRB_CUDA(cudaMemsetAsync(gtree, 0, (cg.T ? cg.T : 1) * kC * sizeof(float), s));
    for (int l = g.l_max; l >= g.l_min; --l) {
        const uint64_t p0 = cg.level_begin[l], p1 = cg.level_begin[l + 1];
        if (p1 == p0) continue;
        const DenseArgs da = dense_args(g, tg, l);
        const uint64_t nc = ncells(da.d);
        __nv_bfloat16 *D = (__nv_bfloat16 *)sc.dense.get(nc * kC * sizeof(__nv_bfloat16));
        // weight and bias gradients from this level's forward operands
        densify16_kernel<<<row_grid(da.d), 256, 0, s>>>(da, cg.xz_end, cg.y_vec, in, cg.t_xz_end, cg.t_y_vec, tree, D);
        ConvArgs ca{da.d, p0, p1, cg.prow, cg.y_vec, D, W, nullptr, nullptr, 0};
        const uint64_t tiles = (p1 - p0 + 15) / 16;
        dweight_kernel<<<blocks_for((tiles + kDWTiles - 1) / kDWTiles, 4), 128, 0, s>>>(ca, gp, dW, db);
        // input gradient: transposed stencil over every cell of the level
        scatter_grad_kernel<<<row_grid(da.d), 256, 0, s>>>(da.d, cg.xz_end, g.level_xz[l], cg.y_vec, gp, D);
        float *G = (float *)sc.gdense.get(nc * kC * sizeof(float));
        ConvArgs cb{da.d, 0, 0, nullptr, nullptr, D, Wt, nullptr, G, 0};
        conv16_kernel<1><<<conv16_grid(nc), 128, 0, s>>>(cb, Wtb);
        route_kernel<<<row_grid(da.d), 256, 0, s>>>(da.d, cg.xz_end, g.level_xz[l], cg.y_vec, G, g_in, 0, da.d);
        count_launch(5);
        if (da.trow_base) {
            route_kernel<<<row_grid(da.d), 256, 0, s>>>(da.d, cg.t_xz_end, tg.level_xz[l], cg.t_y_vec, G, gtree, 1,
                                                        da.d);
            count_launch();
        }
        if (da.prow_base) {
            route_kernel<<<row_grid(da.dp), 256, 0, s>>>(da.dp, cg.xz_end, g.level_xz[l - 1], cg.y_vec, G, g_in, 2,
                                                         da.d);
            count_launch();
        }
    }
    // tree means transposed, coarse to fine
    for (int t = tg.l_min; t <= tg.l_max; ++t) {
        const int l = t + 1;
        if (l > g.l_max || l < g.l_min) continue;
        const TreeMap m = tree_map(g, tg, t, *cg.fi);
        tree_down_kernel<<<row_grid(m.dc), 256, 0, s>>>(m, cg.xz_end, g.level_xz[l], cg.y_vec, g_in, cg.t_xz_end,
                                                        cg.t_y_vec, gtree);
        count_launch();
        if (l <= tg.l_max) {
            tree_down_kernel<<<row_grid(m.dc), 256, 0, s>>>(m, cg.t_xz_end, tg.level_xz[l], cg.t_y_vec, gtree,
                                                            cg.t_xz_end, cg.t_y_vec, gtree);
            count_launch();
        }
    }
    APRB_CHECK_LAUNCH();
}

void cnn_features(const float *u, const float *ratio, const uint16_t *raw, float *f, uint64_t P, cudaStream_t s) {
    features_kernel<<<blocks_for(P, 256), 256, 0, s>>>(u, ratio, raw, f, P);
    count_launch();
    APRB_CHECK_LAUNCH();
}

void cnn_loss(const float *pred, const float *u0, const float *u1, float *g, uint64_t P, double *loss, cudaStream_t s) {
    APRB_CUDA(cudaMemsetAsync(loss, 0, sizeof(double), s));
    loss_kernel<<<blocks_for(P, 256), 256, 0, s>>>(pred, u0, u1, g, P, loss);
    count_launch();
    APRB_CHECK_LAUNCH();
}

void cnn_apply(const float *pred, float *u, uint64_t P, cudaStream_t s) {
    apply_kernel<<<blocks_for(P, 256), 256, 0, s>>>(pred, u, P);
    count_launch();
    APRB_CHECK_LAUNCH();
}

void rl_objective_sum(const float *k, const uint16_t *raw, uint64_t P, double *out, cudaStream_t s) {
    APRB_CUDA(cudaMemsetAsync(out, 0, sizeof(double), s));
    objective_kernel<<<std::min<unsigned>(blocks_for(P, 256), 148 * 8), 256, 0, s>>>(k, raw, P, out);
    count_launch();
    APRB_CHECK_LAUNCH();
}

void cnn_adam(float *p, const float *g, float *m, float *v, const float *mask, uint64_t n, float lr, float b1,
              float b2, float eps, int step, cudaStream_t s) {
    const float c1 = 1.0f - std::pow(b1, (float)step), c2 = 1.0f - std::pow(b2, (float)step);
    adam_kernel<<<blocks_for(n, 256), 256, 0, s>>>(p, g, m, v, mask, n, lr, b1, b2, eps, c1, c2);
    count_launch();
    APRB_CHECK_LAUNCH();
}

}  // namespace aprb
