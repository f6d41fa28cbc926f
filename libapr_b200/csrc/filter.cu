// APR tree means and APR isotropic convolution on the GPU.
//
// Levels are processed from l_max down.  For level l a dense level image is
// built in HBM from the particles of level l, the tree nodes of level l (the
// means of finer particles) and, for the stencil's reach, the particles one
// level coarser (piecewise constant) -- the isotropic neighbourhood that
// APRFilter::update_dense_array builds per pencil (APRFilter.hpp:825-849).
// The same image feeds (a) the tree means of level l-1, accumulated in the
// exact child order of APRTreeNumerics::fill_tree_mean (APRTreeNumerics.hpp:
// 63-203): particle children first, then tree children, each in z, x, y order,
// and (b) the stencil sums of level-l particles in the order of
// run_convolution_pencil (APRFilter.hpp:706-736), without FMA contraction.
#include "kernels.cuh"

namespace aprb {

namespace {

struct LD {
    int yn, xn, zn;
};
LD ld(const Geom &g, int l) { return LD{g.y_num[l], g.x_num[l], g.z_num[l]}; }
uint64_t ncell(const Geom &g, int l) { return (uint64_t)g.y_num[l] * g.x_num[l] * g.z_num[l]; }
uint64_t nrow(const Geom &g, int l) { return (uint64_t)g.x_num[l] * g.z_num[l]; }
unsigned row_blocks(uint64_t rows) { return blocks_for(rows * 32, 256); }

constexpr uint8_t kTypeParticle = 1, kTypeTree = 2, kTypeParent = 3;

// scatter one level's values (particles or tree nodes) into the dense image
__global__ void scatter_kernel(LD d, const uint64_t *__restrict__ xz_end, uint64_t row_base,
                               const uint16_t *__restrict__ y_vec, const float *__restrict__ val,
                               float *__restrict__ D, uint8_t *__restrict__ T, uint8_t type) {
    const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= (uint64_t)d.xn * d.zn) return;
    const uint64_t b = xz_end[row_base + row - 1], e = xz_end[row_base + row];
    const uint64_t o = row * (uint64_t)d.yn;
    for (uint64_t i = b + lane; i < e; i += 32) {
        const uint64_t q = o + y_vec[i];
        D[q] = val[i];
        T[q] = type;
    }
}

// parents one level coarser fill their 2x2x2 children (update_higher_level,
// APRFilter.hpp:766-793), clipped to the level's dims
__global__ void scatter_parent_kernel(LD dp, const uint64_t *__restrict__ xz_end, uint64_t row_base,
                                      const uint16_t *__restrict__ y_vec, const float *__restrict__ val, LD d,
                                      float *__restrict__ D, uint8_t *__restrict__ T) {
    const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= (uint64_t)dp.xn * dp.zn) return;
    const int xp = (int)(row % (uint64_t)dp.xn), zp = (int)(row / (uint64_t)dp.xn);
    const uint64_t b = xz_end[row_base + row - 1], e = xz_end[row_base + row];
    for (uint64_t i = b + lane; i < e; i += 32) {
        const int yp = y_vec[i];
        const float v = val[i];
        for (int z = 2 * zp; z < min(2 * zp + 2, d.zn); ++z)
            for (int x = 2 * xp; x < min(2 * xp + 2, d.xn); ++x)
                for (int y = 2 * yp; y < min(2 * yp + 2, d.yn); ++y) {
                    const uint64_t q = idx3(y, x, z, d.yn, d.xn);
                    D[q] = v;
                    T[q] = kTypeParent;
                }
    }
}

// tree means of level t from the dense image of level t+1
__global__ void tree_gather_kernel(LD dt, const uint64_t *__restrict__ t_xz_end, uint64_t row_base,
                                   const uint16_t *__restrict__ t_y_vec, LD d, const float *__restrict__ D,
                                   const uint8_t *__restrict__ T, float *__restrict__ tree) {
    const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= (uint64_t)dt.xn * dt.zn) return;
    const int x = (int)(row % (uint64_t)dt.xn), z = (int)(row / (uint64_t)dt.xn);
    const uint64_t b = t_xz_end[row_base + row - 1], e = t_xz_end[row_base + row];
    float sxz = (float)((((2 * dt.xn != d.xn) && (x == dt.xn - 1)) + ((2 * dt.zn != d.zn) && (z == dt.zn - 1))) * 2);
    if (sxz == 0) sxz = 1;
    const float syxz = (2 * dt.yn != d.yn) ? sxz * 2 : sxz;
    for (uint64_t i = b + lane; i < e; i += 32) {
        const int y = t_y_vec[i];
        const float s = (y == dt.yn - 1) ? syxz : sxz;
        float acc = 0.0f;
        for (int type = kTypeParticle; type <= kTypeTree; ++type)
            for (int cz = 2 * z; cz < min(2 * z + 2, d.zn); ++cz)
                for (int cx = 2 * x; cx < min(2 * x + 2, d.xn); ++cx)
                    for (int cy = 2 * y; cy < min(2 * y + 2, d.yn); ++cy) {
                        const uint64_t q = idx3(cy, cx, cz, d.yn, d.xn);
                        if (T[q] == type) acc = (s * D[q]) / 8.0f + acc;
                    }
        tree[i] = acc;
    }
}

__device__ __forceinline__ int bc_index(int i, int n, int reflect, int &state) {
    if (i >= 0 && i < n) return i;
    if (!reflect) {
        state = 1;  // zero pad
        return 0;
    }
    const int r = i < 0 ? -i : 2 * (n - 1) - i;
    if (r < 0 || r >= n) {
        state = 2;  // reflection leaves the level: the reference reads stale data
        return 0;
    }
    return r;
}

template <int S>
__global__ void conv_kernel(LD d, const uint64_t *__restrict__ xz_end, uint64_t row_base,
                            const uint16_t *__restrict__ y_vec, const float *__restrict__ D,
                            const uint8_t *__restrict__ T, const float *__restrict__ stencil, int reflect,
                            float *__restrict__ out, int mode, const uint16_t *__restrict__ rl_in,
                            unsigned long long *stale) {
    constexpr int R = (S - 1) / 2;
    __shared__ float st[S * S * S];
    for (int k = threadIdx.x; k < S * S * S; k += blockDim.x) st[k] = stencil[k];
    __syncthreads();
    const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= (uint64_t)d.xn * d.zn) return;
    const int x = (int)(row % (uint64_t)d.xn), z = (int)(row / (uint64_t)d.xn);
    const uint64_t b = xz_end[row_base + row - 1], e = xz_end[row_base + row];
    unsigned nstale = 0;
    for (uint64_t i = b + lane; i < e; i += 32) {
        const int y = y_vec[i];
        float val = 0.0f;
        int cnt = 0;
#pragma unroll
        for (int iz = 0; iz < S; ++iz) {
            int sz = 0;
            const int zz = bc_index(z + iz - R, d.zn, reflect, sz);
#pragma unroll
            for (int ix = 0; ix < S; ++ix) {
                int sx = 0;
                const int xx = bc_index(x + ix - R, d.xn, reflect, sx);
#pragma unroll
                for (int iy = 0; iy < S; ++iy) {
                    int sy = 0;
                    const int yy = bc_index(y + iy - R, d.yn, reflect, sy);
                    float v = 0.0f;
                    const int worst = max(sz, max(sx, sy));
                    if (worst == 0) {
                        const uint64_t q = idx3(yy, xx, zz, d.yn, d.xn);
                        if (T[q])
                            v = D[q];
                        else
                            nstale++;
                    } else if (worst == 2) {
                        nstale++;
                    }
                    val = __fadd_rn(val, __fmul_rn(v, st[cnt]));
                    cnt++;
                }
            }
        }
        if (mode == 0)
            out[i] = val;
        else if (mode == 1)
            out[i] = (float)rl_in[i] / val;
        else
            out[i] = out[i] * val;
    }
    if (nstale) atomicAdd(stale, (unsigned long long)nstale);
}

}  // namespace

void filter_apply(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const Geom &tg,
                  const uint64_t *t_xz_end, const uint16_t *t_y_vec, const float *in, float *tree,
                  const ConvPlan *plan, const float *d_stencils, float *out, int mode, const uint16_t *rl_in,
                  FilterBuffers &fb, cudaStream_t s) {
    APRB_PROF(plan ? "convolve" : "fill_tree_mean", s);
    const int L = g.l_max;
    const uint64_t nmax = ncell(g, L);
    float *D = fb.dense.as<float>(nmax);
    uint8_t *T = fb.type.as<uint8_t>(nmax);
    unsigned long long *stale = fb.stale.as<unsigned long long>(1);
    APRB_CUDA(cudaMemsetAsync(stale, 0, sizeof(unsigned long long), s));
    for (int l = L; l >= g.l_min; --l) {
        const LD d = ld(g, l);
        APRB_CUDA(cudaMemsetAsync(T, 0, ncell(g, l), s));
        scatter_kernel<<<row_blocks(nrow(g, l)), 256, 0, s>>>(d, xz_end, g.level_xz[l], y_vec, in, D, T,
                                                             kTypeParticle);
        count_launch();
        if (l <= tg.l_max) {
            scatter_kernel<<<row_blocks(nrow(tg, l)), 256, 0, s>>>(d, t_xz_end, tg.level_xz[l], t_y_vec, tree, D, T,
                                                                  kTypeTree);
            count_launch();
        }
        int side = 0;
        if (plan) {
            const int sn = std::min(plan->nstencils - 1, L - l);
            side = plan->sides[sn];
            const int r = (side - 1) / 2;
            const int max_npl = (int)std::ceil(std::log2((double)(r + 2)) - 1);
            const int npl = std::min(max_npl, l - g.l_min);
            if (npl >= 1)
                scatter_parent_kernel<<<row_blocks(nrow(g, l - 1)), 256, 0, s>>>(
                    ld(g, l - 1), xz_end, g.level_xz[l - 1], y_vec, in, d, D, T);
            if (npl >= 1) count_launch();
        }
        APRB_CHECK_LAUNCH();
        if (l - 1 >= tg.l_min) {
            tree_gather_kernel<<<row_blocks(nrow(tg, l - 1)), 256, 0, s>>>(ld(tg, l - 1), t_xz_end,
                                                                          tg.level_xz[l - 1], t_y_vec, d, D, T, tree);
            count_launch();
        }
        if (plan) {
            const int sn = std::min(plan->nstencils - 1, L - l);
            const float *st = d_stencils + plan->offsets[sn];
            if (side == 3)
                conv_kernel<3><<<row_blocks(nrow(g, l)), 256, 0, s>>>(d, xz_end, g.level_xz[l], y_vec, D, T, st,
                                                                     plan->reflect, out, mode, rl_in, stale);
            else
                conv_kernel<5><<<row_blocks(nrow(g, l)), 256, 0, s>>>(d, xz_end, g.level_xz[l], y_vec, D, T, st,
                                                                     plan->reflect, out, mode, rl_in, stale);
            count_launch();
        }
        APRB_CHECK_LAUNCH();
    }
}

uint64_t filter_stale_count(FilterBuffers &fb, cudaStream_t s) {
    unsigned long long v = 0;
    APRB_CUDA(cudaMemcpyAsync(&v, fb.stale.as<unsigned long long>(1), sizeof(v), cudaMemcpyDeviceToHost, s));
    APRB_CUDA(cudaStreamSynchronize(s));
    return v;
}

}  // namespace aprb
