// APR tree means and APR isotropic convolution on the GPU.
//
// Row chunk index: for every row of every level (particles and tree), the
// offset of the first element at or after each multiple of 64 in y.  It is
// built once per APR and lets a CTA find the part of a row inside its y
// window with one load instead of a search.
//
// Tree means (APRTreeNumerics::fill_tree_mean, APRTreeNumerics.hpp:63-203):
// one CTA per (parent row, 256-cell y chunk) stages its four child rows in
// shared memory (value + kind: particle or tree node) and every parent sums
// its children in the reference's order -- particle children first, then tree
// children, z then x then y within each -- with the reference's boundary scale
// factors (:97-110).  Levels run from fine to coarse.
//
// Convolution (APRFilter::convolve_pencil, APRFilter.hpp:1094-1216): one CTA
// per (8 x-rows, 128-y chunk, 16-z range) of a level streams z through a ring
// of 2R+1 shared-memory slices.  Each slice is the isotropic neighbourhood the
// reference builds in its pencil buffer (update_dense_array, :825-849):
// same-level particles, parents one level coarser (piecewise constant,
// :766-793) and tree means of the same level (:802-818), with the reflective
// or zero boundary (:287-504) folded into the slice contents.  Each particle
// of the centre slice sums its 27 / 125 taps in the stencil's memory order
// without contraction (run_convolution_pencil, :706-736).  A cell no particle
// covers holds a sentinel; reading it is counted as a stale read (the
// reference would read a stale pencil buffer there) and contributes 0.
#include "kernels.cuh"

namespace aprb {

namespace {

constexpr uint32_t kMissingBits = 0x7fbadbadu;               // NaN payload marking an uncovered cell
constexpr uint64_t kMissingBits64 = 0x7ff7badbadbadbadull;  // the same for double values
constexpr int kYC = 64;                                      // y chunk of the row index

// Value type of the filter: float, or double for the FP64 instantiation of
// richardson_lucy.  Arithmetic goes through the round-to-nearest intrinsics
// so no contraction can change a result.
template <typename T>
struct VT;
template <>
struct VT<float> {
    static __device__ __forceinline__ float miss() { return __uint_as_float(kMissingBits); }
    static __device__ __forceinline__ bool is_miss(float v) { return __float_as_uint(v) == kMissingBits; }
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
};
template <>
struct VT<double> {
    static __device__ __forceinline__ double miss() { return __longlong_as_double((long long)kMissingBits64); }
    static __device__ __forceinline__ bool is_miss(double v) {
        return (uint64_t)__double_as_longlong(v) == kMissingBits64;
    }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
};

struct LD {
    int yn, xn, zn;
};
LD ld(const Geom &g, int l) { return LD{g.y_num[l], g.x_num[l], g.z_num[l]}; }
uint64_t nrow(const Geom &g, int l) { return (uint64_t)g.x_num[l] * g.z_num[l]; }
__host__ __device__ __forceinline__ int nchunk(int yn) { return (yn + kYC - 1) / kYC; }

// Reflection about the edge sample (APRFilter.hpp:287-504), or the zero pad
// (ok = false); a reflection that still leaves the level marks the cell stale.
__device__ __forceinline__ int reflect_idx(int i, int n, int reflect, bool &ok) {
    if (i >= 0 && i < n) return i;
    if (!reflect) {
        ok = false;
        return 0;
    }
    const int r = i < 0 ? -i : 2 * (n - 1) - i;
    if (r < 0 || r >= n) {
        ok = false;
        return 0;
    }
    return r;
}

// cidx[row * (nc + 1) + c] = offset (from the row start) of the first element
// with y >= c * kYC; entry nc is the row length.
__global__ void chunk_index_kernel(const uint64_t *__restrict__ xz_end, uint64_t row_base,
                                   const uint16_t *__restrict__ y_vec, uint64_t rows, int nc,
                                   uint16_t *__restrict__ cidx) {
    const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= rows) return;
    const uint64_t b = xz_end[row_base + row - 1], e = xz_end[row_base + row];
    uint16_t *C = cidx + row * (uint64_t)(nc + 1);
    for (uint64_t i = b + lane; i < e; i += 32) {
        const int c = y_vec[i] / kYC;
        const int pc = (i == b) ? -1 : y_vec[i - 1] / kYC;
        for (int q = pc + 1; q <= c; ++q) C[q] = (uint16_t)(i - b);
    }
    const int lastc = (e > b) ? y_vec[e - 1] / kYC : -1;
    for (int q = lastc + 1 + lane; q <= nc; q += 32) C[q] = (uint16_t)(e - b);
}

// ---------------------------------------------------------------------------
// tree means of tree level t (children at level t+1)
// ---------------------------------------------------------------------------
constexpr int kTW = 256;  // parent cells per CTA along y (a multiple of kYC)

struct TreeLevelArgs {
    LD dt;                  // tree level t dims (== APR level t dims)
    LD dc;                  // child level dims
    uint64_t t_row_base;    // tree level_xz[t]
    uint64_t c_row_base;    // APR level_xz[t+1]
    uint64_t ct_row_base;   // tree level_xz[t+1] (0 when t+1 has no tree level)
    const uint16_t *t_cidx, *c_cidx, *ct_cidx;
};

template <typename T>
__global__ void __launch_bounds__(128) tree_mean_kernel(TreeLevelArgs a, const uint64_t *__restrict__ xz_end,
                                                        const uint16_t *__restrict__ y_vec,
                                                        const T *__restrict__ parts,
                                                        const uint64_t *__restrict__ t_xz_end,
                                                        const uint16_t *__restrict__ t_y_vec,
                                                        T *__restrict__ tree) {
    __shared__ T sv[4][2 * kTW];
    __shared__ uint8_t sk[4][2 * kTW];
    const uint64_t prow = blockIdx.x;  // parent row z*xt + x
    const int xp = (int)(prow % (uint64_t)a.dt.xn), zp = (int)(prow / (uint64_t)a.dt.xn);
    const int y0 = blockIdx.y * kTW;
    const int cy0 = 2 * y0, cy1 = min(2 * y0 + 2 * kTW, a.dc.yn);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int k = threadIdx.x; k < 4 * 2 * kTW; k += blockDim.x) (&sk[0][0])[k] = 0;
    __syncthreads();
    {
        const int cz = 2 * zp + (w >> 1), cx = 2 * xp + (w & 1);
        if (cz < a.dc.zn && cx < a.dc.xn && cy0 < cy1) {
            const uint64_t row = (uint64_t)cz * a.dc.xn + cx;
            const int ncc = nchunk(a.dc.yn);
            {
                const uint64_t b = xz_end[a.c_row_base + row - 1], e = xz_end[a.c_row_base + row];
                const uint64_t s = b + a.c_cidx[row * (uint64_t)(ncc + 1) + cy0 / kYC];
                for (uint64_t i = s + lane; i < e; i += 32) {
                    const int y = y_vec[i];
                    if (y >= cy1) break;
                    sv[w][y - cy0] = parts[i];
                    sk[w][y - cy0] = 1;
                }
            }
            if (a.ct_row_base) {
                const uint64_t b = t_xz_end[a.ct_row_base + row - 1], e = t_xz_end[a.ct_row_base + row];
                const uint64_t s = b + a.ct_cidx[row * (uint64_t)(ncc + 1) + cy0 / kYC];
                for (uint64_t i = s + lane; i < e; i += 32) {
                    const int y = t_y_vec[i];
                    if (y >= cy1) break;
                    sv[w][y - cy0] = tree[i];
                    sk[w][y - cy0] = 2;
                }
            }
        }
    }
    __syncthreads();
    const int nct = nchunk(a.dt.yn);
    const uint64_t pb = t_xz_end[a.t_row_base + prow - 1], pe = t_xz_end[a.t_row_base + prow];
    const uint16_t *PC = a.t_cidx + prow * (uint64_t)(nct + 1);
    const uint64_t ps = pb + PC[y0 / kYC];
    const uint64_t pend = pb + PC[min(y0 / kYC + kTW / kYC, nct)];
    float sxz = (float)((((2 * a.dt.xn != a.dc.xn) && (xp == a.dt.xn - 1)) +
                         ((2 * a.dt.zn != a.dc.zn) && (zp == a.dt.zn - 1))) * 2);
    if (sxz == 0) sxz = 1;
    const float syxz = (2 * a.dt.yn != a.dc.yn) ? sxz * 2 : sxz;
    (void)pe;
    for (uint64_t i = ps + threadIdx.x; i < pend; i += blockDim.x) {
        const int y = t_y_vec[i];
        const float s = (y == a.dt.yn - 1) ? syxz : sxz;
        const int o = 2 * (y - y0);
        T acc = T(0);
#pragma unroll
        for (int kind = 1; kind <= 2; ++kind)
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int d = 0; d < 2; ++d)
                    if (o + d < cy1 - cy0 && sk[q][o + d] == kind)
                        acc = VT<T>::add(VT<T>::div(VT<T>::mul(T(s), sv[q][o + d]), T(8)), acc);
        tree[i] = acc;
    }
}

// ---------------------------------------------------------------------------
// convolution of one level
// ---------------------------------------------------------------------------
constexpr int kBX = 8, kBY = 128, kBZ = 16;
constexpr int kConvK = 4;  // output particles per thread and pass

struct ConvLevelArgs {
    LD d;                 // level dims
    LD dp;                // parent level dims
    uint64_t row_base;    // APR level_xz[l]
    uint64_t prow_base;   // APR level_xz[l-1] (0: no parents used)
    uint64_t trow_base;   // tree level_xz[l] (0: no tree level)
    const uint16_t *cidx, *pcidx, *tcidx;
    int reflect;
    int mode;
};

template <int R, typename T>
struct ConvSmem {
    static constexpr int S = 2 * R + 1, RX = kBX + 2 * R, RY = kBY + 2 * R;
    T ring[S][RX][RY];
    T st[S * S * S];
    uint64_t ob[kBX];
    int ocnt[kBX + 1];
};

// Fills one slice row (level row (zr, xr) over the y window) of the ring.
template <int R, typename T>
__device__ void fill_slice_row(T *__restrict__ rowbuf, int zr, int xr, int y0, const ConvLevelArgs &a,
                               const uint64_t *__restrict__ xz_end, const uint16_t *__restrict__ y_vec,
                               const T *__restrict__ in, const uint64_t *__restrict__ t_xz_end,
                               const uint16_t *__restrict__ t_y_vec, const T *__restrict__ tree, int lane) {
    constexpr int RY = kBY + 2 * R;
    const int ys = y0 - R;  // y of rowbuf[0]
    const T miss = VT<T>::miss();
    for (int k = lane; k < RY; k += 32) rowbuf[k] = miss;
    const int ya = max(ys, 0), yb = min(ys + RY - 1, a.d.yn - 1);  // real y range needed
    if (ya <= yb) {
        // Bounds of the three sources inside the y window: same-level
        // particles, parents one level coarser (each fills its y pair) and
        // tree means of the same level.  They cover disjoint cells, so one
        // merged pass writes them in any order.  Lanes 0-2 fetch the bounds.
        const uint64_t row = (uint64_t)zr * a.d.xn + xr;
        const int nc = nchunk(a.d.yn);
        uint64_t lo = 0, hi = 0;
        if (lane == 0) {
            const uint64_t b = xz_end[a.row_base + row - 1];
            hi = xz_end[a.row_base + row];
            lo = b + a.cidx[row * (uint64_t)(nc + 1) + ya / kYC];
        } else if (lane == 1 && a.prow_base) {
            const uint64_t prow = (uint64_t)(zr / 2) * a.dp.xn + xr / 2;
            const int npc = nchunk(a.dp.yn);
            const uint64_t b = xz_end[a.prow_base + prow - 1];
            hi = xz_end[a.prow_base + prow];
            lo = b + a.pcidx[prow * (uint64_t)(npc + 1) + (ya / 2) / kYC];
        } else if (lane == 2 && a.trow_base) {
            const uint64_t b = t_xz_end[a.trow_base + row - 1];
            hi = t_xz_end[a.trow_base + row];
            lo = b + a.tcidx[row * (uint64_t)(nc + 1) + ya / kYC];
        }
        const uint64_t s0 = __shfl_sync(0xffffffffu, lo, 0), e0 = __shfl_sync(0xffffffffu, hi, 0);
        const uint64_t s1 = __shfl_sync(0xffffffffu, lo, 1), e1 = __shfl_sync(0xffffffffu, hi, 1);
        const uint64_t s2 = __shfl_sync(0xffffffffu, lo, 2), e2 = __shfl_sync(0xffffffffu, hi, 2);
        __syncwarp();
        bool go0 = true, go1 = true, go2 = true;
        for (uint64_t t = lane; go0 || go1 || go2; t += 32) {
            const uint64_t i0 = s0 + t, i1 = s1 + t, i2 = s2 + t;
            const bool h0 = go0 && i0 < e0, h1 = go1 && i1 < e1, h2 = go2 && i2 < e2;
            const int y0v = h0 ? (int)y_vec[i0] : 0x7fffffff;
            const int y1v = h1 ? 2 * (int)y_vec[i1] : 0x7fffffff;
            const int y2v = h2 ? (int)t_y_vec[i2] : 0x7fffffff;
            if (y0v <= yb && y0v >= ya) rowbuf[y0v - ys] = in[i0];
            if (y1v <= yb) {
                const T v = in[i1];
                const int c1 = min(y1v + 1, a.d.yn - 1);
                if (y1v >= ya) rowbuf[y1v - ys] = v;
                if (c1 != y1v && c1 >= ya && c1 <= yb) rowbuf[c1 - ys] = v;
            }
            if (y2v <= yb && y2v >= ya) rowbuf[y2v - ys] = tree[i2];
            // a source ends for the warp once any lane passes its window
            go0 = __all_sync(0xffffffffu, h0 && y0v <= yb);
            go1 = __all_sync(0xffffffffu, h1 && y1v <= yb);
            go2 = __all_sync(0xffffffffu, h2 && y2v <= yb);
        }
    }
    __syncwarp();
    // y boundary: reflection about the edge sample, or zero
    for (int k = lane; k < RY; k += 32) {
        const int y = ys + k;
        if (y >= 0 && y < a.d.yn) continue;
        if (!a.reflect) {
            rowbuf[k] = T(0);
        } else {
            const int r = y < 0 ? -y : 2 * (a.d.yn - 1) - y;
            rowbuf[k] = (r >= 0 && r < a.d.yn && r - ys >= 0 && r - ys < RY) ? rowbuf[r - ys] : miss;
        }
    }
}

template <int R, typename T>
__global__ void __launch_bounds__(32 * (kBX + 2 * R)) conv_tile_kernel(
    ConvLevelArgs a, const uint64_t *__restrict__ xz_end, const uint16_t *__restrict__ y_vec,
    const T *__restrict__ in, const uint64_t *__restrict__ t_xz_end, const uint16_t *__restrict__ t_y_vec,
    const T *__restrict__ tree, const T *__restrict__ stencil, T *__restrict__ out,
    const uint16_t *__restrict__ rl_in, unsigned long long *stale) {
    constexpr int S = 2 * R + 1, RX = kBX + 2 * R, RY = kBY + 2 * R, NT = 32 * RX;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ConvSmem<R, T> &sm = *reinterpret_cast<ConvSmem<R, T> *>(smem_raw);
    const int x0 = blockIdx.x * kBX, y0 = blockIdx.y * kBY, z0 = blockIdx.z * kBZ;
    const int z1 = min(z0 + kBZ, a.d.zn);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int k = threadIdx.x; k < S * S * S; k += NT) sm.st[k] = stencil[k];
    unsigned nstale = 0;
    const int nc = nchunk(a.d.yn);

    // warp w fills ring row w of the slice at z (z may lie outside the level)
    auto load_slice = [&](int zq) {
        T(*slot)[RY] = sm.ring[(zq - (z0 - R)) % S];
        bool ok = true;
        const int zr = reflect_idx(zq, a.d.zn, a.reflect, ok);
        const int xr = reflect_idx(x0 - R + w, a.d.xn, a.reflect, ok);
        if (!ok) {
            const T v = a.reflect ? VT<T>::miss() : T(0);
            for (int k = lane; k < RY; k += 32) slot[w][k] = v;
        } else {
            fill_slice_row<R, T>(slot[w], zr, xr, y0, a, xz_end, y_vec, in, t_xz_end, t_y_vec, tree, lane);
        }
    };

    for (int zq = z0 - R; zq < z0 + R; ++zq) load_slice(zq);
    for (int z = z0; z < z1; ++z) {
        load_slice(z + R);
        if (threadIdx.x < kBX) {  // output particles of the centre rows
            const int x = x0 + threadIdx.x;
            uint64_t b = 0, e = 0;
            if (x < a.d.xn) {
                const uint64_t row = (uint64_t)z * a.d.xn + x;
                const uint64_t rb = xz_end[a.row_base + row - 1];
                const uint16_t *Cr = a.cidx + row * (uint64_t)(nc + 1);
                b = rb + Cr[y0 / kYC];
                e = rb + Cr[min(y0 / kYC + kBY / kYC, nc)];
            }
            sm.ob[threadIdx.x] = b;
            sm.ocnt[threadIdx.x + 1] = (int)(e - b);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            sm.ocnt[0] = 0;
            for (int q = 1; q <= kBX; ++q) sm.ocnt[q] += sm.ocnt[q - 1];
        }
        __syncthreads();
        const int total = sm.ocnt[kBX];
        const T *ring0 = &sm.ring[0][0][0];
        auto slot_of = [&](int iz) { return ring0 + ((z + iz - R - (z0 - R)) % S) * (RX * RY); };
        // Each thread takes kConvK particles; one z-slice of the stencil sits in
        // registers while it is applied to all of them, in the stencil's order.
        for (int base = 0; base < total; base += kConvK * NT) {
            uint64_t ii[kConvK];
            int roff[kConvK];
            bool has[kConvK];
#pragma unroll
            for (int j = 0; j < kConvK; ++j) {
                const int k = base + j * NT + threadIdx.x;
                has[j] = k < total;
                ii[j] = 0;
                roff[j] = 0;
                if (has[j]) {
                    int q = 0;
                    while (q + 1 < kBX && sm.ocnt[q + 1] <= k) ++q;
                    ii[j] = sm.ob[q] + (uint64_t)(k - sm.ocnt[q]);
                    roff[j] = q * RY + ((int)y_vec[ii[j]] - (y0 - R)) - R;  // ring offset of tap (ix, iy) = (0, 0)
                }
            }
            T acc[kConvK];
#pragma unroll
            for (int j = 0; j < kConvK; ++j) acc[j] = T(0);
#pragma unroll 1
            for (int iz = 0; iz < S; ++iz) {
                const T *sl = slot_of(iz);
                T stv[S * S];
#pragma unroll
                for (int t = 0; t < S * S; ++t) stv[t] = sm.st[iz * S * S + t];
#pragma unroll
                for (int ix = 0; ix < S; ++ix)
#pragma unroll
                    for (int iy = 0; iy < S; ++iy)
#pragma unroll
                        for (int j = 0; j < kConvK; ++j)
                            acc[j] = VT<T>::add(acc[j], VT<T>::mul(sl[roff[j] + ix * RY + iy], stv[ix * S + iy]));
            }
#pragma unroll
            for (int j = 0; j < kConvK; ++j) {
                if (!has[j]) continue;
                T val = acc[j];
                if (val != val) {  // NaN: a sentinel (or a NaN input) was read; redo with stale counting
                    val = T(0);
                    int cnt = 0;
                    for (int iz = 0; iz < S; ++iz) {
                        const T *sl = slot_of(iz);
                        for (int ix = 0; ix < S; ++ix)
                            for (int iy = 0; iy < S; ++iy) {
                                T v = sl[roff[j] + ix * RY + iy];
                                if (VT<T>::is_miss(v)) {
                                    v = T(0);
                                    nstale++;
                                }
                                val = VT<T>::add(val, VT<T>::mul(v, sm.st[cnt]));
                                cnt++;
                            }
                    }
                }
                const uint64_t i = ii[j];
                if (a.mode == 0)
                    out[i] = val;
                else if (a.mode == 1)
                    out[i] = VT<T>::div((T)rl_in[i], val);
                else
                    out[i] = VT<T>::mul(out[i], val);
            }
        }
        __syncthreads();
    }
    if (nstale) atomicAdd(stale, (unsigned long long)nstale);
}

template <int R, typename T>
void launch_conv_level(const ConvLevelArgs &a, const uint64_t *xz_end, const uint16_t *y_vec, const T *in,
                       const uint64_t *t_xz_end, const uint16_t *t_y_vec, const T *tree, const T *st, T *out,
                       const uint16_t *rl_in, unsigned long long *stale, cudaStream_t s) {
    const size_t smem = sizeof(ConvSmem<R, T>);
    APRB_CUDA(cudaFuncSetAttribute(conv_tile_kernel<R, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((a.d.xn + kBX - 1) / kBX, (a.d.yn + kBY - 1) / kBY, (a.d.zn + kBZ - 1) / kBZ);
    conv_tile_kernel<R, T><<<grid, 32 * (kBX + 2 * R), smem, s>>>(a, xz_end, y_vec, in, t_xz_end, t_y_vec, tree, st,
                                                                  out, rl_in, stale);
    count_launch();
    APRB_CHECK_LAUNCH();
}

}  // namespace

void build_filter_index(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const Geom &tg,
                        const uint64_t *t_xz_end, const uint16_t *t_y_vec, FilterIndex &fi, cudaStream_t s) {
    APRB_PROF("filter_index", s);
    uint64_t total = 0;
    for (int l = g.l_min; l <= g.l_max; ++l) {
        fi.apr_off[l] = total;
        total += nrow(g, l) * (uint64_t)(nchunk(g.y_num[l]) + 1);
    }
    for (int t = tg.l_min; t <= tg.l_max; ++t) {
        fi.tree_off[t] = total;
        total += nrow(tg, t) * (uint64_t)(nchunk(tg.y_num[t]) + 1);
    }
    uint16_t *c = fi.buf.as<uint16_t>(total ? total : 1);
    for (int l = 0; l < 32; ++l) fi.level_count[l] = 0;
    for (int l = g.l_min; l <= g.l_max; ++l) {
        uint64_t be[2] = {0, 0};
        APRB_CUDA(cudaMemcpyAsync(&be[0], xz_end + g.level_xz[l] - 1, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        APRB_CUDA(cudaMemcpyAsync(&be[1], xz_end + g.level_xz[l + 1] - 1, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        APRB_CUDA(cudaStreamSynchronize(s));
        fi.level_count[l] = be[1] - be[0];
    }
    for (int l = g.l_min; l <= g.l_max; ++l) {
        const uint64_t rows = nrow(g, l);
        if (!rows) continue;
        chunk_index_kernel<<<blocks_for(rows * 32, 256), 256, 0, s>>>(xz_end, g.level_xz[l], y_vec, rows,
                                                                     nchunk(g.y_num[l]), c + fi.apr_off[l]);
        count_launch();
    }
    for (int t = tg.l_min; t <= tg.l_max; ++t) {
        const uint64_t rows = nrow(tg, t);
        if (!rows) continue;
        chunk_index_kernel<<<blocks_for(rows * 32, 256), 256, 0, s>>>(t_xz_end, tg.level_xz[t], t_y_vec, rows,
                                                                     nchunk(tg.y_num[t]), c + fi.tree_off[t]);
        count_launch();
    }
    APRB_CHECK_LAUNCH();
    fi.built = true;
}

template <typename T>
void filter_apply(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const Geom &tg,
                  const uint64_t *t_xz_end, const uint16_t *t_y_vec, const FilterIndex &fi, const T *in, T *tree,
                  const ConvPlan *plan, const T *d_stencils, T *out, int mode, const uint16_t *rl_in,
                  FilterBuffers &fb, cudaStream_t s) {
    APRB_PROF(plan ? "convolve" : "fill_tree_mean", s);
    const int L = g.l_max;
    const uint16_t *cbase = (const uint16_t *)fi.buf.p;
    unsigned long long *stale = fb.stale.as<unsigned long long>(1);
    APRB_CUDA(cudaMemsetAsync(stale, 0, sizeof(unsigned long long), s));
    // tree means, fine to coarse
    for (int t = tg.l_max; t >= tg.l_min; --t) {
        const int l = t + 1;  // child level
        if (l > L || l < g.l_min) continue;
        TreeLevelArgs ta;
        ta.dt = ld(tg, t);
        ta.dc = ld(g, l);
        ta.t_row_base = tg.level_xz[t];
        ta.c_row_base = g.level_xz[l];
        ta.ct_row_base = (l <= tg.l_max) ? tg.level_xz[l] : 0;
        ta.t_cidx = cbase + fi.tree_off[t];
        ta.c_cidx = cbase + fi.apr_off[l];
        ta.ct_cidx = (l <= tg.l_max) ? cbase + fi.tree_off[l] : nullptr;
        const uint64_t rows = (uint64_t)ta.dt.xn * ta.dt.zn;
        const unsigned ych = (unsigned)((ta.dt.yn + kTW - 1) / kTW);
        if (rows == 0 || ych == 0) continue;
        dim3 grid((unsigned)rows, ych);
        tree_mean_kernel<T><<<grid, 128, 0, s>>>(ta, xz_end, y_vec, in, t_xz_end, t_y_vec, tree);
        count_launch();
    }
    APRB_CHECK_LAUNCH();
    if (!plan) return;
    for (int l = L; l >= g.l_min; --l) {
        if (fi.level_count[l] == 0) continue;
        const int sn = std::min(plan->nstencils - 1, L - l);
        const int side = plan->sides[sn];
        const int r = (side - 1) / 2;
        const int max_npl = (int)std::ceil(std::log2((double)(r + 2)) - 1);
        const int npl = std::min(max_npl, l - g.l_min);
        ConvLevelArgs a;
        a.d = ld(g, l);
        a.dp = l > g.l_min ? ld(g, l - 1) : LD{1, 1, 1};
        a.row_base = g.level_xz[l];
        a.prow_base = npl >= 1 ? g.level_xz[l - 1] : 0;
        a.trow_base = l <= tg.l_max ? tg.level_xz[l] : 0;
        a.cidx = cbase + fi.apr_off[l];
        a.pcidx = npl >= 1 ? cbase + fi.apr_off[l - 1] : nullptr;
        a.tcidx = l <= tg.l_max ? cbase + fi.tree_off[l] : nullptr;
        a.reflect = plan->reflect;
        a.mode = mode;
        const T *st = d_stencils + plan->offsets[sn];
        if (side == 3)
            launch_conv_level<1, T>(a, xz_end, y_vec, in, t_xz_end, t_y_vec, tree, st, out, rl_in, stale, s);
        else
            launch_conv_level<2, T>(a, xz_end, y_vec, in, t_xz_end, t_y_vec, tree, st, out, rl_in, stale, s);
    }
}

template void filter_apply<float>(const Geom &, const uint64_t *, const uint16_t *, const Geom &, const uint64_t *,
                                  const uint16_t *, const FilterIndex &, const float *, float *, const ConvPlan *,
                                  const float *, float *, int, const uint16_t *, FilterBuffers &, cudaStream_t);
template void filter_apply<double>(const Geom &, const uint64_t *, const uint16_t *, const Geom &, const uint64_t *,
                                   const uint16_t *, const FilterIndex &, const double *, double *, const ConvPlan *,
                                   const double *, double *, int, const uint16_t *, FilterBuffers &, cudaStream_t);

uint64_t filter_stale_count(FilterBuffers &fb, cudaStream_t s) {
    unsigned long long v = 0;
    APRB_CUDA(cudaMemcpyAsync(&v, fb.stale.as<unsigned long long>(1), sizeof(v), cudaMemcpyDeviceToHost, s));
    APRB_CUDA(cudaStreamSynchronize(s));
    return v;
}

}  // namespace aprb
