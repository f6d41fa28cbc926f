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
// Convolution (APRFilter::convolve_pencil, APRFilter.hpp:1094-1216), per level
// from fine to coarse, in two kernels.  densify writes the level's isotropic
// neighbourhood image -- the values the reference gathers into its pencil
// buffer (update_dense_array, :825-849): same-level particles, parents one
// level coarser (piecewise constant, :766-793) and tree means of the same
// level (:802-818) -- to HBM once, one warp per row.  conv_gather then lets
// every particle of the level sum its 27 / 125 taps from that image in the
// stencil's memory order without contraction (run_convolution_pencil,
// :706-736), reading through L1/L2 (neighbouring rows are shared by the warps
// of a block), with the reflective or zero boundary (:287-504) applied to the
// indices.  A cell no particle covers holds a sentinel; reading it is counted
// as a stale read (the reference would read a stale pencil buffer there) and
// contributes 0.
#include <climits>

#include "kernels.cuh"
#include "tma.cuh"

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
uint64_t ncell_of(const LD &d) { return (uint64_t)d.yn * d.xn * d.zn; }
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

constexpr int kConvK = 4;  // output particles per lane and pass

// ---------------------------------------------------------------------------
// tree means of tree level t (children at level t+1)
// ---------------------------------------------------------------------------
constexpr int kTR = 2;  // parent rows per CTA
// parent cells per CTA along y (a multiple of kYC), within 48 KB of staging
template <typename T>
__host__ __device__ constexpr int tree_tw() {
    return sizeof(T) == 8 ? 256 : 512;
}

// Stage elements [s, e) of one row (y values Y, values X) into the shared
// row V / K (value, kind) at y - cy0.  With vec, whole aligned groups of four
// elements move as one 8-byte y load and one 16-byte (two for double) value
// load, two groups per lane in flight; the at most six elements in partial
// groups at the ends go one per lane.
template <typename T>
__device__ __forceinline__ void stage_row(const uint16_t *__restrict__ Y, const T *__restrict__ X, uint64_t s,
                                          uint64_t e, int cy0, T *V, uint8_t *K, uint8_t kind, int lane, int vec) {
    const int n = (int)(e - s);
    if (!vec) {
#pragma unroll 4
        for (int j = lane; j < n; j += 32) {
            const int yv = (int)Y[s + j] - cy0;
            V[yv] = X[s + j];
            K[yv] = kind;
        }
        return;
    }
    const int g0 = (int)(s & 3);
    const int gfirst = g0 ? 1 : 0, gend = (n + g0) >> 2;
    const int hend = min(n, 4 * gfirst - g0), tbeg = max(hend, 4 * gend - g0);
    if (lane < hend + (n - tbeg)) {
        const int j = lane < hend ? lane : tbeg + lane - hend;
        const int yv = (int)Y[s + j] - cy0;
        V[yv] = X[s + j];
        K[yv] = kind;
    }
    const uint64_t gb = s - (uint64_t)g0;  // element index of group 0 (a multiple of 4)
    constexpr int B = 2;  // groups per lane in flight (more cost resident CTAs: 4.11 / 3.82 / 4.34 / 5.31 ms for 1 / 2 / 3 / 4 at 1.1e9 particles)
    for (int gi0 = gfirst + lane; gi0 < gend; gi0 += 32 * B) {
        uint2 yy[B];
        T vv[B][4];
#pragma unroll
        for (int u = 0; u < B; ++u) {
            const int gi = gi0 + 32 * u;
            if (gi >= gend) continue;
            const uint64_t ge = gb + 4 * (uint64_t)gi;
            yy[u] = *reinterpret_cast<const uint2 *>(Y + ge);
            if constexpr (sizeof(T) == 4) {
                const float4 v = *reinterpret_cast<const float4 *>(X + ge);
                vv[u][0] = v.x, vv[u][1] = v.y, vv[u][2] = v.z, vv[u][3] = v.w;
            } else {
                const double2 v0 = *reinterpret_cast<const double2 *>(X + ge);
                const double2 v1 = *reinterpret_cast<const double2 *>(X + ge + 2);
                vv[u][0] = v0.x, vv[u][1] = v0.y, vv[u][2] = v1.x, vv[u][3] = v1.y;
            }
        }
#pragma unroll
        for (int u = 0; u < B; ++u) {
            if (gi0 + 32 * u >= gend) continue;
            const int y4[4] = {(int)(yy[u].x & 0xffffu), (int)(yy[u].x >> 16), (int)(yy[u].y & 0xffffu),
                               (int)(yy[u].y >> 16)};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                V[y4[q] - cy0] = vv[u][q];
                K[y4[q] - cy0] = kind;
            }
        }
    }
}

struct TreeLevelArgs {
    LD dt;                  // tree level t dims (== APR level t dims)
    LD dc;                  // child level dims
    uint64_t t_row_base;    // tree level_xz[t]
    uint64_t c_row_base;    // APR level_xz[t+1]
    uint64_t ct_row_base;   // tree level_xz[t+1] (0 when t+1 has no tree level)
    const uint16_t *t_cidx, *c_cidx, *ct_cidx;
    int vec;  // y arrays 8-byte and value arrays 16-byte aligned: group loads
};

template <typename T>
__global__ void __launch_bounds__(128 * kTR) tree_mean_kernel(TreeLevelArgs a, uint64_t rows,
                                                              const uint64_t *__restrict__ xz_end,
                                                              const uint16_t *__restrict__ y_vec,
                                                              const T *__restrict__ parts,
                                                              const uint64_t *__restrict__ t_xz_end,
                                                              const uint16_t *__restrict__ t_y_vec,
                                                              T *__restrict__ tree) {
    // kTR parent rows per CTA, four warps (one per child row) for each
    constexpr int TW = tree_tw<T>();
    __shared__ T sv[kTR][4][2 * TW];
    __shared__ __align__(4) uint8_t sk[kTR][4][2 * TW];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pr = w >> 2, q4 = w & 3;
    const uint64_t prow = (uint64_t)blockIdx.x * kTR + pr;  // parent row z*xt + x
    const bool row_ok = prow < rows;
    const int xp = row_ok ? (int)(prow % (uint64_t)a.dt.xn) : 0, zp = row_ok ? (int)(prow / (uint64_t)a.dt.xn) : 0;
    const int y0 = blockIdx.y * TW;
    const int cy0 = 2 * y0, cy1 = min(2 * y0 + 2 * TW, a.dc.yn);
    // the parent range is independent of the children: fetch it first
    uint64_t ps = 0, pend = 0;
    if (row_ok) {
        const int nct = nchunk(a.dt.yn);
        const uint64_t pb = t_xz_end[a.t_row_base + prow - 1];
        const uint16_t *PC = a.t_cidx + prow * (uint64_t)(nct + 1);
        ps = pb + PC[y0 / kYC];
        pend = pb + PC[min(y0 / kYC + TW / kYC, nct)];
    }
    for (int k = threadIdx.x; k < kTR * 4 * 2 * TW / 4; k += blockDim.x)
        reinterpret_cast<uint32_t *>(&sk[0][0][0])[k] = 0u;
    __syncthreads();
    {
        // warp (pr, q4) stages child row (2zp + q4/2, 2xp + q4%2): its
        // particles and tree nodes (disjoint cells) with y in [cy0, cy1).
        // cy0 and cy1 are chunk starts or the row end, so the chunk index
        // gives both ends of the ranges and successive passes' loads are
        // independent.
        const int cz = 2 * zp + (q4 >> 1), cx = 2 * xp + (q4 & 1);
        if (row_ok && cz < a.dc.zn && cx < a.dc.xn && cy0 < cy1) {
            const uint64_t row = (uint64_t)cz * a.dc.xn + cx;
            const int ncc = nchunk(a.dc.yn);
            const uint16_t *CC = a.c_cidx + row * (uint64_t)(ncc + 1);
            const int c0 = cy0 / kYC, c1 = cy1 == a.dc.yn ? ncc : cy1 / kYC;
            const uint64_t r0 = xz_end[a.c_row_base + row - 1];
            const uint64_t s0 = r0 + CC[c0], e0 = r0 + CC[c1];
            T *V = sv[pr][q4];
            uint8_t *K = sk[pr][q4];
            stage_row<T>(y_vec, parts, s0, e0, cy0, V, K, 1, lane, a.vec);
            if (a.ct_row_base) {
                const uint16_t *CT = a.ct_cidx + row * (uint64_t)(ncc + 1);
                const uint64_t r1 = t_xz_end[a.ct_row_base + row - 1];
                const uint64_t s1 = r1 + CT[c0], e1 = r1 + CT[c1];
                stage_row<T>(t_y_vec, tree, s1, e1, cy0, V, K, 2, lane, a.vec);
            }
        }
    }
    __syncthreads();
    if (!row_ok) return;
    float sxz = (float)((((2 * a.dt.xn != a.dc.xn) && (xp == a.dt.xn - 1)) +
                         ((2 * a.dt.zn != a.dc.zn) && (zp == a.dt.zn - 1))) * 2);
    if (sxz == 0) sxz = 1;
    const float syxz = (2 * a.dt.yn != a.dc.yn) ? sxz * 2 : sxz;
    // x / 8 == x * 0.125 exactly: both are the correctly rounded x / 8
    const T eighth = T(0.125);
    for (uint64_t i = ps + (threadIdx.x & 127); i < pend; i += 128) {
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
                    if (o + d < cy1 - cy0 && sk[pr][q][o + d] == kind)
                        acc = VT<T>::add(VT<T>::mul(VT<T>::mul(T(s), sv[pr][q][o + d]), eighth), acc);
        tree[i] = acc;
    }
}

// ---------------------------------------------------------------------------
// convolution of one level
// ---------------------------------------------------------------------------
struct ConvLevelArgs {
    LD d;                 // level dims
    LD dp;                // parent level dims
    uint64_t row_base;    // APR level_xz[l]
    uint64_t prow_base;   // APR level_xz[l-1] (0: no parents used)
    uint64_t trow_base;   // tree level_xz[l] (0: no tree level)
    const uint16_t *cidx, *pcidx, *tcidx;
    int reflect;
    int mode;
    int rad;  // stencil radius of the level (densify skips rows no stencil reaches)
};

// ---------------------------------------------------------------------------
// convolution of one level in two kernels: the level's isotropic
// neighbourhood image is written to HBM once (densify), then every particle
// of the level gathers its taps from it (conv_gather)
// ---------------------------------------------------------------------------

// densify: one warp per row (z, x) of level l.  Cells start as the sentinel;
// same-level particles, the parents one level coarser (each covering its y
// pair) and the tree means of the level write their cells.  The three sources
// cover disjoint cells (APR particle cells partition the volume).
template <typename T>
__global__ void __launch_bounds__(256) densify_kernel(ConvLevelArgs a, const uint64_t *__restrict__ xz_end,
                                                      const uint16_t *__restrict__ y_vec, const T *__restrict__ in,
                                                      const uint64_t *__restrict__ t_xz_end,
                                                      const uint16_t *__restrict__ t_y_vec,
                                                      const T *__restrict__ tree, T *__restrict__ D) {
    const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= (uint64_t)a.d.xn * a.d.zn) return;
    {
        // only rows within the stencil radius of a row holding particles of the
        // level are ever read by conv_gather
        const int z = (int)(row / (uint64_t)a.d.xn), x = (int)(row % (uint64_t)a.d.xn);
        const int S = 2 * a.rad + 1;
        bool any = false;
        for (int k = lane; k < S * S; k += 32) {
            const int zz = z + k / S - a.rad, xx = x + k % S - a.rad;
            if (zz >= 0 && zz < a.d.zn && xx >= 0 && xx < a.d.xn) {
                const uint64_t r = (uint64_t)zz * a.d.xn + xx;
                any = any || xz_end[a.row_base + r] > xz_end[a.row_base + r - 1];
            }
        }
        if (!__any_sync(0xffffffffu, any)) return;
    }
    const int yn = a.d.yn;
    T *Rw = D + row * (uint64_t)yn;
    const T miss = VT<T>::miss();
    if ((yn * sizeof(T)) % 16 == 0) {  // 16-byte rows: vector stores
        constexpr int V = 16 / sizeof(T);
        T pack[V];
#pragma unroll
        for (int k = 0; k < V; ++k) pack[k] = miss;
        const uint4 m4 = *reinterpret_cast<const uint4 *>(pack);
        uint4 *R4 = reinterpret_cast<uint4 *>(Rw);
        for (int k = lane; k < yn / V; k += 32) R4[k] = m4;
    } else {
        for (int y = lane; y < yn; y += 32) Rw[y] = miss;
    }
    __syncwarp();
    {
        const uint64_t b = xz_end[a.row_base + row - 1], e = xz_end[a.row_base + row];
        for (uint64_t i = b + lane; i < e; i += 32) Rw[y_vec[i]] = in[i];
    }
    if (a.prow_base) {
        const int zr = (int)(row / (uint64_t)a.d.xn), xr = (int)(row % (uint64_t)a.d.xn);
        const uint64_t prow = (uint64_t)(zr / 2) * a.dp.xn + xr / 2;
        const uint64_t b = xz_end[a.prow_base + prow - 1], e = xz_end[a.prow_base + prow];
        for (uint64_t i = b + lane; i < e; i += 32) {
            const int c0 = 2 * (int)y_vec[i], c1 = min(c0 + 1, yn - 1);
            const T v = in[i];
            Rw[c0] = v;
            if (c1 != c0) Rw[c1] = v;
        }
    }
    if (a.trow_base) {
        const uint64_t b = t_xz_end[a.trow_base + row - 1], e = t_xz_end[a.trow_base + row];
        for (uint64_t i = b + lane; i < e; i += 32) Rw[t_y_vec[i]] = tree[i];
    }
}

// One tap outside the fast path: reflection about the edge sample (or the
// zero pad), and the sentinel of an uncovered cell counted as a stale read.
template <typename T>
__device__ __forceinline__ T gather_tap(const T *__restrict__ D, const ConvLevelArgs &a, int zz, int xx, int yy,
                                        unsigned &nstale) {
    bool ok = true;
    const int zr = reflect_idx(zz, a.d.zn, a.reflect, ok);
    const int xr = reflect_idx(xx, a.d.xn, a.reflect, ok);
    const int yr = reflect_idx(yy, a.d.yn, a.reflect, ok);
    if (!ok) {
        if (a.reflect) nstale++;
        return T(0);
    }
    const T v = D[((uint64_t)zr * a.d.xn + xr) * (uint64_t)a.d.yn + yr];
    if (VT<T>::is_miss(v)) {
        nstale++;
        return T(0);
    }
    return v;
}

// conv_gather: one warp per row of level l; each lane takes kConvK particles
// of the row (two in FP64, where four cost more in registers than they
// save).  A z-slice of the stencil sits in registers; the taps are
// summed in the stencil's memory order without contraction
// (run_convolution_pencil, APRFilter.hpp:706-736).  Particles whose window
// stays inside the level read D directly; a NaN sum (a sentinel was read) is
// redone through gather_tap, which counts stale reads.
template <int R, typename T>
__global__ void __launch_bounds__(256) conv_gather_kernel(ConvLevelArgs a, const uint64_t *__restrict__ xz_end,
                                                          const uint16_t *__restrict__ y_vec, const T *__restrict__ D,
                                                          const T *__restrict__ stencil, T *__restrict__ out,
                                                          const uint16_t *__restrict__ rl_in,
                                                          unsigned long long *stale) {
    constexpr int S = 2 * R + 1, S3 = S * S * S;
    constexpr int K = sizeof(T) == 8 ? 2 : kConvK;  // particles per lane: two in FP64
    __shared__ T st[S3];
    for (int k = threadIdx.x; k < S3; k += blockDim.x) st[k] = stencil[k];
    __syncthreads();
    const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= (uint64_t)a.d.xn * a.d.zn) return;
    const uint64_t b = xz_end[a.row_base + row - 1], e = xz_end[a.row_base + row];
    if (b == e) return;
    const int z = (int)(row / (uint64_t)a.d.xn), x = (int)(row % (uint64_t)a.d.xn);
    const int yn = a.d.yn;
    // the S x S neighbour rows lie inside the level (warp-uniform)
    const bool rows_in = z - R >= 0 && z + R < a.d.zn && x - R >= 0 && x + R < a.d.xn;
    unsigned nstale = 0;
    for (uint64_t base = b; base < e; base += 32 * K) {
        uint64_t ii[K];
        int yv[K];
        bool has[K];
        bool inner = rows_in;
#pragma unroll
        for (int j = 0; j < K; ++j) {
            ii[j] = base + (uint64_t)(j * 32 + lane);
            has[j] = ii[j] < e;
            yv[j] = has[j] ? (int)y_vec[ii[j]] : R;
            inner = inner && yv[j] - R >= 0 && yv[j] + R < yn;
        }
        T acc[K];
#pragma unroll
        for (int j = 0; j < K; ++j) acc[j] = T(0);
        if (inner) {
#pragma unroll 1
            for (int iz = 0; iz < S; ++iz) {
                T stv[S * S];
#pragma unroll
                for (int t = 0; t < S * S; ++t) stv[t] = st[iz * S * S + t];
                // each particle's tap pointers step by one row per ix; the
                // y taps are immediate offsets from them
                const T *row0 = D + ((uint64_t)(z + iz - R) * a.d.xn + (uint64_t)(x - R)) * (uint64_t)yn - R;
                const T *p[K];
#pragma unroll
                for (int j = 0; j < K; ++j) p[j] = row0 + yv[j];
#pragma unroll
                for (int ix = 0; ix < S; ++ix) {
#pragma unroll
                    for (int iy = 0; iy < S; ++iy)
#pragma unroll
                        for (int j = 0; j < K; ++j)
                            acc[j] = VT<T>::add(acc[j], VT<T>::mul(__ldg(p[j] + iy), stv[ix * S + iy]));
#pragma unroll
                    for (int j = 0; j < K; ++j) p[j] += yn;
                }
            }
        }
#pragma unroll
        for (int j = 0; j < K; ++j) {
            if (!has[j]) continue;
            T val = acc[j];
            if (!inner || val != val) {
                val = T(0);
                int cnt = 0;
                for (int iz = 0; iz < S; ++iz)
                    for (int ix = 0; ix < S; ++ix)
                        for (int iy = 0; iy < S; ++iy) {
                            const T v = gather_tap(D, a, z + iz - R, x + ix - R, yv[j] + iy - R, nstale);
                            val = VT<T>::add(val, VT<T>::mul(v, st[cnt++]));
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
    if (nstale) atomicAdd(stale, (unsigned long long)nstale);
}

template <int R, typename T>
void launch_conv_level_dense(const ConvLevelArgs &a, const uint64_t *xz_end, const uint16_t *y_vec, const T *in,
                             const uint64_t *t_xz_end, const uint16_t *t_y_vec, const T *tree, const T *st, T *out,
                             const uint16_t *rl_in, unsigned long long *stale, T *D, cudaStream_t s) {
    const uint64_t rows = (uint64_t)a.d.xn * a.d.zn;
    {
        APRB_PROF("densify", s);
        densify_kernel<T><<<blocks_for(rows * 32, 256), 256, 0, s>>>(a, xz_end, y_vec, in, t_xz_end, t_y_vec, tree, D);
        count_launch();
        APRB_CHECK_LAUNCH();
    }
    APRB_PROF("conv_gather", s);
    conv_gather_kernel<R, T><<<blocks_for(rows * 32, 256), 256, 0, s>>>(a, xz_end, y_vec, D, st, out, rl_in, stale);
    count_launch();
    APRB_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------
// convolution of one level in one z-streaming kernel: the neighbourhood is
// built in shared memory from the sparse rows, nothing of it goes to HBM
// ---------------------------------------------------------------------------
// A CTA owns TX rows (x) x TY cells (y) of the level and a run of up to kSZ
// planes.  It keeps the S = 2R + 1 planes around the current one in a ring,
// each plane (TX + 2R) rows x (TY + 2R) cells: the cells densify writes
// (same-level particles, parents one level coarser over their y pair, tree
// means of the level) with the boundary folded in -- a cell outside the level
// holds the value of its reflection (the sentinel when the reflection leaves
// the level too), or 0 with the zero pad -- so every tap is a shared-memory
// load at a fixed offset.  Planes with no particle of the level within R are
// never built.  Per plane: (1) the new planes are prefilled with the sentinel
// while one thread per (row, source) finds the source's range from the chunk
// index; (2) a warp per (row, source) scatters the elements, four per lane in
// flight; (3) warp r sums the taps of centre row r's particles in the
// stencil's memory order, two per lane, and a NaN sum is recomputed tap by
// tap with the sentinel counted as a stale read.
constexpr int kSThreads = 256;
constexpr int kSZ = 64;  // planes per CTA run at most (one bit each of a 64-bit mask)

template <int R, typename T>
struct StreamShape {
    static constexpr int S = 2 * R + 1, S3 = S * S * S;
    static constexpr int TX = 8;
    static constexpr int TY = sizeof(T) == 4 ? (R == 1 ? 512 : 256) : (R == 1 ? 256 : 128);
    static constexpr int NR = TX + 2 * R, PY = TY + 2 * R, PLANE = NR * PY;
    static constexpr int NT = 3 * NR;                  // fill tasks (row, source) of one plane
    static constexpr int MT = S * NT;                  // at most S planes are built at once
    static constexpr size_t smem = (size_t)S * PLANE * sizeof(T) + (size_t)MT * 16 + 8 + TX * 12;
    static_assert((PLANE * sizeof(T)) % 16 == 0, "planes keep 16-byte alignment");
    static_assert(TY % kYC == 0, "tiles start on chunk boundaries");
};

template <int R, typename T>
struct StencilArg;
template <int R>
struct StencilArg<R, float> {
    float w[(2 * R + 1) * (2 * R + 1) * (2 * R + 1)];
};
template <int R>
struct StencilArg<R, double> {
    double w[(2 * R + 1) * (2 * R + 1) * (2 * R + 1)];
};

// source index of index i of an axis of length n: i itself, its reflection
// about the edge sample, or -1 (zero pad, or a reflection that leaves the axis)
__device__ __forceinline__ int src_index(int i, int n, int reflect) {
    if (i >= 0 && i < n) return i;
    if (!reflect) return -1;
    const int r = i < 0 ? -i : 2 * (n - 1) - i;
    return (r >= 0 && r < n) ? r : -1;
}

template <typename T>
__device__ __forceinline__ uint4 miss4() {
    T p[16 / sizeof(T)];
#pragma unroll
    for (int k = 0; k < (int)(16 / sizeof(T)); ++k) p[k] = VT<T>::miss();
    return *reinterpret_cast<const uint4 *>(p);
}

// Tap sums of two particles at plane offsets oa / ob (slot of the first plane
// sl0) in the stencil's memory order, scalar multiplies and adds with the
// weights read from the kernel's parameters.  (The paired f32x2 multiply
// needs the weights in registers, which costs a third resident CTA per SM;
// and a paired multiply followed by a paired add is contracted into a fused
// multiply-add by the code generator even with explicit round-to-nearest and
// fmad off -- about half of all 27-tap sums differed.)
template <int R, int PY, int PLANE>
__device__ __forceinline__ float2 taps2(const float *__restrict__ planes, int sl0, int oa, int ob,
                                        const StencilArg<R, float> &sw) {
    constexpr int S = 2 * R + 1;
    float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int iz = 0; iz < S; ++iz) {
        int sl = sl0 + iz;
        if (sl >= S) sl -= S;
        const float *P = planes + sl * PLANE;
        const float *pa = P + oa, *pb = P + ob;
#pragma unroll
        for (int ix = 0; ix < S; ++ix)
#pragma unroll
            for (int iy = 0; iy < S; ++iy) {
                const int o = ix * PY + iy;
                const float w = sw.w[(iz * S + ix) * S + iy];
                acc.x = __fadd_rn(acc.x, __fmul_rn(pa[o], w));
                acc.y = __fadd_rn(acc.y, __fmul_rn(pb[o], w));
            }
    }
    return acc;
}

template <int R, int PY, int PLANE>
__device__ __forceinline__ double2 taps2(const double *__restrict__ planes, int sl0, int oa, int ob,
                                         const StencilArg<R, double> &sw) {
    constexpr int S = 2 * R + 1;
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll 1
    for (int iz = 0; iz < S; ++iz) {
        int sl = sl0 + iz;
        if (sl >= S) sl -= S;
        const double *P = planes + sl * PLANE;
        const double *pa = P + oa, *pb = P + ob;
#pragma unroll
        for (int ix = 0; ix < S; ++ix)
#pragma unroll
            for (int iy = 0; iy < S; ++iy) {
                const int o = ix * PY + iy;
                const double w = sw.w[(iz * S + ix) * S + iy];
                acc.x = __dadd_rn(acc.x, __dmul_rn(pa[o], w));
                acc.y = __dadd_rn(acc.y, __dmul_rn(pb[o], w));
            }
    }
    return acc;
}

template <int R, typename T>
__global__ void __launch_bounds__(kSThreads, 3) conv_stream_kernel(
    ConvLevelArgs a, const __grid_constant__ StencilArg<R, T> sw, const uint64_t *__restrict__ xz_end,
    const uint16_t *__restrict__ y_vec, const T *__restrict__ in, const uint64_t *__restrict__ t_xz_end,
    const uint16_t *__restrict__ t_y_vec, const T *__restrict__ tree, const T *__restrict__ st,
    T *__restrict__ out, const uint16_t *__restrict__ rl_in, unsigned long long *stale, int zrun) {
    using SS = StreamShape<R, T>;
    constexpr int S = SS::S, TX = SS::TX, TY = SS::TY, NR = SS::NR, PY = SS::PY, PLANE = SS::PLANE;
    constexpr int NT = SS::NT, MT = SS::MT;
    constexpr int NW = kSThreads / 32;
    static_assert(NW == TX, "one warp per centre row");
    extern __shared__ __align__(16) unsigned char smraw[];
    T *planes = reinterpret_cast<T *>(smraw);
    uint64_t *task_s = reinterpret_cast<uint64_t *>(planes + S * PLANE);  // task: first index
    uint32_t *task_n = reinterpret_cast<uint32_t *>(task_s + MT);         // task: elements
    uint32_t *task_m = task_n + MT;                                       // slot << 8 | row << 2 | source
    uint64_t *cfirst = reinterpret_cast<uint64_t *>(task_m + MT + (MT & 1));  // centre rows: first index
    uint32_t *ccnt = reinterpret_cast<uint32_t *>(cfirst + TX);             // centre rows: particles
    __shared__ unsigned long long zmask;

    const int yn = a.d.yn, xn = a.d.xn, zn = a.d.zn;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, zs = blockIdx.z * zrun, ze = min(zs + zrun, zn);
    const int wy0 = max(0, y0 - R), wy1 = min(yn, y0 + TY + R);  // cells of the window inside the level
    const int nc = nchunk(yn), ncp = nchunk(a.dp.yn);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int cc0 = y0 / kYC, cc1 = min((y0 + TY) / kYC, nc);  // centre cells: exactly these chunks

    // planes of the run with particles of the level in the tile
    if (tid == 0) zmask = 0ull;
    __syncthreads();
    for (int k = tid; k < (ze - zs) * TX; k += kSThreads) {
        const int x = x0 + k % TX;
        if (x < xn) {
            const uint64_t row = (uint64_t)(zs + k / TX) * xn + x;
            const uint16_t *C = a.cidx + row * (uint64_t)(nc + 1);
            if (C[cc0] != C[cc1]) atomicOr(&zmask, 1ull << (k / TX));
        }
    }
    __syncthreads();
    const unsigned long long zm = zmask;
    if (zm == 0ull) return;

    const bool mirror = a.reflect && (y0 - R < 0 || y0 + TY + R > yn);
    const bool vec_prefill = a.reflect || (x0 - R >= 0 && x0 + TX + R <= xn && y0 - R >= 0 && y0 + TY + R <= yn);
    unsigned nstale = 0;
    int top = INT_MIN / 2;  // planes (top - S, top] sit in their slots
    for (int z = zs; z < ze; ++z) {
        if (!((zm >> (z - zs)) & 1ull)) continue;
        const int f0 = max(z - R, top + 1), nfill = z + R - f0 + 1;  // planes f0 .. z + R are built now
        top = z + R;
        const int ntask = nfill * NT;
        // (1) source ranges of the new planes (one thread per task), the
        // centre rows (the last warp) and the prefill (everyone)
        for (int k = tid; k < ntask; k += kSThreads) {
            const int zz = f0 + k / NT, rem = k % NT, src = rem / NR, r = rem % NR;
            const int zsrc = src_index(zz, zn, a.reflect), xsrc = src_index(x0 - R + r, xn, a.reflect);
            uint64_t s = 0;
            int n = 0;
            if (zsrc >= 0 && xsrc >= 0) {
                if (src == 0 || (src == 2 && a.trow_base)) {
                    const uint64_t row = (uint64_t)zsrc * xn + xsrc;
                    const uint16_t *C = (src == 0 ? a.cidx : a.tcidx) + row * (uint64_t)(nc + 1);
                    const uint64_t rs = src == 0 ? xz_end[a.row_base + row - 1] : t_xz_end[a.trow_base + row - 1];
                    const int c0 = C[wy0 / kYC];
                    s = rs + c0;
                    n = C[(wy1 + kYC - 1) / kYC] - c0;
                } else if (src == 1 && a.prow_base) {
                    const uint64_t prow = (uint64_t)(zsrc / 2) * a.dp.xn + xsrc / 2;
                    const int pv0 = wy0 / 2, pv1 = min((wy1 + 1) / 2, a.dp.yn);
                    const uint16_t *C = a.pcidx + prow * (uint64_t)(ncp + 1);
                    const int c0 = C[pv0 / kYC];
                    s = xz_end[a.prow_base + prow - 1] + c0;
                    n = C[min((pv1 + kYC - 1) / kYC, ncp)] - c0;
                }
            }
            task_s[k] = s;
            task_n[k] = (uint32_t)n;
            task_m[k] = (uint32_t)((((zz + S) % S) << 8) | (r << 2) | src);
        }
        if (warp == NW - 1 && lane < TX) {
            const int x = x0 + lane;
            uint64_t f = 0;
            int n = 0;
            if (x < xn) {
                const uint64_t row = (uint64_t)z * xn + x;
                const uint16_t *C = a.cidx + row * (uint64_t)(nc + 1);
                f = xz_end[a.row_base + row - 1] + C[cc0];
                n = C[cc1] - C[cc0];
            }
            cfirst[lane] = f;
            ccnt[lane] = (uint32_t)n;
        }
        for (int p = 0; p < nfill; ++p) {
            const int zz = f0 + p;
            T *P = planes + ((zz + S) % S) * PLANE;
            if (vec_prefill && (a.reflect || (zz >= 0 && zz < zn))) {
                const uint4 m4 = miss4<T>();
                for (int k = tid; k < (int)(PLANE * sizeof(T) / 16); k += kSThreads)
                    reinterpret_cast<uint4 *>(P)[k] = m4;
            } else {
                for (int k = tid; k < PLANE; k += kSThreads) {
                    const int xr = x0 - R + k / PY, yy = y0 - R + k % PY;
                    const bool in_level = zz >= 0 && zz < zn && xr >= 0 && xr < xn && yy >= 0 && yy < yn;
                    P[k] = (a.reflect || in_level) ? VT<T>::miss() : T(0);
                }
            }
        }
        __syncthreads();
        // (2) scatter: a warp per task, its lanes over the task's elements,
        // four per lane in flight
        for (int t = warp; t < ntask; t += NW) {
            const int n = (int)task_n[t];
            if (n == 0) continue;
            const uint32_t m = task_m[t];
            const uint64_t s = task_s[t];
            const int src = m & 3;
            T *row = planes + (m >> 8) * PLANE + ((m >> 2) & 63) * PY - (y0 - R);  // [cell y]
            const uint16_t *YV = (src == 2 ? t_y_vec : y_vec) + s;
            const T *V = (src == 2 ? tree : in) + s;
            auto put = [&](int c, T v) {
                if (c >= wy0 && c < wy1) row[c] = v;
                if (mirror) {
                    if (c > 0 && -c >= y0 - R) row[-c] = v;
                    const int m2 = 2 * (yn - 1) - c;
                    if (c <= yn - 2 && m2 < y0 + TY + R) row[m2] = v;
                }
            };
            for (int j0 = lane; j0 < n; j0 += 128) {
                int yv[4];
                T vv[4];
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    const int j = j0 + 32 * h;
                    yv[h] = -1;
                    if (j < n) {
                        yv[h] = YV[j];
                        vv[h] = V[j];
                    }
                }
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    if (yv[h] < 0) continue;
                    if (src != 1) {
                        put(yv[h], vv[h]);
                    } else {
                        const int c0 = 2 * yv[h], c1 = min(c0 + 1, yn - 1);
                        put(c0, vv[h]);
                        if (c1 != c0) put(c1, vv[h]);
                    }
                }
            }
        }
        __syncthreads();
        // (3) the centre plane: warp r takes centre row r, each lane the
        // particles k = k0 + lane and k0 + lane + 32 (the next pair's y
        // loaded before the taps of this one)
        {
            const int r = warp;
            const int n = (int)ccnt[r];
            const uint64_t f = cfirst[r];
            const uint16_t *YV = y_vec + f;
            const int sl0 = (z - R + S) % S;
            int ya = lane < n ? (int)YV[lane] : y0, yb = lane + 32 < n ? (int)YV[lane + 32] : y0;
            for (int k0 = 0; k0 < n; k0 += 64) {
                const int ka = k0 + lane, kb = ka + 32;
                const int oa = r * PY + ya - y0, ob = r * PY + yb - y0;
                if (k0 + 64 < n) {
                    ya = ka + 64 < n ? (int)YV[ka + 64] : y0;
                    yb = kb + 64 < n ? (int)YV[kb + 64] : y0;
                }
                if (ka >= n) break;
                const auto acc = taps2<R, PY, PLANE>(planes, sl0, oa, ob, sw);
                const T val[2] = {acc.x, acc.y};
                const int off[2] = {oa, ob};
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int k = ka + 32 * h;
                    if (k >= n) break;
                    T v = val[h];
                    if (v != v) {
                        v = T(0);
                        int cnt = 0;
                        for (int iz = 0; iz < S; ++iz) {
                            int sl = sl0 + iz;
                            if (sl >= S) sl -= S;
                            const T *P = planes + sl * PLANE + off[h];
                            for (int ix = 0; ix < S; ++ix)
                                for (int iy = 0; iy < S; ++iy) {
                                    T d = P[ix * PY + iy];
                                    if (VT<T>::is_miss(d)) {
                                        nstale++;
                                        d = T(0);
                                    }
                                    v = VT<T>::add(v, VT<T>::mul(d, st[cnt++]));
                                }
                        }
                    }
                    const uint64_t i = f + (uint64_t)k;
                    if (a.mode == 0)
                        out[i] = v;
                    else if (a.mode == 1)
                        out[i] = VT<T>::div((T)rl_in[i], v);
                    else
                        out[i] = VT<T>::mul(out[i], v);
                }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nstale += __shfl_down_sync(0xffffffffu, nstale, o);
    if (lane == 0 && nstale) atomicAdd(stale, (unsigned long long)nstale);
}

// The streaming kernel of one level; false (nothing launched) when the
// stencil values are not on the host.
template <int R, typename T>
bool launch_conv_level_stream(const ConvLevelArgs &a, const ConvPlan &plan, int sn, const uint64_t *xz_end,
                              const uint16_t *y_vec, const T *in, const uint64_t *t_xz_end, const uint16_t *t_y_vec,
                              const T *tree, const T *st, T *out, const uint16_t *rl_in,
                              unsigned long long *stale, cudaStream_t s) {
    using SS = StreamShape<R, T>;
    if (plan.values.size() < (size_t)plan.offsets[sn] + SS::S3) return false;
    StencilArg<R, T> sw;
    for (int t = 0; t < SS::S3; ++t) {
        const T w = (T)plan.values[plan.offsets[sn] + t];
        sw.w[t] = w;
    }
    APRB_PROF("conv_stream", s);
    set_smem_once<conv_stream_kernel<R, T>>((int)SS::smem);
    // runs of kSZ planes, shorter (down to 8) on levels too small to give
    // every SM two waves of its three CTAs
    const unsigned gx = (unsigned)((a.d.xn + SS::TX - 1) / SS::TX), gy = (unsigned)((a.d.yn + SS::TY - 1) / SS::TY);
    int zrun = kSZ;
    while (zrun > 8 && (uint64_t)gx * gy * ((a.d.zn + zrun - 1) / zrun) < 2ull * 3 * 148) zrun /= 2;
    dim3 grid(gx, gy, (unsigned)((a.d.zn + zrun - 1) / zrun));
    conv_stream_kernel<R, T><<<grid, kSThreads, SS::smem, s>>>(a, sw, xz_end, y_vec, in, t_xz_end, t_y_vec, tree,
                                                                st, out, rl_in, stale, zrun);
    count_launch();
    APRB_CHECK_LAUNCH();
    return true;
}

// Gradient magnitude of one level (APRNumerics::gradient_magnitude_cfd /
// _sobel, APRNumerics.hpp:227-287) in one pass over the level's
// neighbourhood image: every direction's 3x3x3 stencil with its zero taps
// dropped and the others kept in memory order, then y^2 (+ x^2) (+ z^2) and
// the square root, as the per-direction path (one convolution per
// direction, squares and a root) computes them.  A zero tap adds +-0 to a
// finite sum, which changes the sum only when it is itself zero, and then
// only its sign, which the square removes.  Each cell of the union of the
// directions' taps is loaded once.
struct GradTaps {
    int nu;         // cells with a nonzero weight in some direction, memory order
    int active[3];  // direction enters the magnitude
    float w[27][3]; // weights of those cells per direction (0: tap dropped)
    signed char dz[27], dx[27], dy[27];
};

template <int K>
__global__ void __launch_bounds__(256) grad_mag_gather_kernel(ConvLevelArgs a, const uint64_t *__restrict__ xz_end,
                                                              const uint16_t *__restrict__ y_vec,
                                                              const float *__restrict__ D, GradTaps gt,
                                                              float *__restrict__ out, unsigned long long *stale) {
    __shared__ long long so[27];
    __shared__ float sw[27][3];
    const int yn = a.d.yn;
    for (int k = threadIdx.x; k < 27; k += blockDim.x) {
        so[k] = ((long long)gt.dz[k] * a.d.xn + gt.dx[k]) * (long long)yn + gt.dy[k];
        sw[k][0] = gt.w[k][0];
        sw[k][1] = gt.w[k][1];
        sw[k][2] = gt.w[k][2];
    }
    __syncthreads();
    const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= (uint64_t)a.d.xn * a.d.zn) return;
    const uint64_t b = xz_end[a.row_base + row - 1], e = xz_end[a.row_base + row];
    if (b == e) return;
    const int z = (int)(row / (uint64_t)a.d.xn), x = (int)(row % (uint64_t)a.d.xn);
    const bool rows_in = z - 1 >= 0 && z + 1 < a.d.zn && x - 1 >= 0 && x + 1 < a.d.xn;
    const float *Drow = D + ((uint64_t)z * a.d.xn + (uint64_t)x) * (uint64_t)yn;
    const int nu = gt.nu;
    unsigned nstale = 0;
    for (uint64_t base = b; base < e; base += 32 * K) {
        uint64_t ii[K];
        int yv[K];
        bool has[K];
        bool inner = rows_in;
#pragma unroll
        for (int j = 0; j < K; ++j) {
            ii[j] = base + (uint64_t)(j * 32 + lane);
            has[j] = ii[j] < e;
            yv[j] = has[j] ? (int)y_vec[ii[j]] : 1;
            inner = inner && yv[j] - 1 >= 0 && yv[j] + 1 < yn;
        }
        float g[3][K];
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
            for (int j = 0; j < K; ++j) g[d][j] = 0.0f;
        if (inner) {
            // one load per cell, every direction with a weight there in turn:
            // each direction still sums its taps in memory order
            for (int c = 0; c < nu; ++c) {
                const long long o = so[c];
                const float w0 = sw[c][0], w1 = sw[c][1], w2 = sw[c][2];
                float v[K];
#pragma unroll
                for (int j = 0; j < K; ++j) v[j] = __ldg(Drow + yv[j] + o);
                if (w0 != 0.0f) {
#pragma unroll
                    for (int j = 0; j < K; ++j) g[0][j] = __fadd_rn(g[0][j], __fmul_rn(v[j], w0));
                }
                if (w1 != 0.0f) {
#pragma unroll
                    for (int j = 0; j < K; ++j) g[1][j] = __fadd_rn(g[1][j], __fmul_rn(v[j], w1));
                }
                if (w2 != 0.0f) {
#pragma unroll
                    for (int j = 0; j < K; ++j) g[2][j] = __fadd_rn(g[2][j], __fmul_rn(v[j], w2));
                }
            }
        }
#pragma unroll
        for (int j = 0; j < K; ++j) {
            if (!has[j]) continue;
            float gv[3] = {g[0][j], g[1][j], g[2][j]};
            bool redo = !inner;
#pragma unroll
            for (int d = 0; d < 3; ++d) redo = redo || gv[d] != gv[d];
            if (redo) {
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    float acc = 0.0f;
                    for (int c = 0; c < nu; ++c) {
                        const float w = gt.w[c][d];
                        if (w == 0.0f) continue;
                        const float vv = gather_tap(D, a, z + gt.dz[c], x + gt.dx[c], yv[j] + gt.dy[c], nstale);
                        acc = __fadd_rn(acc, __fmul_rn(vv, w));
                    }
                    gv[d] = acc;
                }
            }
            float m = __fmul_rn(gv[0], gv[0]);
            if (gt.active[1]) m = __fadd_rn(m, __fmul_rn(gv[1], gv[1]));
            if (gt.active[2]) m = __fadd_rn(m, __fmul_rn(gv[2], gv[2]));
            out[ii[j]] = __fsqrt_rn(m);
        }
    }
    if (nstale) atomicAdd(stale, (unsigned long long)nstale);
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

// Tree means of every tree level, fine to coarse.
template <typename T>
static void tree_means_all(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const Geom &tg,
                           const uint64_t *t_xz_end, const uint16_t *t_y_vec, const FilterIndex &fi, const T *in,
                           T *tree, cudaStream_t s) {
    APRB_PROF("tree_mean", s);
    const int L = g.l_max;
    const uint16_t *cbase = (const uint16_t *)fi.buf.p;
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
        auto al = [](const void *p, uintptr_t b) { return ((uintptr_t)p & (b - 1)) == 0; };
        ta.vec = al(y_vec, 8) && al(t_y_vec, 8) && al(in, 16) && al(tree, 16);
        const uint64_t rows = (uint64_t)ta.dt.xn * ta.dt.zn;
        const unsigned ych = (unsigned)((ta.dt.yn + tree_tw<T>() - 1) / tree_tw<T>());
        if (rows == 0 || ych == 0) continue;
        dim3 grid((unsigned)((rows + kTR - 1) / kTR), ych);
        tree_mean_kernel<T><<<grid, 128 * kTR, 0, s>>>(ta, rows, xz_end, y_vec, in, t_xz_end, t_y_vec, tree);
        count_launch();
    }
    APRB_CHECK_LAUNCH();
}

// Neighbourhood arguments of level l for a stencil of the given side
// (parents used up to ceil(log2(r + 2) - 1) levels coarser, APRFilter.hpp:1118-1124).
static ConvLevelArgs conv_level_args(const Geom &g, const Geom &tg, const FilterIndex &fi, int l, int side,
                                     int reflect, int mode) {
    const uint16_t *cbase = (const uint16_t *)fi.buf.p;
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
    a.reflect = reflect;
    a.mode = mode;
    a.rad = r;
    return a;
}

template <typename T>
void filter_apply(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const Geom &tg,
                  const uint64_t *t_xz_end, const uint16_t *t_y_vec, const FilterIndex &fi, const T *in, T *tree,
                  const ConvPlan *plan, const T *d_stencils, T *out, int mode, const uint16_t *rl_in,
                  FilterBuffers &fb, cudaStream_t s) {
    APRB_PROF(plan ? "convolve" : "fill_tree_mean", s);
    const int L = g.l_max;
    unsigned long long *stale = fb.stale.as<unsigned long long>(1);
    APRB_CUDA(cudaMemsetAsync(stale, 0, sizeof(unsigned long long), s));
    tree_means_all<T>(g, xz_end, y_vec, tg, t_xz_end, t_y_vec, fi, in, tree, s);
    if (!plan) return;
    for (int l = L; l >= g.l_min; --l) {
        if (fi.level_count[l] == 0) continue;
        const int sn = std::min(plan->nstencils - 1, L - l);
        const int side = plan->sides[sn];
        const ConvLevelArgs a = conv_level_args(g, tg, fi, l, side, plan->reflect, mode);
        const T *st = d_stencils + plan->offsets[sn];
        // The streaming kernel builds every plane of its tile that a particle
        // of the level reaches: on a large level with particles in under 40 %
        // of its cells that costs more than the level image in HBM (measured
        // on B200: 1.68 against 1.32 ms for 70 M particles in 268 M cells);
        // on levels of up to 2^26 cells and on dense ones it is the faster.
        // It reads level l's inputs while other CTAs write level l's outputs,
        // so in place the level image is built first.
        const uint64_t cells = ncell_of(a.d);
        const bool stream = (const void *)in != (const void *)out &&
                            (cells <= (uint64_t(1) << 26) || (double)fi.level_count[l] >= 0.4 * (double)cells);
        bool done = false;
        if (stream) {
            if (side == 3)
                done = launch_conv_level_stream<1, T>(a, *plan, sn, xz_end, y_vec, in, t_xz_end, t_y_vec, tree, st,
                                                      out, rl_in, stale, s);
            else
                done = launch_conv_level_stream<2, T>(a, *plan, sn, xz_end, y_vec, in, t_xz_end, t_y_vec, tree, st,
                                                      out, rl_in, stale, s);
        }
        if (done) continue;
        T *D = (T *)fb.dense.get(ncell_of(a.d) * sizeof(T));
        if (side == 3)
            launch_conv_level_dense<1, T>(a, xz_end, y_vec, in, t_xz_end, t_y_vec, tree, st, out, rl_in, stale, D, s);
        else
            launch_conv_level_dense<2, T>(a, xz_end, y_vec, in, t_xz_end, t_y_vec, tree, st, out, rl_in, stale, D, s);
    }
}

template void filter_apply<float>(const Geom &, const uint64_t *, const uint16_t *, const Geom &, const uint64_t *,
                                  const uint16_t *, const FilterIndex &, const float *, float *, const ConvPlan *,
                                  const float *, float *, int, const uint16_t *, FilterBuffers &, cudaStream_t);
template void filter_apply<double>(const Geom &, const uint64_t *, const uint16_t *, const Geom &, const uint64_t *,
                                   const uint16_t *, const FilterIndex &, const double *, double *, const ConvPlan *,
                                   const double *, double *, int, const uint16_t *, FilterBuffers &, cudaStream_t);

void filter_gradient_magnitude(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const Geom &tg,
                               const uint64_t *t_xz_end, const uint16_t *t_y_vec, const FilterIndex &fi,
                               const float *in, float *tree, const float *const stencils[3], const int active[3],
                               int nstencils, float *out, FilterBuffers &fb, cudaStream_t s) {
    APRB_PROF("gradient_magnitude", s);
    const int L = g.l_max;
    unsigned long long *stale = fb.stale.as<unsigned long long>(1);
    APRB_CUDA(cudaMemsetAsync(stale, 0, sizeof(unsigned long long), s));
    tree_means_all<float>(g, xz_end, y_vec, tg, t_xz_end, t_y_vec, fi, in, tree, s);
    for (int l = L; l >= g.l_min; --l) {
        if (fi.level_count[l] == 0) continue;
        const int sn = std::min(nstencils - 1, L - l);
        const ConvLevelArgs a = conv_level_args(g, tg, fi, l, 3, 1, 0);
        GradTaps gt{};
        for (int d = 0; d < 3; ++d) gt.active[d] = active[d];
        for (int k = 0; k < 27; ++k) {
            float w[3];
            bool any = false;
            for (int d = 0; d < 3; ++d) {
                w[d] = active[d] ? stencils[d][27 * sn + k] : 0.0f;
                if (w[d] == 0.0f) w[d] = 0.0f;  // -0 too: the tap is dropped
                any = any || w[d] != 0.0f;
            }
            if (!any) continue;
            const int c = gt.nu++;
            for (int d = 0; d < 3; ++d) gt.w[c][d] = w[d];
            gt.dz[c] = (signed char)(k / 9 - 1);
            gt.dx[c] = (signed char)((k / 3) % 3 - 1);
            gt.dy[c] = (signed char)(k % 3 - 1);
        }
        const uint64_t rows = (uint64_t)a.d.xn * a.d.zn;
        float *D = (float *)fb.dense.get(ncell_of(a.d) * sizeof(float));
        {
            APRB_PROF("densify", s);
            densify_kernel<float><<<blocks_for(rows * 32, 256), 256, 0, s>>>(a, xz_end, y_vec, in, t_xz_end, t_y_vec,
                                                                           tree, D);
            count_launch();
            APRB_CHECK_LAUNCH();
        }
        APRB_PROF("grad_mag_gather", s);
        // four particles per lane for the few taps of central differences,
        // two for the 26 cells of Sobel (fewer registers, more warps)
        if (gt.nu <= 8)
            grad_mag_gather_kernel<4><<<blocks_for(rows * 32, 256), 256, 0, s>>>(a, xz_end, y_vec, D, gt, out, stale);
        else
            grad_mag_gather_kernel<2><<<blocks_for(rows * 32, 256), 256, 0, s>>>(a, xz_end, y_vec, D, gt, out, stale);
        count_launch();
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
