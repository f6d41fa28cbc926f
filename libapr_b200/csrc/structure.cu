// Particle-cell pyramid, Pulling Scheme, linear access structure, particle
// sampling and the APR tree, on the GPU.
//
// The Pulling Scheme's per-level steps are "set-if-status" transitions whose
// sources are never targets within the same step (PullingScheme.hpp:250-393),
// so each step is written here as a gather over the target cells; the
// equivalence optimisation runs levels in ascending order as the reference
// does (LinearAccess.hpp:262-293).  Row counts are scanned on the device and
// rows are filled by warp-ballot compaction, which keeps the reference's
// level -> z -> x -> y particle order.
#include "kernels.cuh"

namespace aprb {

namespace {

struct LevelDims {
    int yn, xn, zn;
};

__device__ __forceinline__ void cell_of(uint64_t g, int yn, int xn, int &y, int &x, int &z) {
    y = (int)(g % (uint64_t)yn);
    uint64_t r = g / (uint64_t)yn;
    x = (int)(r % (uint64_t)xn);
    z = (int)(r / (uint64_t)xn);
}

// PullingScheme::fill below the top level (PullingScheme.hpp:137-168) on the
// max-downsampled level image (LocalParticleCellSet.hpp:74-88).
__global__ void pyramid_fill_kernel(const uint8_t *__restrict__ lev_in, LevelDims di, uint8_t *__restrict__ lev_out,
                                    uint8_t *__restrict__ status, LevelDims d, int level, int is_min) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (uint64_t)d.yn * d.xn * d.zn) return;
    int y, x, z;
    cell_of(g, d.yn, d.xn, y, x, z);
    const int y1 = min(2 * y + 1, di.yn - 1), x1 = min(2 * x + 1, di.xn - 1), z1 = min(2 * z + 1, di.zn - 1);
    uint8_t m = lev_in[idx3(2 * y, 2 * x, 2 * z, di.yn, di.xn)];
    m = max(m, lev_in[idx3(y1, 2 * x, 2 * z, di.yn, di.xn)]);
    m = max(m, lev_in[idx3(2 * y, x1, 2 * z, di.yn, di.xn)]);
    m = max(m, lev_in[idx3(y1, x1, 2 * z, di.yn, di.xn)]);
    m = max(m, lev_in[idx3(2 * y, 2 * x, z1, di.yn, di.xn)]);
    m = max(m, lev_in[idx3(y1, 2 * x, z1, di.yn, di.xn)]);
    m = max(m, lev_in[idx3(2 * y, x1, z1, di.yn, di.xn)]);
    m = max(m, lev_in[idx3(y1, x1, z1, di.yn, di.xn)]);
    lev_out[g] = m;
    if (!status) return;  // level pyramid of a z-tile only
    const bool seed = is_min ? (m <= level) : (m == level);
    status[g] = seed ? kSeed : kEmpty;
}

// The same for four output cells per thread (row grid as the row kernels
// below): each of the four input rows of a 2x2 (x, z) block arrives as one
// 8-byte load (input y extent a multiple of 8, so no y clamp).
__global__ void pyramid_fill4_kernel(const uint8_t *__restrict__ lev_in, LevelDims di, uint8_t *__restrict__ lev_out,
                                     uint8_t *__restrict__ status, LevelDims d, int level, int is_min) {
    const int gidx = blockIdx.x * blockDim.x + threadIdx.x, x = blockIdx.y, z = blockIdx.z;
    if (gidx >= d.yn / 4) return;
    const int y0 = 4 * gidx;
    const int x1 = min(2 * x + 1, di.xn - 1), z1 = min(2 * z + 1, di.zn - 1);
    const int xs[2] = {2 * x, x1}, zs[2] = {2 * z, z1};
    uint32_t mlo = 0, mhi = 0;  // byte-wise maxima of the four rows
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const uint2 v = *reinterpret_cast<const uint2 *>(lev_in + idx3(2 * y0, xs[b], zs[a], di.yn, di.xn));
            mlo = __vmaxu4(mlo, v.x);
            mhi = __vmaxu4(mhi, v.y);
        }
    // output k = max of input bytes 2k and 2k + 1
    uint32_t out = 0, st = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t w = k < 2 ? mlo : mhi;
        const int sh = 16 * (k & 1);
        const uint32_t m = max((w >> sh) & 0xffu, (w >> (sh + 8)) & 0xffu);
        out |= m << (8 * k);
        const bool seed = is_min ? (m <= (uint32_t)level) : (m == (uint32_t)level);
        st |= (uint32_t)(seed ? kSeed : kEmpty) << (8 * k);
    }
    const uint64_t o = ((uint64_t)z * d.xn + x) * d.yn + y0;
    *reinterpret_cast<uint32_t *>(lev_out + o) = out;
    if (status) *reinterpret_cast<uint32_t *>(status + o) = st;
}

// PullingScheme::fill_patch (PullingScheme.hpp:175-247) for a z-tile: the
// tile's level image at one pct level (tile-local planes zlo..zhi-1) marks
// SEED cells of the global level at plane z + offz.  mode 0: level >= k (top),
// 1: level <= k (l_min), 2: level == k.  Planes past the global level are
// skipped (the reference writes beyond the level's array there).
__global__ void fill_patch_kernel(const uint8_t *__restrict__ lev, LevelDims dp, uint8_t *__restrict__ status,
                                  LevelDims d, int zlo, int zhi, int offz, int level, int mode) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (uint64_t)(zhi - zlo) * dp.xn * dp.yn) return;
    int y, x, z;
    cell_of(g, dp.yn, dp.xn, y, x, z);
    z += zlo;
    const int zg = z + offz;
    if (zg < 0 || zg >= d.zn) return;
    const int v = lev[idx3(y, x, z, dp.yn, dp.xn)];
    const bool sd = mode == 0 ? v >= level : (mode == 1 ? v <= level : v == level);
    if (sd) status[idx3(y, x, zg, d.yn, d.xn)] = kSeed;
}

// set_filler (:291-343): children of ASCENDANTNEIGHBOUR / PROPOGATE cells
__global__ void set_filler_kernel(const uint8_t *__restrict__ parent, LevelDims dp, uint8_t *__restrict__ child,
                                  LevelDims dc) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (uint64_t)dc.yn * dc.xn * dc.zn) return;
    if (child[g] != kEmpty) return;
    int y, x, z;
    cell_of(g, dc.yn, dc.xn, y, x, z);
    const uint8_t s = parent[idx3(y / 2, x / 2, z / 2, dp.yn, dp.xn)];
    if (s == kAscendantNeighbour || s == kPropagate) child[g] = kFiller;
}

// 3x3x3 neighbourhood marking as a tiled OR-dilation, for the two
// neighbour steps of the pulling scheme:
//   MODE 0, set_ascendant_neighbours (:250-289): source ASCENDANT; an EMPTY
//           cell next to one becomes ASCENDANTNEIGHBOUR, a SEED cell PROPOGATE;
//   MODE 1, fill_neighbours (:345-381): source SEED or PROPOGATE; an EMPTY cell
//           next to one becomes BOUNDARY.
// A CTA owns 128 (y) x 8 (x) x 8 (z) cells.  Each warp turns one row of the
// tile plus its one-cell halo into four 32-bit words of the y-dilated source
// mask (warp ballots, neighbours by shuffles), the words are ORed over the
// 3 x 3 (x, z) neighbourhood from shared memory, and the targets are written.
// Writes never create a source value, so concurrent CTAs reading their halo
// see the same sources in any order.
constexpr int kDY = 128, kDX = 8, kDZ = 8, kDRows = (kDX + 2) * (kDZ + 2), kDWords = kDY / 32;

template <int MODE>
__device__ __forceinline__ bool dil_source(uint8_t s) {
    return MODE == 0 ? s == kAscendant : (s == kSeed || s == kPropagate);
}

template <int MODE>
__global__ void __launch_bounds__(256) dilate_kernel(uint8_t *__restrict__ st, LevelDims d) {
    __shared__ uint32_t W[kDRows][kDWords];
    const int y0 = blockIdx.x * kDY, x0 = blockIdx.y * kDX, z0 = blockIdx.z * kDZ;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int r = w; r < kDRows; r += 8) {
        const int x = x0 - 1 + r % (kDX + 2), z = z0 - 1 + r / (kDX + 2);
        const bool row_in = x >= 0 && x < d.xn && z >= 0 && z < d.zn;
        const uint8_t *R = st + ((uint64_t)(row_in ? z : 0) * d.xn + (row_in ? x : 0)) * (uint64_t)d.yn;
        for (int k = 0; k < kDWords; ++k) {
            const int y = y0 + 32 * k + lane;
            const bool p = row_in && y < d.yn && dil_source<MODE>(R[y]);
            bool pl = __shfl_up_sync(0xffffffffu, p, 1), pr = __shfl_down_sync(0xffffffffu, p, 1);
            if (lane == 0) pl = row_in && y >= 1 && y - 1 < d.yn && dil_source<MODE>(R[y - 1]);
            if (lane == 31) pr = row_in && y + 1 < d.yn && dil_source<MODE>(R[y + 1]);
            const uint32_t word = __ballot_sync(0xffffffffu, p || pl || pr);
            if (lane == 0) W[r][k] = word;
        }
    }
    __syncthreads();
    for (int task = w; task < kDX * kDZ * kDWords; task += 8) {
        const int k = task % kDWords, xx = (task / kDWords) % kDX, zz = task / (kDWords * kDX);
        const int x = x0 + xx, z = z0 + zz, y = y0 + 32 * k + lane;
        if (x >= d.xn || z >= d.zn) continue;
        uint32_t m = 0;
#pragma unroll
        for (int dz = 0; dz < 3; ++dz)
#pragma unroll
            for (int dx = 0; dx < 3; ++dx) m |= W[(zz + dz) * (kDX + 2) + xx + dx][k];
        if (y >= d.yn || !((m >> lane) & 1u)) continue;
        uint8_t *c = st + ((uint64_t)z * d.xn + x) * (uint64_t)d.yn + y;
        const uint8_t s = *c;
        if (MODE == 0) {
            if (s == kEmpty) *c = kAscendantNeighbour;
            else if (s == kSeed) *c = kPropagate;
        } else {
            if (s == kEmpty) *c = kBoundary;
        }
    }
}

// Byte-parallel helpers on 32-bit words of four cells (byte j = cell j).
// bytes_eq: 0x80 in each byte equal to the corresponding byte of c4, 0 in the
// others; exact, since (t & 0x7F) + 0x7F never carries out of its byte.
__device__ __forceinline__ uint32_t bytes_eq(uint32_t w, uint32_t c4) {
    const uint32_t t = w ^ c4;
    return ~((((t & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | t) | 0x7F7F7F7Fu);
}
// The high bits of the four bytes of h (h holds no other bits) as bits 0..3:
// the product's partial sums land on distinct bits, so nothing carries.
__device__ __forceinline__ unsigned high_bits4(uint32_t h) { return (h * 0x00204081u) >> 28; }
// Bits 0..3 of n (n < 16) as 0x80 / 0x00 in bytes 0..3.
__device__ __forceinline__ uint32_t nibble_high_bytes(unsigned n) { return ((n * 0x00204081u) & 0x01010101u) << 7; }
// 0x80 in each byte b of w with 1 <= b <= m (0 <= m < 128), 0 in the others:
// (b | 0x80) - (m + 1) never borrows across bytes, and its high bit is clear
// exactly when b < m + 1 (for b < 128).
__device__ __forceinline__ uint32_t bytes_in_1_to(uint32_t w, int m) {
    const uint32_t lt = ~(((w | 0x80808080u) - (uint32_t)(m + 1) * 0x01010101u) | w) & 0x80808080u;
    return lt & ~bytes_eq(w, 0u);
}

template <int MODE>
__device__ __forceinline__ uint32_t dil_source4(uint32_t w) {
    return MODE == 0 ? bytes_eq(w, kAscendant * 0x01010101u)
                     : bytes_eq(w, kSeed * 0x01010101u) | bytes_eq(w, kPropagate * 0x01010101u);
}

template <int MODE>
__device__ __forceinline__ unsigned dil_bits16(const uint4 v) {
    return high_bits4(dil_source4<MODE>(v.x)) | high_bits4(dil_source4<MODE>(v.y)) << 4 |
           high_bits4(dil_source4<MODE>(v.z)) << 8 | high_bits4(dil_source4<MODE>(v.w)) << 12;
}

// The targets among the four cells of w whose bits in n (0..3) are set:
// MODE 0 turns EMPTY into ASCENDANTNEIGHBOUR and SEED into PROPOGATE, MODE 1
// EMPTY into BOUNDARY.  Each selected byte gains the difference of the two
// status values, which never carries into the next byte.
static_assert(kEmpty == 0 && kPropagate > kSeed, "EMPTY and SEED targets are formed by adding to the byte");
template <int MODE>
__device__ __forceinline__ uint32_t dil_target4(uint32_t w, unsigned n) {
    const uint32_t sel = nibble_high_bytes(n);
    const uint32_t e = bytes_eq(w, 0u) & sel;
    if (MODE == 0) {
        const uint32_t sd = bytes_eq(w, kSeed * 0x01010101u) & sel;
        return w + (e >> 7) * kAscendantNeighbour + (sd >> 7) * (uint32_t)(kPropagate - kSeed);
    }
    return w + (e >> 7) * kBoundary;
}

// The same dilation for rows of a multiple of 16 cells and 16-byte aligned
// rows: a lane moves 16 consecutive cells as one 16-byte word, a warp reads
// 512 y of a row in one load, and the shared mask holds per row and lane the
// 16 bits of the lane's cells.  Sources and targets are found four cells at
// a time with byte-parallel arithmetic on 32-bit words, not cell by cell.
constexpr int kD16Y = 512;
template <int MODE>
__global__ void __launch_bounds__(256) dilate16_kernel(uint8_t *__restrict__ st, LevelDims d) {
    __shared__ uint16_t W[kDRows][32];
    const int y0 = blockIdx.x * kD16Y, x0 = blockIdx.y * kDX, z0 = blockIdx.z * kDZ;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y = y0 + 16 * lane;  // first of the lane's cells; yn % 16 == 0, so all 16 are in or out
    for (int r = w; r < kDRows; r += 8) {
        const int x = x0 - 1 + r % (kDX + 2), z = z0 - 1 + r / (kDX + 2);
        const bool row_in = x >= 0 && x < d.xn && z >= 0 && z < d.zn;
        const uint8_t *R = st + ((uint64_t)(row_in ? z : 0) * d.xn + (row_in ? x : 0)) * (uint64_t)d.yn;
        const bool in = row_in && y < d.yn;
        const uint4 v = in ? *reinterpret_cast<const uint4 *>(R + y) : make_uint4(0u, 0u, 0u, 0u);
        const unsigned p = dil_bits16<MODE>(v);
        unsigned pl = (__shfl_up_sync(0xffffffffu, p, 1) >> 15) & 1u;
        unsigned pr = __shfl_down_sync(0xffffffffu, p, 1) & 1u;
        if (lane == 0) pl = row_in && y >= 1 && y - 1 < d.yn && dil_source<MODE>(R[y - 1]);
        if (lane == 31) pr = row_in && y + 16 < d.yn && dil_source<MODE>(R[y + 16]);
        W[r][lane] = (uint16_t)((p | (p << 1) | (p >> 1) | pl | (pr << 15)) & 0xFFFFu);
    }
    __syncthreads();
    for (int task = w; task < kDX * kDZ; task += 8) {
        const int xx = task % kDX, zz = task / kDX;
        const int x = x0 + xx, z = z0 + zz;
        if (x >= d.xn || z >= d.zn || y >= d.yn) continue;
        unsigned m = 0;
#pragma unroll
        for (int dz = 0; dz < 3; ++dz)
#pragma unroll
            for (int dx = 0; dx < 3; ++dx) m |= W[(zz + dz) * (kDX + 2) + xx + dx][lane];
        if (!m) continue;
        uint4 *c = reinterpret_cast<uint4 *>(st + ((uint64_t)z * d.xn + x) * (uint64_t)d.yn + y);
        const uint4 v = *c;
        const uint4 nv = make_uint4(dil_target4<MODE>(v.x, m & 15u), dil_target4<MODE>(v.y, (m >> 4) & 15u),
                                    dil_target4<MODE>(v.z, (m >> 8) & 15u), dil_target4<MODE>(v.w, m >> 12));
        if (nv.x != v.x || nv.y != v.y || nv.z != v.z || nv.w != v.w) *c = nv;
    }
}

// The same dilation for rows of a multiple of 4 cells: a lane moves 4
// consecutive cells of a row as one 32-bit word, so a warp reads the block's
// 128 y of a row in one load, and the shared mask holds per row and lane the
// 4 bits of the lane's cells.  Phase 2 writes the words whose cells change.
template <int MODE>
__global__ void __launch_bounds__(256) dilate4_kernel(uint8_t *__restrict__ st, LevelDims d) {
    __shared__ uint8_t W[kDRows][32];
    const int y0 = blockIdx.x * kDY, x0 = blockIdx.y * kDX, z0 = blockIdx.z * kDZ;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y = y0 + 4 * lane;  // first of the lane's cells; yn % 4 == 0, so all 4 are in or out
    for (int r = w; r < kDRows; r += 8) {
        const int x = x0 - 1 + r % (kDX + 2), z = z0 - 1 + r / (kDX + 2);
        const bool row_in = x >= 0 && x < d.xn && z >= 0 && z < d.zn;
        const uint8_t *R = st + ((uint64_t)(row_in ? z : 0) * d.xn + (row_in ? x : 0)) * (uint64_t)d.yn;
        const bool in = row_in && y < d.yn;
        const uint32_t v = in ? *reinterpret_cast<const uint32_t *>(R + y) : 0u;
        unsigned p = 0;
#pragma unroll
        for (int e = 0; e < 4; ++e)
            if (in && dil_source<MODE>((uint8_t)(v >> (8 * e)))) p |= 1u << e;
        unsigned pl = (__shfl_up_sync(0xffffffffu, p, 1) >> 3) & 1u;
        unsigned pr = __shfl_down_sync(0xffffffffu, p, 1) & 1u;
        if (lane == 0) pl = row_in && y >= 1 && y - 1 < d.yn && dil_source<MODE>(R[y - 1]);
        if (lane == 31) pr = row_in && y + 4 < d.yn && dil_source<MODE>(R[y + 4]);
        W[r][lane] = (uint8_t)((p | (p << 1) | (p >> 1) | pl | (pr << 3)) & 0xFu);
    }
    __syncthreads();
    for (int task = w; task < kDX * kDZ; task += 8) {
        const int xx = task % kDX, zz = task / kDX;
        const int x = x0 + xx, z = z0 + zz;
        if (x >= d.xn || z >= d.zn || y >= d.yn) continue;
        unsigned m = 0;
#pragma unroll
        for (int dz = 0; dz < 3; ++dz)
#pragma unroll
            for (int dx = 0; dx < 3; ++dx) m |= W[(zz + dz) * (kDX + 2) + xx + dx][lane];
        if (!m) continue;
        uint32_t *c = reinterpret_cast<uint32_t *>(st + ((uint64_t)z * d.xn + x) * (uint64_t)d.yn + y);
        const uint32_t v = *c;
        uint32_t nv = v;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            if (!((m >> e) & 1u)) continue;
            const uint8_t s = (uint8_t)(v >> (8 * e));
            uint8_t t = s;
            if (MODE == 0) {
                if (s == kEmpty) t = kAscendantNeighbour;
                else if (s == kSeed) t = kPropagate;
            } else {
                if (s == kEmpty) t = kBoundary;
            }
            nv = (nv & ~(0xFFu << (8 * e))) | ((uint32_t)t << (8 * e));
        }
        if (nv != v) *c = nv;
    }
}

// fill_neighbours -> fill_parent (:372-393), as a gather over the parents
__global__ void fill_parent_kernel(const uint8_t *__restrict__ child, LevelDims dc, uint8_t *__restrict__ parent,
                                   LevelDims dp) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (uint64_t)dp.yn * dp.xn * dp.zn) return;
    if (parent[g] == kSeed) return;
    int y, x, z;
    cell_of(g, dp.yn, dp.xn, y, x, z);
    for (int cz = 2 * z; cz < min(2 * z + 2, dc.zn); ++cz)
        for (int cx = 2 * x; cx < min(2 * x + 2, dc.xn); ++cx)
            for (int cy = 2 * y; cy < min(2 * y + 2, dc.yn); ++cy) {
                const uint8_t q = child[idx3(cy, cx, cz, dc.yn, dc.xn)];
                if (q == kSeed || q == kPropagate || q == kAscendant) {
                    parent[g] = kAscendant;
                    return;
                }
            }
}

// Vector forms of set_filler, fill_parent and the equivalence optimisation for
// levels whose rows are multiples of 8 cells (child) / 4 cells (parent): a
// thread moves 8 child cells (uint2) or 4 parent cells (uint32) at once, with
// the same per-cell rules as the scalar kernels.

// Grid of the row kernels below (set_filler8, fill_parent4): (groups of a row
// / blockDim.x, x, z), so a thread finds its row without integer division.
__device__ __forceinline__ bool row_group(int groups, int xn, int &gidx, int &x, int &z, uint64_t &row) {
    gidx = blockIdx.x * blockDim.x + threadIdx.x;
    x = blockIdx.y;
    z = blockIdx.z;
    row = (uint64_t)z * xn + x;
    return gidx < groups;
}

__global__ void set_filler8_kernel(const uint8_t *__restrict__ parent, LevelDims dp, uint8_t *__restrict__ child,
                                   LevelDims dc) {
    const int groups = dc.yn / 8;
    int gidx, x, z;
    uint64_t row;
    if (!row_group(groups, dc.xn, gidx, x, z, row)) return;
    const int y0 = gidx * 8;
    uint2 *cp = reinterpret_cast<uint2 *>(child + row * (uint64_t)dc.yn + y0);
    const uint2 cv = *cp;
    const uint32_t pv = *reinterpret_cast<const uint32_t *>(parent + idx3(y0 / 2, x / 2, z / 2, dp.yn, dp.xn));
    // parents ASCENDANTNEIGHBOUR or PROPOGATE, each byte spread over its two child cells
    const uint32_t pt = bytes_eq(pv, kAscendantNeighbour * 0x01010101u) | bytes_eq(pv, kPropagate * 0x01010101u);
    const uint32_t lo = bytes_eq(cv.x, 0u) & __byte_perm(pt, 0u, 0x1100u);
    const uint32_t hi = bytes_eq(cv.y, 0u) & __byte_perm(pt, 0u, 0x3322u);
    if (lo | hi) *cp = make_uint2(cv.x + (lo >> 7) * kFiller, cv.y + (hi >> 7) * kFiller);  // EMPTY -> FILLER
}

// Grid (groups x rows of a plane / 256, z): one 32-bit division per thread
// finds the row; the many threads whose parents hold no seed end at once, so
// blocks of 256 keep the block count low.
__global__ void eqopt8_kernel(const uint8_t *__restrict__ parent, LevelDims dp, uint8_t *__restrict__ st,
                              LevelDims d, int min_type) {
    const unsigned groups = (unsigned)d.yn / 8u;
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= groups * (unsigned)d.xn) return;
    const int x = (int)(t / groups), z = blockIdx.y;
    const int y0 = (int)(t - (unsigned)x * groups) * 8;
    const uint32_t pv = *reinterpret_cast<const uint32_t *>(parent + idx3(y0 / 2, x / 2, z / 2, dp.yn, dp.xn));
    const uint32_t seeds = bytes_in_1_to(pv, min_type);
    if (!seeds) return;
    uint2 *cp = reinterpret_cast<uint2 *>(st + idx3(y0, x, z, d.yn, d.xn));
    const uint2 cv = *cp;
    const uint32_t lo = (__byte_perm(seeds, 0u, 0x1100u) >> 7) * 0xFFu, hi = (__byte_perm(seeds, 0u, 0x3322u) >> 7) * 0xFFu;
    const uint32_t up = kUpsamplingSeed * 0x01010101u;
    *cp = make_uint2((cv.x & ~lo) | (up & lo), (cv.y & ~hi) | (up & hi));
}

__global__ void fill_parent4_kernel(const uint8_t *__restrict__ child, LevelDims dc, uint8_t *__restrict__ parent,
                                    LevelDims dp) {
    const int groups = dp.yn / 4;
    int gidx, x, z;
    uint64_t row;
    if (!row_group(groups, dp.xn, gidx, x, z, row)) return;
    const int y0 = gidx * 4;
    uint32_t *pp = reinterpret_cast<uint32_t *>(parent + row * (uint64_t)dp.yn + y0);
    const uint32_t pv = *pp;
    uint2 cv[4];  // the (up to) four child rows under the parent row, all loaded before any is used
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int cz = 2 * z + (k >> 1), cx = 2 * x + (k & 1);
        cv[k] = cz < dc.zn && cx < dc.xn ? *reinterpret_cast<const uint2 *>(child + idx3(2 * y0, cx, cz, dc.yn, dc.xn))
                                         : make_uint2(0u, 0u);
    }
    uint32_t lo = 0, hi = 0;  // 0x80 in the child bytes 0..3 / 4..7 that are SEED, PROPOGATE or ASCENDANT in a row
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        lo |= bytes_eq(cv[k].x, kSeed * 0x01010101u) | bytes_eq(cv[k].x, kPropagate * 0x01010101u) |
              bytes_eq(cv[k].x, kAscendant * 0x01010101u);
        hi |= bytes_eq(cv[k].y, kSeed * 0x01010101u) | bytes_eq(cv[k].y, kPropagate * 0x01010101u) |
              bytes_eq(cv[k].y, kAscendant * 0x01010101u);
    }
    lo |= lo >> 8;  // bytes 0 and 2: either child of parents 0 and 1
    hi |= hi >> 8;
    const unsigned hit = ((lo >> 7) & 1u) | ((lo >> 22) & 2u) | ((hi >> 5) & 4u) | ((hi >> 20) & 8u);
    // parents with such a child, unless SEED, become ASCENDANT
    const uint32_t m = ((nibble_high_bytes(hit) & ~bytes_eq(pv, kSeed * 0x01010101u)) >> 7) * 0xFFu;
    const uint32_t nv = (pv & ~m) | (kAscendant * 0x01010101u & m);
    if (nv != pv) *pp = nv;
}

// equivalence optimisation (LinearAccess.hpp:262-293) for one level
__global__ void eqopt_kernel(const uint8_t *__restrict__ parent, LevelDims dp, uint8_t *__restrict__ st, LevelDims d,
                             int min_type) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (uint64_t)d.yn * d.xn * d.zn) return;
    int y, x, z;
    cell_of(g, d.yn, d.xn, y, x, z);
    const uint8_t s = parent[idx3(y / 2, x / 2, z / 2, dp.yn, dp.xn)];
    if (s > 0 && s <= min_type) st[g] = kUpsamplingSeed;
}

__device__ __forceinline__ bool is_particle(uint8_t s, int min_type) { return s > min_type && s <= kUpsamplingSeed; }
__device__ __forceinline__ bool is_seed(uint8_t s, int min_type) { return s > 0 && s <= min_type; }

// row counts (LinearAccess.hpp:297-407): one warp per (z, x) row
__global__ void row_count_kernel(const uint8_t *__restrict__ st, LevelDims d, uint64_t *__restrict__ xz_end,
                                 uint64_t row_base, int min_type) {
    const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= (uint64_t)d.xn * d.zn) return;
    const uint8_t *R = st + row * (uint64_t)d.yn;
    unsigned c = 0;
    for (int y = lane; y < d.yn; y += 32) c += is_particle(R[y], min_type);
    c = __reduce_add_sync(0xffffffffu, c);
    if (lane == 0) xz_end[row_base + row] = c;
}

// top pct level: its own particles plus the l_max particles of its seeds,
// copied to every l_max row the cell covers (:339-407)
__global__ void row_count_top_kernel(const uint8_t *__restrict__ st, LevelDims d, uint64_t *__restrict__ xz_end,
                                     uint64_t row_base, uint64_t row_base_m, int ylm, int xlm, int zlm,
                                     int min_type, int vec16) {
    const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= (uint64_t)d.xn * d.zn) return;
    const uint8_t *R = st + row * (uint64_t)d.yn;
    unsigned c = 0, cl = 0;
    if (vec16) {
        // 16 cells per lane and step, counted four at a time with byte-wise
        // compares (particle: min_type < s <= UPSAMPLING_SEED; seed:
        // 0 < s <= min_type, two finest-level cells each but where the pair's
        // second cell lies beyond the finest level)
        const uint32_t mt4 = 0x01010101u * (uint32_t)min_type, up4 = 0x01010101u * (uint32_t)kUpsamplingSeed;
        unsigned seeds = 0;
        for (int y = 16 * lane; y < d.yn; y += 512) {
            const uint4 v = *reinterpret_cast<const uint4 *>(R + y);
            const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                c += __popc(__vcmpgtu4(w[q], mt4) & __vcmpleu4(w[q], up4)) >> 3;
                seeds += __popc(__vcmpgtu4(w[q], 0u) & __vcmpleu4(w[q], mt4)) >> 3;
            }
        }
        cl = 2 * seeds;
        if (lane == 0 && 2 * (d.yn - 1) >= ylm - 1 && is_seed(R[d.yn - 1], min_type)) cl -= 1;
    } else {
        for (int y = lane; y < d.yn; y += 32) {
            const uint8_t s = R[y];
            if (is_particle(s, min_type))
                c++;
            else if (is_seed(s, min_type))
                cl += 1 + (2 * y < ylm - 1);
        }
    }
    c = __reduce_add_sync(0xffffffffu, c);
    cl = __reduce_add_sync(0xffffffffu, cl);
    if (lane < 4) {
        const int x = (int)(row % (uint64_t)d.xn), z = (int)(row / (uint64_t)d.xn);
        const int zz = 2 * z + (lane >> 1), xx = 2 * x + (lane & 1);
        if (zz < zlm && xx < xlm) xz_end[row_base_m + (uint64_t)zz * xlm + xx] = cl;
        if (lane == 0) xz_end[row_base + row] = c;
    }
}

// y fill by ordered warp compaction (:414-497)
__global__ void row_fill_kernel(const uint8_t *__restrict__ st, LevelDims d, const uint64_t *__restrict__ xz_end,
                                uint64_t row_base, uint16_t *__restrict__ y_vec, int min_type) {
    const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= (uint64_t)d.xn * d.zn) return;
    const uint8_t *R = st + row * (uint64_t)d.yn;
    uint64_t o = xz_end[row_base + row - 1];
    const unsigned lt = (1u << lane) - 1u;
    for (int y0 = 0; y0 < d.yn; y0 += 32) {
        const int y = y0 + lane;
        const bool f = y < d.yn && is_particle(R[y], min_type);
        const unsigned m = __ballot_sync(0xffffffffu, f);
        if (f) y_vec[o + __popc(m & lt)] = (uint16_t)y;
        o += __popc(m);
    }
}

__global__ void __launch_bounds__(256) row_fill_top_kernel(const uint8_t *__restrict__ st, LevelDims d,
                                                             const uint64_t *__restrict__ xz_end, uint64_t row_base,
                                                             uint64_t row_base_m, int ylm, int xlm, int zlm,
                                                             uint16_t *__restrict__ y_vec, int min_type, int vec4) {
    // 128 cells of the row per step, four per lane: one scan of the packed
    // per-lane counts (level l_max - 1 particles << 16 | level l_max outputs)
    // places both; the step's l_max outputs are staged in shared memory and
    // copied to the four child rows with coalesced stores
    __shared__ uint16_t stage[8][256];
    const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    uint16_t *S = stage[threadIdx.x >> 5];
    if (row >= (uint64_t)d.xn * d.zn) return;
    const int x = (int)(row % (uint64_t)d.xn), z = (int)(row / (uint64_t)d.xn);
    const uint8_t *R = st + row * (uint64_t)d.yn;
    uint64_t o = xz_end[row_base + row - 1];
    uint16_t *Q[4];
    int nq = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int zz = 2 * z + (q >> 1), xx = 2 * x + (q & 1);
        Q[q] = nullptr;
        if (zz < zlm && xx < xlm) {
            Q[q] = y_vec + xz_end[row_base_m + (uint64_t)zz * xlm + xx - 1];
            nq = q + 1;
        }
    }
    for (int y0 = 0; y0 < d.yn; y0 += 128) {
        const int yb = y0 + 4 * lane;
        uint32_t w = 0;  // the lane's four cells, zero (EMPTY) beyond the row
        if (vec4 && yb + 4 <= d.yn) {
            w = *reinterpret_cast<const uint32_t *>(R + yb);
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (yb + k < d.yn) w |= (uint32_t)R[yb + k] << (8 * k);
        }
        // 0x80 in the bytes of seeds (1..min_type) and of particles (min_type < s <= UPSAMPLING_SEED)
        const uint32_t seedm = bytes_in_1_to(w, min_type);
        const uint32_t partm = bytes_in_1_to(w, kUpsamplingSeed) & ~seedm;
        // a seed cell y has the level l_max children 2y and 2y + 1, the second
        // only where 2y + 1 < ylm, i.e. below y = ylm / 2
        const int kcut = (ylm >> 1) - yb;
        const uint32_t one_child = kcut <= 0 ? 0x80808080u : (kcut >= 4 ? 0u : 0x80808080u << (8 * kcut));
        const int pc = __popc(partm), cc = 2 * __popc(seedm) - __popc(seedm & one_child);
        const int mine = (pc << 16) | cc;
        int incl = mine;
#pragma unroll
        for (int k = 1; k < 32; k <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, k);
            if (lane >= k) incl += t;
        }
        const int tot = __shfl_sync(0xffffffffu, incl, 31);
        const int excl = incl - mine;
        int pp = excl >> 16, cp = excl & 0xffff;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int y = yb + k;
            if ((partm >> (8 * k + 7)) & 1u) y_vec[o + pp++] = (uint16_t)y;
            if ((seedm >> (8 * k + 7)) & 1u) {
                S[cp++] = (uint16_t)(2 * y);
                if (2 * y + 1 < ylm) S[cp++] = (uint16_t)(2 * y + 1);
            }
        }
        o += (uint64_t)(tot >> 16);
        const int nc = tot & 0xffff;
        __syncwarp();
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (q >= nq || Q[q] == nullptr) continue;
            for (int j = lane; j < nc; j += 32) Q[q][j] = S[j];
            Q[q] += nc;
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// APRReconstruction::reconstruct_constant / reconstruct_level
// (APRReconstruction.hpp:80-123, 132-170): every full-resolution pixel takes
// the value, or the level, of the particle whose cell covers it.  A warp per
// pixel row (z, x) walks the covering row (z >> d, x >> d) of every level
// l = l_max - d; a particle of level l fills its 2^d samples of the row,
// clipped at the image edge.  The particle cells partition the image, so
// every pixel is written once.
// ---------------------------------------------------------------------------
template <typename V, bool LEVEL>
__global__ void reconstruct_kernel(Geom g, const uint64_t *__restrict__ xz_end, const uint16_t *__restrict__ y_vec,
                                   const V *__restrict__ parts, V *__restrict__ img) {
    const int L = g.l_max;
    const int yn = g.y_num[L], xn = g.x_num[L];
    const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= (uint64_t)xn * g.z_num[L]) return;
    const int x = (int)(row % (uint64_t)xn), z = (int)(row / (uint64_t)xn);
    V *R = img + row * (uint64_t)yn;
    for (int l = L; l >= g.l_min; --l) {
        const int d = L - l;
        const uint64_t r = (uint64_t)(z >> d) * g.x_num[l] + (x >> d);
        const uint64_t b = xz_end[g.level_xz[l] + r - 1], e = xz_end[g.level_xz[l] + r];
        if (d == 0) {
            for (uint64_t i = b + lane; i < e; i += 32) R[y_vec[i]] = LEVEL ? (V)l : parts[i];
        } else {
            for (uint64_t i = b + lane; i < e; i += 32) {
                const int y0 = (int)y_vec[i] << d, y1 = min(y0 + (1 << d), yn);
                const V v = LEVEL ? (V)l : parts[i];
                for (int y = y0; y < y1; ++y) R[y] = v;
            }
        }
    }
}

// l_max <= 2: every pixel is a particle (LinearAccess.hpp:226-259)
__global__ void full_res_counts_kernel(uint64_t *xz_end, uint64_t base, int yn, uint64_t rows) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < rows) xz_end[base + r] = (r + 1) * (uint64_t)yn;
}
__global__ void full_res_fill_kernel(uint16_t *y_vec, int yn, uint64_t n) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y_vec[i] = (uint16_t)(i % (uint64_t)yn);
}

// ---------------------------------------------------------------------------
// inclusive scan of uint64 (three phases: block sums, scan of sums, apply)
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 256, kScanItems = 8, kScanBlock = kScanThreads * kScanItems;

__device__ __forceinline__ uint64_t block_exclusive_scan(uint64_t v, uint64_t *sh, uint64_t &total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint64_t x = v;
    for (int k = 1; k < 32; k <<= 1) {
        uint64_t t = __shfl_up_sync(0xffffffffu, x, k);
        if (lane >= k) x += t;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        uint64_t s = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0;
        for (int k = 1; k < 32; k <<= 1) {
            uint64_t t = __shfl_up_sync(0xffffffffu, s, k);
            if (lane >= k) s += t;
        }
        if (lane < (int)(blockDim.x >> 5)) sh[lane] = s;
    }
    __syncthreads();
    const uint64_t before = w > 0 ? sh[w - 1] : 0;
    total = sh[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before + x - v;
}

__global__ void scan_sums_kernel(const uint64_t *__restrict__ d, uint64_t n, uint64_t *__restrict__ sums) {
    __shared__ uint64_t sh[32];
    const uint64_t base = (uint64_t)blockIdx.x * kScanBlock + (uint64_t)threadIdx.x * kScanItems;
    uint64_t s = 0;
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < n) s += d[base + k];
    uint64_t total;
    block_exclusive_scan(s, sh, total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void scan_sums_serial_kernel(uint64_t *sums, uint64_t nb) {
    __shared__ uint64_t sh[32];
    uint64_t carry = 0;
    for (uint64_t b0 = 0; b0 < nb; b0 += blockDim.x) {
        const uint64_t i = b0 + threadIdx.x;
        const uint64_t v = i < nb ? sums[i] : 0;
        uint64_t total;
        const uint64_t ex = block_exclusive_scan(v, sh, total);
        if (i < nb) sums[i] = carry + ex;
        carry += total;
    }
}

__global__ void scan_apply_kernel(uint64_t *__restrict__ d, uint64_t n, const uint64_t *__restrict__ sums) {
    __shared__ uint64_t sh[32];
    const uint64_t base = (uint64_t)blockIdx.x * kScanBlock + (uint64_t)threadIdx.x * kScanItems;
    uint64_t v[kScanItems];
    uint64_t s = 0;
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n ? d[base + k] : 0;
        s += v[k];
    }
    uint64_t total;
    uint64_t run = block_exclusive_scan(s, sh, total) + sums[blockIdx.x];
    for (int k = 0; k < kScanItems; ++k) {
        run += v[k];
        if (base + k < n) d[base + k] = run;
    }
}

// ---------------------------------------------------------------------------
// sampling
// ---------------------------------------------------------------------------
// downsample(sum, x/8.0f) into uint16 (PixelData.hpp:1037-1058): the 8-term
// float sum is exact, so the stored value is floor(sum / 8).
__global__ void pyr_mean_u16_kernel(const uint16_t *__restrict__ in, LevelDims di, uint16_t *__restrict__ out,
                                    LevelDims d) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (uint64_t)d.yn * d.xn * d.zn) return;
    int y, x, z;
    cell_of(g, d.yn, d.xn, y, x, z);
    const int y1 = min(2 * y + 1, di.yn - 1), x1 = min(2 * x + 1, di.xn - 1), z1 = min(2 * z + 1, di.zn - 1);
    const int y0 = 2 * y, x0 = 2 * x, z0 = 2 * z;
    unsigned s = in[idx3(y0, x0, z0, di.yn, di.xn)];
    s += in[idx3(y1, x0, z0, di.yn, di.xn)];
    s += in[idx3(y0, x1, z0, di.yn, di.xn)];
    s += in[idx3(y1, x1, z0, di.yn, di.xn)];
    s += in[idx3(y0, x0, z1, di.yn, di.xn)];
    s += in[idx3(y1, x0, z1, di.yn, di.xn)];
    s += in[idx3(y0, x1, z1, di.yn, di.xn)];
    s += in[idx3(y1, x1, z1, di.yn, di.xn)];
    out[g] = (uint16_t)(s >> 3);
}

// sample_parts_from_img_downsampled_patch (ParticleData.hpp:330-372): the
// particles of global rows (zlo + offz .. zhi - 1 + offz, x) of one level take
// the tile's pyramid value at tile-local plane z.
// The same mean for input rows that are multiples of 4 samples: a thread
// reads 4 x uint2 (4 samples each) and writes two outputs as one uint32.
__global__ void pyr_mean_u16x2_kernel(const uint16_t *__restrict__ in, LevelDims di, uint16_t *__restrict__ out,
                                      LevelDims d) {
    // grid (pairs of a row / blockDim.x, x, z): no integer division
    const int gidx = blockIdx.x * blockDim.x + threadIdx.x, x = blockIdx.y, z = blockIdx.z;
    if (gidx >= d.yn / 2) return;
    const uint64_t row = (uint64_t)z * d.xn + x;
    const int y = 2 * gidx;
    const int x1 = min(2 * x + 1, di.xn - 1), z1 = min(2 * z + 1, di.zn - 1);
    const int xs[2] = {2 * x, x1}, zs[2] = {2 * z, z1};
    unsigned s0 = 0, s1 = 0;
    // same summation order per output as pyr_mean_u16_kernel: (y0,x0,z0) (y1,x0,z0)
    // (y0,x1,z0) (y1,x1,z0) then z1; integer sums, so the order is immaterial
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const uint2 v = *reinterpret_cast<const uint2 *>(in + idx3(2 * y, xs[b], zs[a], di.yn, di.xn));
            s0 += (v.x & 0xffffu) + (v.x >> 16);
            s1 += (v.y & 0xffffu) + (v.y >> 16);
        }
    *reinterpret_cast<uint32_t *>(out + row * (uint64_t)d.yn + y) = (s0 >> 3) | ((s1 >> 3) << 16);
}

__global__ void gather_patch_kernel(const uint16_t *__restrict__ im, LevelDims dp, int zlo, int zhi, int offz,
                                    int gzn, const uint64_t *__restrict__ xz_end, uint64_t row_base,
                                    const uint16_t *__restrict__ y_vec, uint16_t *__restrict__ parts) {
    const uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= (uint64_t)(zhi - zlo) * dp.xn) return;
    const int x = (int)(r % (uint64_t)dp.xn), z = zlo + (int)(r / (uint64_t)dp.xn);
    const int zg = z + offz;
    if (zg < 0 || zg >= gzn) return;
    const uint64_t row = (uint64_t)zg * dp.xn + x;
    const uint64_t b = xz_end[row_base + row - 1], e = xz_end[row_base + row];
    const uint16_t *R = im + ((uint64_t)z * dp.xn + x) * (uint64_t)dp.yn;
    for (uint64_t i = b + lane; i < e; i += 32) parts[i] = R[y_vec[i]];
}

__global__ void gather_kernel(const uint16_t *__restrict__ im, LevelDims d, const uint64_t *__restrict__ xz_end,
                              uint64_t row_base, const uint16_t *__restrict__ y_vec, uint16_t *__restrict__ parts) {
    const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= (uint64_t)d.xn * d.zn) return;
    const uint64_t b = xz_end[row_base + row - 1], e = xz_end[row_base + row];
    const uint16_t *R = im + row * (uint64_t)d.yn;
    for (uint64_t i = b + lane; i < e; i += 32) parts[i] = R[y_vec[i]];
}

// The same gather with four particles per lane and step (8-byte y and value
// accesses, four independent image reads in flight per lane); the particles
// before the first index that is a multiple of four and after the last whole
// group of four go one per lane.  y_vec and parts must be 8-byte aligned.
__global__ void gather4_kernel(const uint16_t *__restrict__ im, LevelDims d, const uint64_t *__restrict__ xz_end,
                               uint64_t row_base, const uint16_t *__restrict__ y_vec, uint16_t *__restrict__ parts) {
    const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= (uint64_t)d.xn * d.zn) return;
    const uint64_t b = xz_end[row_base + row - 1], e = xz_end[row_base + row];
    const uint16_t *R = im + row * (uint64_t)d.yn;
    const uint64_t i0 = min((b + 3) & ~uint64_t(3), e), i1 = i0 + ((e - i0) & ~uint64_t(3));
    if ((uint64_t)lane < i0 - b) parts[b + lane] = R[y_vec[b + lane]];
    for (uint64_t i = i0 + 4 * (uint64_t)lane; i < i1; i += 128) {
        const uint2 yv = *reinterpret_cast<const uint2 *>(y_vec + i);
        const uint32_t v0 = R[yv.x & 0xffffu], v1 = R[yv.x >> 16], v2 = R[yv.y & 0xffffu], v3 = R[yv.y >> 16];
        *reinterpret_cast<uint2 *>(parts + i) = make_uint2(v0 | v1 << 16, v2 | v3 << 16);
    }
    if ((uint64_t)lane < e - i1) parts[i1 + lane] = R[y_vec[i1 + lane]];
}


// ---------------------------------------------------------------------------
// APR tree (APR.hpp:633-689, LinearAccess.hpp:67-122)
// ---------------------------------------------------------------------------
__global__ void tree_mark_kernel(LevelDims d, const uint64_t *__restrict__ xz_end, uint64_t row_base,
                                 const uint16_t *__restrict__ y_vec, uint8_t *__restrict__ flags, LevelDims dp) {
    const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= (uint64_t)d.xn * d.zn) return;
    const int x = (int)(row % (uint64_t)d.xn), z = (int)(row / (uint64_t)d.xn);
    const uint64_t b = xz_end[row_base + row - 1], e = xz_end[row_base + row];
    uint8_t *P = flags + idx3(0, x / 2, z / 2, dp.yn, dp.xn);
    for (uint64_t i = b + lane; i < e; i += 32) P[y_vec[i] / 2] = 1;
}

__global__ void tree_prop_kernel(uint8_t *__restrict__ p, LevelDims d, const uint8_t *__restrict__ c, LevelDims dc) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (uint64_t)d.yn * d.xn * d.zn) return;
    int y, x, z;
    cell_of(g, d.yn, d.xn, y, x, z);
    p[g] = p[g] | c[idx3(2 * y, 2 * x, 2 * z, dc.yn, dc.xn)];
}

__global__ void flag_count_kernel(const uint8_t *__restrict__ f, LevelDims d, uint64_t *__restrict__ xz_end,
                                  uint64_t row_base) {
    const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= (uint64_t)d.xn * d.zn) return;
    const uint8_t *R = f + row * (uint64_t)d.yn;
    unsigned c = 0;
    for (int y = lane; y < d.yn; y += 32) c += R[y];
    c = __reduce_add_sync(0xffffffffu, c);
    if (lane == 0) xz_end[row_base + row] = c;
}

__global__ void flag_fill_kernel(const uint8_t *__restrict__ f, LevelDims d, const uint64_t *__restrict__ xz_end,
                                 uint64_t row_base, uint16_t *__restrict__ y_vec) {
    const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= (uint64_t)d.xn * d.zn) return;
    const uint8_t *R = f + row * (uint64_t)d.yn;
    uint64_t o = xz_end[row_base + row - 1];
    const unsigned lt = (1u << lane) - 1u;
    for (int y0 = 0; y0 < d.yn; y0 += 32) {
        const int y = y0 + lane;
        const bool fl = y < d.yn && R[y] != 0;
        const unsigned m = __ballot_sync(0xffffffffu, fl);
        if (fl) y_vec[o + __popc(m & lt)] = (uint16_t)y;
        o += __popc(m);
    }
}

LevelDims dims(const Geom &g, int l) { return LevelDims{g.y_num[l], g.x_num[l], g.z_num[l]}; }
uint64_t ncell(const Geom &g, int l) { return (uint64_t)g.y_num[l] * g.x_num[l] * g.z_num[l]; }
uint64_t nrow(const Geom &g, int l) { return (uint64_t)g.x_num[l] * g.z_num[l]; }
unsigned row_blocks(uint64_t rows) { return blocks_for(rows * 32, 256); }

void launch_gather(const uint16_t *im, LevelDims d, const uint64_t *xz_end, uint64_t row_base, const uint16_t *y_vec,
                   uint16_t *parts, uint64_t rows, cudaStream_t s) {
    if ((((uintptr_t)y_vec | (uintptr_t)parts) & 7) == 0)
        gather4_kernel<<<row_blocks(rows), 256, 0, s>>>(im, d, xz_end, row_base, y_vec, parts);
    else
        gather_kernel<<<row_blocks(rows), 256, 0, s>>>(im, d, xz_end, row_base, y_vec, parts);
}

// (groups of a row / kRowThreads, x, z) of level l: the grid of the row kernels
constexpr int kRowThreads = 128;
dim3 row_grid(int groups, int xn, int zn) {
    return dim3((unsigned)std::max((groups + kRowThreads - 1) / kRowThreads, 1), (unsigned)xn, (unsigned)zn);
}
dim3 row_grid(int groups, const Geom &g, int l) { return row_grid(groups, g.x_num[l], g.z_num[l]); }

}  // namespace

template <typename V>
void launch_reconstruct(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const V *parts, V *img,
                        bool level, cudaStream_t s) {
    APRB_PROF("reconstruct", s);
    const uint64_t rows = nrow(g, g.l_max);
    if (!rows) return;
    if (level)
        reconstruct_kernel<V, true><<<row_blocks(rows), 256, 0, s>>>(g, xz_end, y_vec, parts, img);
    else
        reconstruct_kernel<V, false><<<row_blocks(rows), 256, 0, s>>>(g, xz_end, y_vec, parts, img);
    count_launch();
    APRB_CHECK_LAUNCH();
}
template void launch_reconstruct<uint16_t>(const Geom &, const uint64_t *, const uint16_t *, const uint16_t *,
                                           uint16_t *, bool, cudaStream_t);
template void launch_reconstruct<float>(const Geom &, const uint64_t *, const uint16_t *, const float *, float *, bool,
                                        cudaStream_t);
template void launch_reconstruct<uint8_t>(const Geom &, const uint64_t *, const uint16_t *, const uint8_t *,
                                          uint8_t *, bool, cudaStream_t);



void inclusive_scan_u64(uint64_t *data, uint64_t n, DevBuf &tmp, cudaStream_t s) {
    const uint64_t nb = (n + kScanBlock - 1) / kScanBlock;
    uint64_t *sums = tmp.as_on<uint64_t>(nb + 1, s);
    scan_sums_kernel<<<(unsigned)nb, kScanThreads, 0, s>>>(data, n, sums);
    scan_sums_serial_kernel<<<1, 1024, 0, s>>>(sums, nb);
    scan_apply_kernel<<<(unsigned)nb, kScanThreads, 0, s>>>(data, n, sums);
    count_launch(3);
    APRB_CHECK_LAUNCH();
}

void launch_pulling_scheme(const Geom &g, Pyramid &pm, cudaStream_t s, bool fill_pyramid) {
    const int top = g.l_max - 1, lmin = g.l_min;
    if (top < lmin) return;
    APRB_PROF("pulling_scheme", s);
    for (int l = top - 1; l >= lmin && fill_pyramid; --l) {
        const bool v4 = g.y_num[l + 1] % 8 == 0 && g.y_num[l] % 4 == 0 && ((uintptr_t)pm.level[l + 1] & 7) == 0 &&
                        ((uintptr_t)pm.level[l] & 3) == 0 && ((uintptr_t)pm.status[l] & 3) == 0;
        if (v4)
            pyramid_fill4_kernel<<<row_grid(g.y_num[l] / 4, g, l), kRowThreads, 0, s>>>(
                pm.level[l + 1], dims(g, l + 1), pm.level[l], pm.status[l], dims(g, l), l, l == lmin);
        else
            pyramid_fill_kernel<<<blocks_for(ncell(g, l), 256), 256, 0, s>>>(pm.level[l + 1], dims(g, l + 1),
                                                                            pm.level[l], pm.status[l], dims(g, l), l,
                                                                            l == lmin);
        count_launch();
    }
    APRB_CHECK_LAUNCH();
    for (int l = top; l >= lmin; --l) {
        const dim3 dgrid((g.y_num[l] + kDY - 1) / kDY, (g.x_num[l] + kDX - 1) / kDX, (g.z_num[l] + kDZ - 1) / kDZ);
        const dim3 dgrid16((g.y_num[l] + kD16Y - 1) / kD16Y, dgrid.y, dgrid.z);
        const bool by16 = g.y_num[l] % 16 == 0 && ((uintptr_t)pm.status[l] & 15) == 0;
        const bool by4 = g.y_num[l] % 4 == 0 && ((uintptr_t)pm.status[l] & 3) == 0;
        if (l != top) {
            if (by16)
                dilate16_kernel<0><<<dgrid16, 256, 0, s>>>(pm.status[l], dims(g, l));
            else if (by4)
                dilate4_kernel<0><<<dgrid, 256, 0, s>>>(pm.status[l], dims(g, l));
            else
                dilate_kernel<0><<<dgrid, 256, 0, s>>>(pm.status[l], dims(g, l));
            if (g.y_num[l + 1] % 8 == 0)
                set_filler8_kernel<<<row_grid(g.y_num[l + 1] / 8, g, l + 1), kRowThreads, 0, s>>>(
                    pm.status[l], dims(g, l), pm.status[l + 1], dims(g, l + 1));
            else
                set_filler_kernel<<<blocks_for(ncell(g, l + 1), 256), 256, 0, s>>>(pm.status[l], dims(g, l),
                                                                                  pm.status[l + 1], dims(g, l + 1));
            count_launch(2);
        }
        if (by16)
            dilate16_kernel<1><<<dgrid16, 256, 0, s>>>(pm.status[l], dims(g, l));
        else if (by4)
            dilate4_kernel<1><<<dgrid, 256, 0, s>>>(pm.status[l], dims(g, l));
        else
            dilate_kernel<1><<<dgrid, 256, 0, s>>>(pm.status[l], dims(g, l));
        count_launch();
        if (l - 1 >= lmin) {
            if (g.y_num[l] % 8 == 0)
                fill_parent4_kernel<<<row_grid(g.y_num[l - 1] / 4, g, l - 1), kRowThreads, 0, s>>>(
                    pm.status[l], dims(g, l), pm.status[l - 1], dims(g, l - 1));
            else
                fill_parent_kernel<<<blocks_for(ncell(g, l - 1), 256), 256, 0, s>>>(pm.status[l], dims(g, l),
                                                                                   pm.status[l - 1], dims(g, l - 1));
            count_launch();
        }
    }
    APRB_CHECK_LAUNCH();
}

uint64_t launch_linear_counts(const Geom &g, Pyramid &pm, uint64_t *xz_end, uint64_t n_xz, int min_type,
                              DevBuf &scan_tmp, cudaStream_t s) {
    APRB_PROF("linear_counts", s);
    const int L = g.l_max, lmin = g.l_min;
    APRB_CUDA(cudaMemsetAsync(xz_end, 0, n_xz * sizeof(uint64_t), s));
    for (int l = lmin + 1; l < L; ++l) {
        const uint64_t plane8 = (uint64_t)(g.y_num[l] / 8) * (uint64_t)g.x_num[l];
        if (g.y_num[l] % 8 == 0 && plane8 < (1ull << 31))
            eqopt8_kernel<<<dim3((unsigned)((plane8 + 255) / 256), (unsigned)g.z_num[l]), 256, 0, s>>>(
                pm.status[l - 1], dims(g, l - 1), pm.status[l], dims(g, l), min_type);
        else
            eqopt_kernel<<<blocks_for(ncell(g, l), 256), 256, 0, s>>>(pm.status[l - 1], dims(g, l - 1), pm.status[l],
                                                                     dims(g, l), min_type);
        count_launch();
    }
    for (int l = lmin; l < L - 1; ++l) {
        row_count_kernel<<<row_blocks(nrow(g, l)), 256, 0, s>>>(pm.status[l], dims(g, l), xz_end, g.level_xz[l],
                                                               min_type);
        count_launch();
    }
    const int vec16 = g.y_num[L - 1] % 16 == 0 && ((uintptr_t)pm.status[L - 1] & 15) == 0;
    row_count_top_kernel<<<row_blocks(nrow(g, L - 1)), 256, 0, s>>>(pm.status[L - 1], dims(g, L - 1), xz_end,
                                                                   g.level_xz[L - 1], g.level_xz[L], g.y_num[L],
                                                                   g.x_num[L], g.z_num[L], min_type, vec16);
    count_launch();
    APRB_CHECK_LAUNCH();
    inclusive_scan_u64(xz_end, n_xz, scan_tmp, s);
    uint64_t P = 0;
    APRB_CUDA(cudaMemcpyAsync(&P, xz_end + n_xz - 1, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    APRB_CUDA(cudaStreamSynchronize(s));
    return P;
}

void launch_linear_fill(const Geom &g, const Pyramid &pm, const uint64_t *xz_end, uint16_t *y_vec, int min_type,
                        cudaStream_t s) {
    APRB_PROF("linear_fill", s);
    const int L = g.l_max, lmin = g.l_min;
    for (int l = lmin; l < L - 1; ++l) {
        row_fill_kernel<<<row_blocks(nrow(g, l)), 256, 0, s>>>(pm.status[l], dims(g, l), xz_end, g.level_xz[l], y_vec,
                                                              min_type);
        count_launch();
    }
    const int vec4 = g.y_num[L - 1] % 4 == 0 && ((uintptr_t)pm.status[L - 1] & 3) == 0;
    row_fill_top_kernel<<<row_blocks(nrow(g, L - 1)), 256, 0, s>>>(pm.status[L - 1], dims(g, L - 1), xz_end,
                                                                  g.level_xz[L - 1], g.level_xz[L], g.y_num[L],
                                                                  g.x_num[L], g.z_num[L], y_vec, min_type, vec4);
    count_launch();
    APRB_CHECK_LAUNCH();
}

void launch_full_resolution_structure(const Geom &g, uint64_t *xz_end, uint16_t *y_vec, cudaStream_t s) {
    const int L = g.l_max;
    const uint64_t rows = nrow(g, L);
    full_res_counts_kernel<<<blocks_for(rows, 256), 256, 0, s>>>(xz_end, g.level_xz[L], g.y_num[L], rows);
    if (y_vec) full_res_fill_kernel<<<blocks_for(ncell(g, L), 256), 256, 0, s>>>(y_vec, g.y_num[L], ncell(g, L));
    count_launch(y_vec ? 2 : 1);
    APRB_CHECK_LAUNCH();
}

void launch_sample(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const uint16_t *img,
                   uint16_t *parts, DevBuf &pyr, cudaStream_t s) {
    APRB_PROF("sample_image", s);
    const int L = g.l_max, lmin = g.l_min;
    uint64_t total = 0;
    uint64_t off[32] = {};
    for (int l = lmin; l < L; ++l) {
        off[l] = total;
        total += (ncell(g, l) + 7) & ~uint64_t(7);
    }
    uint16_t *base = pyr.as<uint16_t>(total ? total : 8);
    const uint16_t *lev[32] = {};
    lev[L] = img;
    for (int l = L - 1; l >= lmin; --l) {
        uint16_t *o = base + off[l];
        if (g.y_num[l + 1] % 4 == 0 && (l + 1 < L || ((uintptr_t)img & 7) == 0))
            pyr_mean_u16x2_kernel<<<row_grid(g.y_num[l] / 2, g, l), kRowThreads, 0, s>>>(lev[l + 1], dims(g, l + 1), o,
                                                                                dims(g, l));
        else
            pyr_mean_u16_kernel<<<blocks_for(ncell(g, l), 256), 256, 0, s>>>(lev[l + 1], dims(g, l + 1), o,
                                                                            dims(g, l));
        count_launch();
        lev[l] = o;
    }
    for (int l = lmin; l <= L; ++l) {
        launch_gather(lev[l], dims(g, l), xz_end, g.level_xz[l], y_vec, parts, nrow(g, l), s);
        count_launch();
    }
    APRB_CHECK_LAUNCH();
}

// Pieces of launch_sample for a host-buffer call that overlaps its transfers:
// the level l_max - 1 means and the level l_max gather of the full-resolution
// planes [z0, z1) (z0 even; z1 even or the last plane), then the coarser
// levels once level l_max - 1 is complete.
uint16_t *sample_pyramid(const Geom &g, DevBuf &pyr, uint64_t off[32]) {
    uint64_t total = 0;
    for (int l = g.l_min; l < g.l_max; ++l) {
        off[l] = total;
        total += (ncell(g, l) + 7) & ~uint64_t(7);
    }
    return pyr.as<uint16_t>(total ? total : 8);
}

void launch_sample_slab(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const uint16_t *img, int z0,
                        int z1, uint16_t *pyr_top, uint16_t *parts, cudaStream_t s) {
    const int L = g.l_max;
    const uint64_t plane = (uint64_t)g.y_num[L] * g.x_num[L];
    const LevelDims di{g.y_num[L], g.x_num[L], z1 - z0};
    const uint16_t *slab = img + (uint64_t)z0 * plane;
    if (L > g.l_min) {
        const LevelDims d{g.y_num[L - 1], g.x_num[L - 1], (z1 - z0 + 1) / 2};
        uint16_t *o = pyr_top + (uint64_t)(z0 / 2) * d.yn * d.xn;
        const uint64_t nout = (uint64_t)d.yn * d.xn * d.zn;
        if (di.yn % 4 == 0 && ((uintptr_t)slab & 7) == 0)
            pyr_mean_u16x2_kernel<<<row_grid(d.yn / 2, d.xn, d.zn), kRowThreads, 0, s>>>(slab, di, o, d);
        else
            pyr_mean_u16_kernel<<<blocks_for(nout, 256), 256, 0, s>>>(slab, di, o, d);
        count_launch();
    }
    const uint64_t rows = (uint64_t)(z1 - z0) * di.xn;
    launch_gather(slab, di, xz_end, g.level_xz[L] + (uint64_t)z0 * di.xn, y_vec, parts, rows, s);
    count_launch();
    APRB_CHECK_LAUNCH();
}

void launch_sample_coarse(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, uint16_t *base,
                          const uint64_t off[32], uint16_t *parts, cudaStream_t s) {
    const int L = g.l_max, lmin = g.l_min;
    for (int l = L - 2; l >= lmin; --l) {
        uint16_t *o = base + off[l];
        const uint16_t *in = base + off[l + 1];
        if (g.y_num[l + 1] % 4 == 0)
            pyr_mean_u16x2_kernel<<<row_grid(g.y_num[l] / 2, g, l), kRowThreads, 0, s>>>(in, dims(g, l + 1), o,
                                                                                       dims(g, l));
        else
            pyr_mean_u16_kernel<<<blocks_for(ncell(g, l), 256), 256, 0, s>>>(in, dims(g, l + 1), o, dims(g, l));
        count_launch();
    }
    for (int l = lmin; l < L; ++l) {
        launch_gather(base + off[l], dims(g, l), xz_end, g.level_xz[l], y_vec, parts, nrow(g, l), s);
        count_launch();
    }
    APRB_CHECK_LAUNCH();
}

uint64_t sample_scratch_elems(const Geom &g) {
    uint64_t total = 0;
    for (int l = g.l_min; l < g.l_max; ++l) total += (ncell(g, l) + 7) & ~uint64_t(7);
    return total;
}

void launch_sample_scratch(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const uint16_t *img,
                           uint16_t *parts, uint16_t *scratch, cudaStream_t s) {
    APRB_PROF("sample", s);
    const int L = g.l_max, lmin = g.l_min;
    uint64_t off = 0;
    const uint16_t *lev[32] = {};
    uint16_t *slot[32] = {};
    for (int l = lmin; l < L; ++l) {
        slot[l] = scratch + off;
        off += (ncell(g, l) + 7) & ~uint64_t(7);
    }
    lev[L] = img;
    for (int l = L - 1; l >= lmin; --l) {
        pyr_mean_u16_kernel<<<blocks_for(ncell(g, l), 256), 256, 0, s>>>(lev[l + 1], dims(g, l + 1), slot[l],
                                                                        dims(g, l));
        count_launch();
        lev[l] = slot[l];
    }
    for (int l = lmin; l <= L; ++l) {
        gather_kernel<<<row_blocks(nrow(g, l)), 256, 0, s>>>(lev[l], dims(g, l), xz_end, g.level_xz[l], y_vec, parts);
        count_launch();
    }
    APRB_CHECK_LAUNCH();
}

// z-tiling of APRConverterBatch (APRConverterBatch.hpp:125-160)
ZTile z_tile(int b, int nb, int zn, int zblock, int ghost) {
    ZTile t;
    t.z0 = b * zblock;
    t.zf = (b == nb - 1) ? zn : (b + 1) * zblock;
    t.gl = std::min(t.z0, ghost);
    t.gr = std::min(zn - t.zf, ghost);
    t.pz = t.zf + t.gr - (t.z0 - t.gl);
    return t;
}

// fill_global_particle_cell_tree (APRConverterBatch.hpp:282-314): the tile's
// levels at pct l_max (lev_top, ds tile dims) and their max pyramid fill the
// global particle-cell pyramid.  tmp holds the tile pyramid.
void launch_fill_patch(const Geom &g, Pyramid &pm, const uint8_t *lev_top, const ZTile &t, DevBuf &tmp,
                       cudaStream_t s) {
    const int top = g.l_max - 1, lmin = g.l_min;
    if (top < lmin) return;
    APRB_PROF("fill_patch", s);
    LevelDims pd[32];
    pd[top] = LevelDims{g.y_num[top], g.x_num[top], (t.pz + 1) / 2};
    uint64_t off[32] = {}, total = 0;
    for (int l = top - 1; l >= lmin; --l) {
        pd[l] = LevelDims{g.y_num[l], g.x_num[l], (pd[l + 1].zn + 1) / 2};
        off[l] = total;
        total += ((uint64_t)pd[l].yn * pd[l].xn * pd[l].zn + 15) & ~uint64_t(15);
    }
    uint8_t *base = tmp.as_on<uint8_t>(total ? total : 16, s);
    const uint8_t *lev = lev_top;
    for (int l = top; l >= lmin; --l) {
        uint8_t *cur = nullptr;
        if (l != top) {
            cur = base + off[l];
            pyramid_fill_kernel<<<blocks_for((uint64_t)pd[l].yn * pd[l].xn * pd[l].zn, 256), 256, 0, s>>>(
                lev, pd[l + 1], cur, nullptr, pd[l], l, 0);
            count_launch();
            lev = cur;
        }
        const int lf = 1 << (top + 1 - l);
        const int zlo = t.gl / lf, zhi = pd[l].zn - t.gr / lf, offz = t.z0 / lf - t.gl / lf;
        const int mode = l == top ? 0 : (l == lmin ? 1 : 2);
        if (zhi > zlo) {
            fill_patch_kernel<<<blocks_for((uint64_t)(zhi - zlo) * pd[l].xn * pd[l].yn, 256), 256, 0, s>>>(
                lev, pd[l], pm.status[l], dims(g, l), zlo, zhi, offz, l, mode);
            count_launch();
        }
    }
    APRB_CHECK_LAUNCH();
}

void launch_sample_by_block(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const uint16_t *img,
                            uint16_t *parts, int zblock, int ghost, DevBuf &pyr, cudaStream_t s) {
    APRB_PROF("sample_image_by_block", s);
    const int L = g.l_max, lmin = g.l_min;
    const int zn = g.z_num[L];
    const int nb = std::max(zn / zblock, 1);
    for (int b = 0; b < nb; ++b) {
        const ZTile t = z_tile(b, nb, zn, zblock, ghost);
        LevelDims pd[32];
        pd[L] = LevelDims{g.y_num[L], g.x_num[L], t.pz};
        uint64_t off[32] = {}, total = 0;
        for (int l = L - 1; l >= lmin; --l) {
            pd[l] = LevelDims{g.y_num[l], g.x_num[l], (pd[l + 1].zn + 1) / 2};
            off[l] = total;
            total += ((uint64_t)pd[l].yn * pd[l].xn * pd[l].zn + 7) & ~uint64_t(7);
        }
        uint16_t *base = pyr.as<uint16_t>(total ? total : 8);
        const uint16_t *lev[32] = {};
        lev[L] = img + (uint64_t)(t.z0 - t.gl) * g.x_num[L] * g.y_num[L];
        for (int l = L - 1; l >= lmin; --l) {
            uint16_t *o = base + off[l];
            pyr_mean_u16_kernel<<<blocks_for((uint64_t)pd[l].yn * pd[l].xn * pd[l].zn, 256), 256, 0, s>>>(
                lev[l + 1], pd[l + 1], o, pd[l]);
            count_launch();
            lev[l] = o;
        }
        for (int l = lmin; l <= L; ++l) {
            const int lf = 1 << (L - l);
            const int zlo = t.gl / lf, zhi = pd[l].zn - t.gr / lf, offz = t.z0 / lf - t.gl / lf;
            if (zhi <= zlo) continue;
            gather_patch_kernel<<<row_blocks((uint64_t)(zhi - zlo) * pd[l].xn), 256, 0, s>>>(
                lev[l], pd[l], zlo, zhi, offz, g.z_num[l], xz_end, g.level_xz[l], y_vec, parts);
            count_launch();
        }
        APRB_CHECK_LAUNCH();
    }
}

uint64_t launch_tree_build(const Geom &g, const uint64_t *xz_end, const uint16_t *y_vec, const Geom &tg,
                           uint64_t *t_xz_end, uint64_t t_n_xz, DevBuf &flags, DevBuf &scan_tmp, cudaStream_t s) {
    APRB_PROF("tree_build", s);
    uint64_t total = 0;
    uint64_t off[32] = {};
    for (int t = tg.l_min; t <= tg.l_max; ++t) {
        off[t] = total;
        total += (ncell(tg, t) + 15) & ~uint64_t(15);
    }
    uint8_t *f = flags.as<uint8_t>(total ? total : 16);
    APRB_CUDA(cudaMemsetAsync(f, 0, total ? total : 16, s));
    for (int l = g.l_max; l >= g.l_min; --l) {
        if (l - 1 < tg.l_min) continue;
        tree_mark_kernel<<<row_blocks(nrow(g, l)), 256, 0, s>>>(dims(g, l), xz_end, g.level_xz[l], y_vec,
                                                               f + off[l - 1], dims(tg, l - 1));
        count_launch();
    }
    for (int t = tg.l_max - 1; t >= tg.l_min; --t) {
        tree_prop_kernel<<<blocks_for(ncell(tg, t), 256), 256, 0, s>>>(f + off[t], dims(tg, t), f + off[t + 1],
                                                                       dims(tg, t + 1));
        count_launch();
    }
    APRB_CUDA(cudaMemsetAsync(t_xz_end, 0, t_n_xz * sizeof(uint64_t), s));
    for (int t = tg.l_min; t <= tg.l_max; ++t) {
        flag_count_kernel<<<row_blocks(nrow(tg, t)), 256, 0, s>>>(f + off[t], dims(tg, t), t_xz_end, tg.level_xz[t]);
        count_launch();
    }
    APRB_CHECK_LAUNCH();
    inclusive_scan_u64(t_xz_end, t_n_xz, scan_tmp, s);
    uint64_t T = 0;
    APRB_CUDA(cudaMemcpyAsync(&T, t_xz_end + t_n_xz - 1, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    APRB_CUDA(cudaStreamSynchronize(s));
    return T;
}

void launch_tree_fill(const Geom &tg, const DevBuf &flags, const uint64_t *t_xz_end, uint16_t *t_y_vec,
                      cudaStream_t s) {
    uint64_t total = 0;
    const uint8_t *f = (const uint8_t *)flags.p;
    for (int t = tg.l_min; t <= tg.l_max; ++t) {
        flag_fill_kernel<<<row_blocks(nrow(tg, t)), 256, 0, s>>>(f + total, dims(tg, t), t_xz_end, tg.level_xz[t],
                                                                t_y_vec);
        count_launch();
        total += (ncell(tg, t) + 15) & ~uint64_t(15);
    }
    APRB_CHECK_LAUNCH();
}

}  // namespace aprb
