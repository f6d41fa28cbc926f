// Host stand-ins for the CUDA names used by the byte-parallel and row kernels
// of libapr_b200/csrc/structure.cu, so that tests/test_bytewise_host.py can
// compile those kernels' source with g++ and run every thread of a launch in
// turn on the CPU.
#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <random>
#include <vector>

using std::max;
using std::min;

struct HostDim3 {
    unsigned x, y, z;
};
static HostDim3 blockIdx, threadIdx, blockDim;

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __restrict__

struct uint2 {
    uint32_t x, y;
};
struct uint4 {
    uint32_t x, y, z, w;
};
inline uint2 make_uint2(uint32_t a, uint32_t b) { return {a, b}; }
inline uint4 make_uint4(uint32_t a, uint32_t b, uint32_t c, uint32_t d) { return {a, b, c, d}; }

// __byte_perm(x, y, s): byte i of the result is byte (s >> 4i) & 7 of the
// eight bytes y:x (the selector's sign-replicate bit is not used here).
inline uint32_t __byte_perm(uint32_t x, uint32_t y, uint32_t s) {
    const uint64_t v = ((uint64_t)y << 32) | x;
    uint32_t r = 0;
    for (int i = 0; i < 4; ++i) r |= (uint32_t)((v >> (8 * ((s >> (4 * i)) & 7u))) & 0xFFu) << (8 * i);
    return r;
}

// __vmaxu4(a, b): byte-wise unsigned maximum.
inline uint32_t __vmaxu4(uint32_t a, uint32_t b) {
    uint32_t r = 0;
    for (int i = 0; i < 4; ++i) r |= std::max((a >> (8 * i)) & 0xFFu, (b >> (8 * i)) & 0xFFu) << (8 * i);
    return r;
}

struct LevelDims {
    int yn, xn, zn;
};
