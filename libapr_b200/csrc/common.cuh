// Shared device helpers and host plumbing for libaprb200.
//
// Every kernel in this library is compiled for sm_100a with -fmad=false and
// IEEE division/sqrt, so each float operation rounds where the reference's
// strict-IEEE CPU build rounds.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <string>
#include <utility>

#include "../../include/aprb200.h"

namespace aprb {

// ------------------------------------------------------------------ errors
void set_error(const std::string &msg);
struct Error {
    aprb_status status;
};
#define APRB_CUDA(call)                                                                        \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            ::aprb::set_error(std::string(#call) + ": " + cudaGetErrorString(e_));             \
            throw ::aprb::Error{e_ == cudaErrorMemoryAllocation ? APRB_ERR_OUT_OF_MEMORY       \
                                                                : APRB_ERR_CUDA};              \
        }                                                                                      \
    } while (0)
#define APRB_CHECK_LAUNCH() APRB_CUDA(cudaGetLastError())

void count_launch(uint64_t n = 1);

// Stage timing: a scope that records a CUDA event pair on the stream when
// profiling is enabled (aprb_profile_enable).
void prof_record(const char *name, cudaStream_t s, bool begin);
struct ProfScope {
    const char *name;
    cudaStream_t s;
    ProfScope(const char *n, cudaStream_t st) : name(n), s(st) { prof_record(name, s, true); }
    ~ProfScope() { prof_record(name, s, false); }
};
#define APRB_PROF_CAT2(a, b) a##b
#define APRB_PROF_CAT(a, b) APRB_PROF_CAT2(a, b)
#define APRB_PROF(name, s) ::aprb::ProfScope APRB_PROF_CAT(prof_scope_, __LINE__)(name, s)

inline unsigned blocks_for(uint64_t n, unsigned threads) {
    uint64_t b = (n + threads - 1) / threads;
    return (unsigned)(b == 0 ? 1 : b);
}

// ------------------------------------------------------------------ device buffers
// Stream-ordered allocation from the device's default memory pool, whose
// release threshold is raised so that freed blocks stay reserved for the next
// APR instead of going back to the driver (cudaMalloc/cudaFree synchronise
// the device and cost milliseconds at these sizes).
void *pool_alloc(size_t bytes, cudaStream_t s);

// A device allocation that grows on demand and is reused across calls, as the
// reference converter keeps its scratch images as members.  Pooled buffers
// (get_pooled) come from pool_alloc; release() waits for the device before it
// hands them back, as cudaFree would.
struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    bool pooled = false;
    void *get(size_t bytes) {
        if (bytes > cap) {
            release();
            size_t want = bytes ? bytes : 16;
            APRB_CUDA(cudaMalloc(&p, want));
            cap = want;
        }
        return p;
    }
    void *get_pooled(size_t bytes, cudaStream_t s) {
        if (bytes > cap) {
            release();
            size_t want = bytes ? bytes : 16;
            p = pool_alloc(want, s);
            cap = want;
            pooled = true;
        }
        return p;
    }
    template <typename T>
    T *as(size_t n) {
        return (T *)get(n * sizeof(T));
    }
    template <typename T>
    T *as_pooled(size_t n, cudaStream_t s) {
        return (T *)get_pooled(n * sizeof(T), s);
    }
    // Grows through the pool without a device synchronisation: the old block
    // is freed in the order of stream s.  For buffers whose every use is on
    // the stream of a call that synchronises that stream before it returns
    // (the converter's), so no other stream can still be using the block.
    void *get_on(size_t bytes, cudaStream_t s) {
        if (bytes > cap) {
            if (p) {
                if (pooled)
                    cudaFreeAsync(p, s);
                else
                    cudaFree(p);
            }
            p = nullptr;
            cap = 0;
            const size_t want = bytes ? bytes : 16;
            p = pool_alloc(want, s);
            cap = want;
            pooled = true;
        }
        return p;
    }
    template <typename T>
    T *as_on(size_t n, cudaStream_t s) {
        return (T *)get_on(n * sizeof(T), s);
    }
    void release() {
        if (p) {
            if (pooled) {
                cudaDeviceSynchronize();
                cudaFreeAsync(p, 0);
            } else {
                cudaFree(p);
            }
        }
        p = nullptr;
        cap = 0;
        pooled = false;
    }
    // Back to the pool in the order of stream s, without waiting for the
    // device: only for a block that no stream can still be using.
    void release_idle(cudaStream_t s) {
        if (p) {
            if (pooled)
                cudaFreeAsync(p, s);
            else
                cudaFree(p);
        }
        p = nullptr;
        cap = 0;
        pooled = false;
    }
    void swap(DevBuf &o) {
        std::swap(p, o.p);
        std::swap(cap, o.cap);
        std::swap(pooled, o.pooled);
    }
    ~DevBuf() { release(); }
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
};

// ------------------------------------------------------------------ conversions
// ImageType = uint16 stores convert like the reference's x86-64 build:
// truncate toward zero to 32 bit, keep the low 16 bits; NaN and out-of-range
// give 0.
__host__ __device__ __forceinline__ float cvt_u16(float v) {
    if (!(v > -2147483648.0f && v < 2147483648.0f)) return 0.0f;
    return (float)(uint16_t)(int32_t)v;
}
__host__ __device__ __forceinline__ float cvt_u16d(double v) {
    if (!(v > -2147483648.0 && v < 2147483648.0)) return 0.0f;
    return (float)(uint16_t)(int32_t)v;
}
// round<T> (ComputeGradient.hpp:220-244): std::round then range check.
__device__ __forceinline__ float round_u16(float v, unsigned &err) {
    v = roundf(v);
    if (v < 0.0f || v > 65535.0f) err++;
    return cvt_u16(v);
}
// float -> uint32 as the x86-64 build converts (64-bit truncation, low 32 bits).
__device__ __forceinline__ uint32_t cvt_u32(float v) {
    if (!(v > -9223372036854775808.0f && v < 9223372036854775808.0f)) return 0u;
    return (uint32_t)(long long)v;
}

// x / d, correctly rounded, for a divisor d fixed over a kernel with r its
// correctly rounded reciprocal: Markstein's correction of the product
// (P. Markstein, IA-64 and Elementary Functions, 2000, Theorem 8.10): q =
// RN(x r) is within one ulp of x / d, the remainder e = x - q d is exact in
// one fused multiply-add, and RN(q + e r) is the correctly rounded quotient.
// Quotients that are zero, tiny or not finite take the IEEE division.
// aprb_check_division_by_constant compares it with the IEEE division on all
// 2^32 inputs.
#ifdef __CUDACC__
__device__ __forceinline__ float div_const(float x, float d, float r) {
    const float q = __fmul_rn(x, r);
    const float aq = fabsf(q);
    if (!(aq >= 0x1p-100f && aq <= 0x1p100f)) return __fdiv_rn(x, d);
    const float e = __fmaf_rn(-q, d, x);
    return __fmaf_rn(e, r, q);
}
#endif

__host__ __device__ __forceinline__ size_t idx3(int y, int x, int z, int yn, int xn) {
    return ((size_t)z * (size_t)xn + (size_t)x) * (size_t)yn + (size_t)y;
}

// Level geometry of GenInfo (GenInfo.hpp:33-98), shared host/device.
struct Geom {
    int l_min, l_max;
    int y_num[32], x_num[32], z_num[32];
    uint64_t level_xz[34];
};

}  // namespace aprb
