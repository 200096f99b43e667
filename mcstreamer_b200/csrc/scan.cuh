// scan.cuh -- exclusive scan of n uint32 counts into 64-bit bases: per-tile sums, one CTA
// scanning the tile sums, and a per-tile apply.  Three passes, exact, deterministic.  Each
// translation unit that includes it gets its own copy of the kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace mcs {
namespace {

constexpr int kScanThreads = 1024, kScanPer = 4, kScanTile = kScanThreads * kScanPer;

__global__ void __launch_bounds__(kScanThreads) k_scan_sums(const uint32_t* in, long long n,
                                                            unsigned long long* sums) {
    __shared__ unsigned long long sh[kScanThreads / 32];
    const long long base = (long long)blockIdx.x * kScanTile;
    unsigned long long v = 0;
#pragma unroll
    for (int q = 0; q < kScanPer; ++q) {
        const long long i = base + (long long)q * kScanThreads + threadIdx.x;
        if (i < n) v += in[i];
    }
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned long long t = threadIdx.x < kScanThreads / 32 ? sh[threadIdx.x] : 0;
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (threadIdx.x == 0) sums[blockIdx.x] = t;
    }
}

// Exclusive scan of the block sums in place (one CTA); total in *total.
__global__ void __launch_bounds__(kScanThreads) k_scan_top(unsigned long long* sums, int nb,
                                                           unsigned long long* total) {
    __shared__ unsigned long long sh[kScanThreads];
    unsigned long long carry = 0;
    for (int b0 = 0; b0 < nb; b0 += kScanThreads) {
        const int i = b0 + threadIdx.x;
        const unsigned long long v = i < nb ? sums[i] : 0;
        sh[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < kScanThreads; o <<= 1) {
            const unsigned long long a = threadIdx.x >= (unsigned)o ? sh[threadIdx.x - o] : 0;
            __syncthreads();
            sh[threadIdx.x] += a;
            __syncthreads();
        }
        if (i < nb) sums[i] = carry + sh[threadIdx.x] - v;
        const unsigned long long blk = sh[kScanThreads - 1];
        __syncthreads();
        carry += blk;
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const uint32_t* in, long long n,
                                                             const unsigned long long* sums,
                                                             unsigned long long* out) {
    __shared__ unsigned long long sh[kScanThreads];
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanPer;
    uint32_t v[kScanPer];
    unsigned long long t = 0;
#pragma unroll
    for (int q = 0; q < kScanPer; ++q) {
        v[q] = base + q < n ? in[base + q] : 0u;
        t += v[q];
    }
    sh[threadIdx.x] = t;
    __syncthreads();
    for (int o = 1; o < kScanThreads; o <<= 1) {
        const unsigned long long a = threadIdx.x >= (unsigned)o ? sh[threadIdx.x - o] : 0;
        __syncthreads();
        sh[threadIdx.x] += a;
        __syncthreads();
    }
    unsigned long long run = sums[blockIdx.x] + sh[threadIdx.x] - t;
#pragma unroll
    for (int q = 0; q < kScanPer; ++q)
        if (base + q < n) {
            out[base + q] = run;
            run += v[q];
        }
}

}  // namespace
}  // namespace mcs
