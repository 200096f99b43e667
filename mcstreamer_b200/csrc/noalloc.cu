// noalloc.cu -- mcs_moments_noalloc: the population moments for callers that cannot
// allocate device memory.
//
// Some callers are not allowed to call cudaMalloc at the point where they need the
// diagnostics: a host loop that runs under a fixed memory budget decided at start-up, an
// embedding application whose allocator owns all device memory, or code running where an
// allocation would synchronise the device or is forbidden outright.  They hold the particle
// arrays themselves and only need the reduction.  This entry point reads caller-owned
// device arrays, writes to a caller-owned device output, and keeps its per-chunk partial
// sums in a fixed array compiled into the library (below), so it performs no allocation of
// any kind.
//
// The fixed array holds kNoallocMaxChunks chunks of kNoallocChunk particles, so one call
// accepts at most MCS_NOALLOC_MAX_PARTICLES particles; larger sizes are rejected with
// MCS_ERR_ARG before anything runs.  Every call shares the array and it keeps the previous
// call's contents; each call rewrites every partial it reads, so nothing has to start at
// zero, but calls whose kernels overlap on the GPU (different streams, or several host
// threads) race on it and must be serialised by the caller.
#include <mutex>

#include "host_util.h"
#include "mcs_device.cuh"

namespace {

constexpr int kNoallocBlock = 256;
constexpr int kNoallocItems = 32;
constexpr long long kNoallocChunk = (long long)kNoallocBlock * kNoallocItems;   // 8192 particles
constexpr int kNoallocMaxChunks = 8192;
constexpr int kNoallocMoments = MCS_MOMENTS_BASE;                               // 18 sums
static_assert(kNoallocChunk * kNoallocMaxChunks == MCS_NOALLOC_MAX_PARTICLES, "limit mismatch");

// Per-chunk partial sums: 8192 x 18 doubles = 1.18 MB per device that loads the library,
// held until the process exits.
static __device__ __align__(256) double g_noalloc_partials[kNoallocMaxChunks * kNoallocMoments];

// Device address of g_noalloc_partials, looked up once per device.
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_addr[kMaxDevices] = {};

int noalloc_scratch(int device, double** out) {
    if (device < 0 || device >= kMaxDevices) return MCS_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[device]) {
        int prev = 0;
        if (cudaGetDevice(&prev) != cudaSuccess) return MCS_ERR_CUDA;
        if (cudaSetDevice(device) != cudaSuccess) return MCS_ERR_CUDA;
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        cudaSetDevice(prev);
        if (e != cudaSuccess || !p) return MCS_ERR_CUDA;
        g_noalloc_addr[device] = static_cast<double*>(p);
    }
    *out = g_noalloc_addr[device];
    return MCS_OK;
}

template <typename T>
struct RawArrays {
    const T* f[7];   // x y z vx vy vz w
    const uint8_t* act;
};

// Chunk c (kNoallocChunk consecutive particles) -> partials[c][0..18), fixed order.
template <typename T>
__global__ void __launch_bounds__(kNoallocBlock) k_noalloc_partials(RawArrays<T> a, long long n, double* partials) {
    __shared__ double red[kNoallocBlock / 32][kNoallocMoments];
    double acc[kNoallocMoments];
#pragma unroll
    for (int q = 0; q < kNoallocMoments; ++q) acc[q] = 0.0;
    acc[MCS_M_EMAX] = -INFINITY;
    const long long base = (long long)blockIdx.x * kNoallocChunk;
    for (int it = 0; it < kNoallocItems; ++it) {
        const long long i = base + (long long)it * kNoallocBlock + threadIdx.x;
        if (i >= n) break;
        const double vx = a.f[3][i], vy = a.f[4][i], vz = a.f[5][i];
        const double eng = 0.5 * mcs::kElectronMass * (vx * vx + vy * vy + vz * vz);
        acc[MCS_M_EMAX] = fmax(acc[MCS_M_EMAX], eng);
        if (!a.act[i]) continue;
        const double x = a.f[0][i], y = a.f[1][i], z = a.f[2][i], w = a.f[6][i];
        acc[MCS_M_COUNT] += 1.0;
        acc[MCS_M_W] += w;
        acc[MCS_M_X] += x; acc[MCS_M_X + 1] += y; acc[MCS_M_X + 2] += z;
        acc[MCS_M_X2] += x * x; acc[MCS_M_X2 + 1] += y * y; acc[MCS_M_X2 + 2] += z * z;
        acc[MCS_M_V] += vx; acc[MCS_M_V + 1] += vy; acc[MCS_M_V + 2] += vz;
        acc[MCS_M_E] += eng;
        acc[MCS_M_WE] += w * eng;
        acc[MCS_M_WX] += w * x; acc[MCS_M_WX + 1] += w * y; acc[MCS_M_WX + 2] += w * z;
        acc[MCS_M_WX2] += w * (x * x + y * y + z * z);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kNoallocMoments; ++q) {
        const double v = q == MCS_M_EMAX ? mcs::warp_max(acc[q]) : mcs::warp_sum(acc[q]);
        if (lane == 0) red[wid][q] = v;
    }
    __syncthreads();
    if (threadIdx.x < kNoallocMoments) {
        const int q = threadIdx.x;
        double r = q == MCS_M_EMAX ? -INFINITY : 0.0;
        for (int wv = 0; wv < kNoallocBlock / 32; ++wv) r = q == MCS_M_EMAX ? fmax(r, red[wv][q]) : r + red[wv][q];
        partials[(long long)blockIdx.x * kNoallocMoments + q] = r;
    }
}

// Block q reduces moment q over the chunks in a fixed order (Kahan per thread).
__global__ void __launch_bounds__(kNoallocBlock) k_noalloc_finish(const double* partials, int nchunks, double* out) {
    __shared__ double red[kNoallocBlock / 32];
    const int q = blockIdx.x;
    const bool mx = q == MCS_M_EMAX;
    double a = mx ? -INFINITY : 0.0, comp = 0.0;
    for (int c = threadIdx.x; c < nchunks; c += kNoallocBlock) {
        const double v = partials[(long long)c * kNoallocMoments + q];
        if (mx) { a = fmax(a, v); continue; }
        const double y = v - comp, s = a + y;
        comp = (s - a) - y;
        a = s;
    }
    a = mx ? mcs::warp_max(a) : mcs::warp_sum(a);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = mx ? -INFINITY : 0.0;
        for (int wv = 0; wv < kNoallocBlock / 32; ++wv) r = mx ? fmax(r, red[wv]) : r + red[wv];
        out[q] = r;
    }
}

template <typename T>
int launch_noalloc(const void* const* arrays, const uint8_t* active, long long n, double* out, double* scratch,
                   cudaStream_t s) {
    RawArrays<T> a;
    for (int q = 0; q < 7; ++q) a.f[q] = static_cast<const T*>(arrays[q]);
    a.act = active;
    const int nchunks = (int)((n + kNoallocChunk - 1) / kNoallocChunk);
    if (nchunks > 0) {
        k_noalloc_partials<T><<<nchunks, kNoallocBlock, 0, s>>>(a, n, scratch);
        if (cudaGetLastError() != cudaSuccess) return MCS_ERR_CUDA;
    }
    k_noalloc_finish<<<kNoallocMoments, kNoallocBlock, 0, s>>>(scratch, nchunks, out);
    return cudaGetLastError() == cudaSuccess ? MCS_OK : MCS_ERR_CUDA;
}

}  // namespace

extern "C" MCS_API int mcs_moments_noalloc(int device, void* stream, int precision, const void* const* arrays,
                                           const uint8_t* active, int64_t n, double* moments_out) {
    if (!arrays || !moments_out || n < 0 || (precision != MCS_FP32 && precision != MCS_FP64)) return MCS_ERR_ARG;
    if (n > MCS_NOALLOC_MAX_PARTICLES) return MCS_ERR_ARG;  // beyond the fixed scratch
    if (n > 0) {
        if (!active) return MCS_ERR_ARG;
        for (int q = 0; q < 7; ++q)
            if (!arrays[q]) return MCS_ERR_ARG;
    }
    double* scratch = nullptr;
    if (int st = noalloc_scratch(device, &scratch)) return st;
    int cur = 0;
    if (cudaGetDevice(&cur) != cudaSuccess) return MCS_ERR_CUDA;
    if (cur != device && cudaSetDevice(device) != cudaSuccess) return MCS_ERR_CUDA;
    const int st = precision == MCS_FP32
                       ? launch_noalloc<float>(arrays, active, n, moments_out, scratch, static_cast<cudaStream_t>(stream))
                       : launch_noalloc<double>(arrays, active, n, moments_out, scratch, static_cast<cudaStream_t>(stream));
    if (cur != device) cudaSetDevice(cur);
    return st;
}
