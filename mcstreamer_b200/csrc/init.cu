// init.cu -- initfromfiles! (MCStreamer/src/initdens.jl:64-102) on the device: electrons
// sampled cell by cell from the densities of the init files (nsample, :109-142, with
// randround, :145-159), qfixed's density part set per cell, and the cells above
// fluid_threshold handed to the fluid.
//
// Two passes over the cells.  k_init_count draws every cell's electron count; an exact
// exclusive scan of the counts gives each cell its first slot, so the electrons land in the
// reference's serial order (cells with r fastest, then the electrons of a cell).  After the
// capacity check, k_init_place draws the same counts again from the same streams and writes
// the electrons, qfixed and the fluid.  Compiled with -fmad=false: the arithmetic is the
// reference's, unfused, as the oracle restates it.
//
// Streams: cell c = (i-1) + (j-1) M counts from {c, 0, k/4, TAG_DENSITY}; its electron k
// takes r, z, phi and s from the four words of {c, k, 0, TAG_DENSITY | TAG_DENSITY_PARTICLE}.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/mcs.h"
#include "host_util.h"
#include "mcs_device.cuh"
#include "mcs_internal.h"
#include "pop_ops.h"
#include "scan.cuh"

namespace mcs {
namespace {

constexpr int kInitThreads = 256;

struct InitArgs {
    const double* ne;   // M x N, r fastest
    const double* q;
    int M, N;
    double dr, dz, p, thr;
    int method;
    long long pint;
    unsigned long long seed;
};

struct CellSample {
    long long nume;
    double qf, w;
};

// dV(grid, i) = 2 pi rc dr dz (grid.jl:76) with rc = (i - 1/2) dr.
__device__ __forceinline__ double cell_volume(const InitArgs& a, int i) {
    const double rc = ((double)(i - 1) + 0.5) * a.dr;
    return 2.0 * M_PI * rc * a.dr * a.dz;
}

// max(1, x) of Julia: NaN propagates.
__device__ __forceinline__ double max1(double x) { return (x > 1.0 || isnan(x)) ? x : 1.0; }

// nsample(::NoiselessInitSampling) (:109-127) and nsample(::PoissonInitSampling) (:130-142).
__device__ CellSample nsample(const InitArgs& a, uint32_t c, double ne, double q, double V) {
    Rng r;
    r.init(a.seed, c, 0u, TAG_DENSITY);
    CellSample s;
    if (a.method == MCS_INIT_NOISELESS) {
        const double n = ne * V;
        if (n < 1) {
            s.nume = poisson_draw(r, n);
            s.w = 1.0;
        } else if (n < a.p) {
            const double m = floor(n);   // randround
            s.nume = r.u64() > n - m ? (long long)m : (long long)m + 1;
            s.w = 1.0;
        } else {
            s.nume = a.pint;
            s.w = n / a.p;
        }
        s.qf = q / kElementaryCharge + s.w * (double)s.nume / V;
    } else {
        s.w = max1(ne * V / a.p);
        s.nume = poisson_draw(r, ne * V / s.w);
        const double ni = ne + q / kElementaryCharge;
        const double wi = max1(fabs(ni) * V / a.p);
        const long long numi = poisson_draw(r, fabs(ni) * V / wi);
        const double sg = ni > 0 ? 1.0 : (ni < 0 ? -1.0 : ni);   // sign(ni)
        s.qf = sg * (double)numi * wi / V;
    }
    return s;
}

__global__ void __launch_bounds__(kInitThreads) k_init_count(InitArgs a, uint32_t* counts, uint32_t* status) {
    const long long n = (long long)a.M * a.N;
    for (long long t = blockIdx.x * (long long)kInitThreads + threadIdx.x; t < n;
         t += (long long)gridDim.x * kInitThreads) {
        const int j = (int)(t / a.M) + 1, i = (int)(t - (long long)(j - 1) * a.M) + 1;
        const double ne = a.ne[t];
        uint32_t k = 0;
        if (!(ne > a.thr)) {
            const CellSample s = nsample(a, (uint32_t)t, ne, a.q[t], cell_volume(a, i));
            if (s.nume > 0xffffffffLL) atomicOr(status, ST_CAPACITY);
            k = (uint32_t)std::min<long long>(std::max<long long>(s.nume, 0), 0xffffffffLL);
        }
        counts[t] = k;
    }
}

template <typename T>
__global__ void __launch_bounds__(kInitThreads) k_init_place(InitArgs a, const unsigned long long* base,
                                                            long long n0, PopView<T> P, double* qfd,
                                                            double* ne_fluid) {
    const long long n = (long long)a.M * a.N;
    for (long long t = blockIdx.x * (long long)kInitThreads + threadIdx.x; t < n;
         t += (long long)gridDim.x * kInitThreads) {
        const int j = (int)(t / a.M) + 1, i = (int)(t - (long long)(j - 1) * a.M) + 1;
        const double ne = a.ne[t], q = a.q[t];
        const long long qk = (long long)i + (long long)j * (a.M + 2);
        if (ne > a.thr) {   // initdens.jl:79-83
            ne_fluid[(long long)(i + 1) + (long long)(j + 1) * (a.M + 4)] = ne;
            qfd[qk] = q / kElementaryCharge + ne;
            continue;
        }
        const CellSample s = nsample(a, (uint32_t)t, ne, q, cell_volume(a, i));
        qfd[qk] = s.qf;
        const double rf = (double)(i - 1) * a.dr, zf = (double)(j - 1) * a.dz;
        long long slot = n0 + (long long)base[t];
        for (long long k = 0; k < s.nume; ++k, ++slot) {
            const U4 b = philox10(U4{(uint32_t)t, (uint32_t)k, 0u, TAG_DENSITY | TAG_DENSITY_PARTICLE},
                                  (uint32_t)a.seed, (uint32_t)(a.seed >> 32));
            const double r = a.dr * uni64(b.x) + rf;
            const double z = a.dz * uni64(b.y) + zf;
            const double phi = 2.0 * M_PI * uni64(b.z);
            P.f[0][slot] = (T)(r * cos(phi));
            P.f[1][slot] = (T)(r * sin(phi));
            P.f[2][slot] = (T)z;
            P.f[3][slot] = (T)0;
            P.f[4][slot] = (T)0;
            P.f[5][slot] = (T)0;
            P.f[6][slot] = (T)s.w;
            P.f[7][slot] = (T)(-log(uni64(b.w)));   // nextcoll()
            P.act[slot] = 1;
        }
    }
}

__global__ void k_init_set_count(long long* n, long long v) { *n = v; }

template <typename T>
int place(mcs_pop* p, const InitArgs& a, const unsigned long long* base, long long n0, double* qfd,
          double* ne_fluid, int grid) {
    k_init_place<T><<<grid, kInitThreads, 0, p->ctx->stream>>>(a, base, n0, pop_view<T>(p), qfd, ne_fluid);
    MCS_CK_LAUNCH(p->ctx);
    return MCS_OK;
}

struct DevBuf {
    void* ptr = nullptr;
    ~DevBuf() { if (ptr) cudaFree(ptr); }
};

template <typename T>
int dev_alloc(mcs_ctx* c, DevBuf& b, size_t count, T** out) {
    if (cudaMalloc(&b.ptr, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        b.ptr = nullptr;
        return set_err(c, MCS_ERR_NOMEM, "init: device allocation failed");
    }
    *out = static_cast<T*>(b.ptr);
    return MCS_OK;
}

}  // namespace
}  // namespace mcs

using namespace mcs;

extern "C" {

MCS_API int mcs_init_from_density_device(mcs_pop* p, mcs_grid* g, const double* ne, const double* q, int method,
                                         int64_t ppc, double fluid_threshold, uint64_t seed, int64_t* added) {
    if (!p || !g || !ne || !q) return MCS_ERR_ARG;
    mcs_ctx* c = p->ctx;
    if (g->ctx != c) return set_err(c, MCS_ERR_ARG, "init: population and grid on different contexts");
    if (g->v.type != GRID_CYL) return set_err(c, MCS_ERR_ARG, "init: needs a cylindrical grid");
    if (p->cells) return set_err(c, MCS_ERR_UNSUPPORTED, "init: needs absolute positions (no cell layout)");
    if ((method != MCS_INIT_NOISELESS && method != MCS_INIT_POISSON) || ppc < 1)
        return set_err(c, MCS_ERR_ARG, "init: bad sampling method or particles per cell");
    if (fluid_threshold == fluid_threshold && fluid_threshold < HUGE_VAL && !g->fluid)
        return set_err(c, MCS_ERR_ARG, "init: a finite fluid_threshold needs a fluid on the grid");
    const long long cells = (long long)g->v.M * g->v.N;
    if (cells >= (1LL << 32)) return set_err(c, MCS_ERR_ARG, "init: more than 2^32 cells");
    MCS_CK(c, cudaSetDevice(c->device));
    double* qfd = grid_qfd(g);
    if (!qfd) return MCS_ERR_NOMEM;
    InitArgs a{};
    a.ne = ne;
    a.q = q;
    a.M = g->v.M;
    a.N = g->v.N;
    a.dr = g->v.dr;
    a.dz = g->v.dz;
    a.p = (double)ppc;
    a.pint = ppc;
    a.thr = fluid_threshold;
    a.method = method;
    a.seed = seed;
    // the workspace stays with the grid: counts (4 B per cell), bases (8 B), tile sums, total
    const long long nb = std::max(1LL, (cells + kScanTile - 1) / kScanTile);
    const size_t o_base = ((size_t)cells * 4 + 255) / 256 * 256;
    const size_t o_sums = o_base + ((size_t)cells * 8 + 255) / 256 * 256;
    const size_t o_tot = o_sums + ((size_t)nb * 8 + 255) / 256 * 256;
    const size_t need = o_tot + 256;
    if (g->init_ws_bytes < need) {
        cudaFree(g->d_init_ws);
        g->d_init_ws = nullptr;
        g->init_ws_bytes = 0;
        if (cudaMalloc(&g->d_init_ws, need) != cudaSuccess) {
            cudaGetLastError();
            g->d_init_ws = nullptr;
            return set_err(c, MCS_ERR_NOMEM, "init: device allocation failed");
        }
        g->init_ws_bytes = need;
    }
    char* ws = static_cast<char*>(g->d_init_ws);
    uint32_t* counts = reinterpret_cast<uint32_t*>(ws);
    unsigned long long* base = reinterpret_cast<unsigned long long*>(ws + o_base);
    unsigned long long* sums = reinterpret_cast<unsigned long long*>(ws + o_sums);
    unsigned long long* total = reinterpret_cast<unsigned long long*>(ws + o_tot);
    cudaStream_t st = c->stream;
    const int grid = (int)std::min<long long>((cells + kInitThreads - 1) / kInitThreads, (long long)c->num_sms * 16);
    k_init_count<<<grid, kInitThreads, 0, st>>>(a, counts, c->d_status);
    k_scan_sums<<<(int)nb, kScanThreads, 0, st>>>(counts, cells, sums);
    k_scan_top<<<1, kScanThreads, 0, st>>>(sums, (int)nb, total);
    k_scan_apply<<<(int)nb, kScanThreads, 0, st>>>(counts, cells, sums, base);
    MCS_CK_LAUNCH(c);
    unsigned long long tot = 0;
    long long n0 = 0;
    MCS_CK(c, cudaMemcpyAsync(&tot, total, sizeof(tot), cudaMemcpyDeviceToHost, st));
    MCS_CK(c, cudaMemcpyAsync(&n0, p->d_n + p->cur, sizeof(n0), cudaMemcpyDeviceToHost, st));
    if (int e = sync_status(c)) return e;
    if ((long long)tot > p->cap - n0)   // "Particle limit reached" (initdens.jl:92-94)
        return set_err(c, MCS_ERR_CAPACITY, "init: the sampled electrons exceed the population's capacity");
    double* ne_fluid = g->fluid ? g->fluid->ne[g->fluid->cur] : nullptr;
    const int e = p->precision == MCS_FP32 ? place<float>(p, a, base, n0, qfd, ne_fluid, grid)
                                           : place<double>(p, a, base, n0, qfd, ne_fluid, grid);
    if (e) return e;
    k_init_set_count<<<1, 1, 0, st>>>(p->d_n + p->cur, n0 + (long long)tot);
    MCS_CK_LAUNCH(c);
    if (int e2 = sync_status(c)) return e2;
    if (added) *added = (int64_t)tot;
    return MCS_OK;
}

MCS_API int mcs_grid_read_qfixed_density(mcs_grid* g, double* out) {
    if (!g || !out) return MCS_ERR_ARG;
    mcs_ctx* c = g->ctx;
    if (g->v.type != GRID_CYL) return set_err(c, MCS_ERR_ARG, "qfixed density: needs a cylindrical grid");
    const size_t n = (size_t)(g->v.M + 2) * (g->v.N + 2);
    MCS_CK(c, cudaSetDevice(c->device));
    if (!g->d_qfd) {
        std::fill(out, out + n, 0.0);
        return sync_status(c);
    }
    MCS_CK(c, cudaMemcpyAsync(out, g->d_qfd, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return sync_status(c);
}

MCS_API int mcs_grid_write_qfixed_density(mcs_grid* g, const double* in) {
    if (!g || !in) return MCS_ERR_ARG;
    mcs_ctx* c = g->ctx;
    if (g->v.type != GRID_CYL) return set_err(c, MCS_ERR_ARG, "qfixed density: needs a cylindrical grid");
    MCS_CK(c, cudaSetDevice(c->device));
    double* d = grid_qfd(g);
    if (!d) return MCS_ERR_NOMEM;
    MCS_CK(c, cudaMemcpyAsync(d, in, (size_t)(g->v.M + 2) * (g->v.N + 2) * sizeof(double), cudaMemcpyHostToDevice,
                              c->stream));
    MCS_CK(c, cudaStreamSynchronize(c->stream));
    return MCS_OK;
}

MCS_API int mcs_init_from_density(mcs_pop* p, mcs_grid* g, const double* ne, const double* q, int method,
                                  int64_t ppc, double fluid_threshold, uint64_t seed, int64_t* added) {
    if (!p || !g || !ne || !q) return MCS_ERR_ARG;
    mcs_ctx* c = p->ctx;
    if (g->v.type != GRID_CYL) return set_err(c, MCS_ERR_ARG, "init: needs a cylindrical grid");
    const size_t cells = (size_t)g->v.M * g->v.N;
    MCS_CK(c, cudaSetDevice(c->device));
    DevBuf bn, bq;
    double *dn = nullptr, *dq = nullptr;
    if (int e = dev_alloc(c, bn, cells, &dn)) return e;
    if (int e = dev_alloc(c, bq, cells, &dq)) return e;
    MCS_CK(c, cudaMemcpyAsync(dn, ne, cells * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    MCS_CK(c, cudaMemcpyAsync(dq, q, cells * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    const int e = mcs_init_from_density_device(p, g, dn, dq, method, ppc, fluid_threshold, seed, added);
    cudaStreamSynchronize(c->stream);
    return e;
}

}  // extern "C"
