// pop_ops.cu -- population-level kernels: host-layout conversion, device-wide scan,
// repack! (JuMC/src/population.jl:191-215), Swarm.resample! (Swarm/src/Swarm.jl:193-223),
// moments (Swarm.jl:126-166, population.jl:114-183) and density! (poisson.jl:65-84).
#include "host_util.h"
#include "pop_ops.h"
#include "step.cuh"

namespace mcs {

constexpr uint32_t kOutside = 0xffffffffu;  // mesh layout: particle outside the mesh

// ---------------------------------------------------------------------------------------
// Host layout (AoS doubles, Julia memory layout) <-> device SoA.
// ---------------------------------------------------------------------------------------
template <typename T>
__global__ void k_upload(const double* __restrict__ x, const double* __restrict__ v, const double* __restrict__ w,
                         const double* __restrict__ s, const uint8_t* __restrict__ a, long long n, PopView<T> P,
                         GridView g, int mesh, unsigned int* __restrict__ w_lossy) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double px = x[3 * i], py = x[3 * i + 1], pz = x[3 * i + 2];
        if (mesh) {
            const double u[3] = {(px - g.x0) / g.h, (py - g.y0) / g.h, (pz - g.z0) / g.h};
            const int nc[3] = {g.nx, g.ny, g.nz};
            double fl[3];
            bool in = true;
            for (int d = 0; d < 3; ++d) {
                fl[d] = floor(u[d]);
                in = in && fl[d] >= 0.0 && fl[d] < (double)nc[d];
            }
            if (in) {
                P.cell[i] = (uint32_t)((long long)fl[0] + (long long)g.nx * ((long long)fl[1] + (long long)g.ny * (long long)fl[2]));
                for (int d = 0; d < 3; ++d) {
                    T r = (T)(u[d] - fl[d]);
                    if (r >= (T)1) r = sizeof(T) == 4 ? (T)0x1.fffffep-1f : (T)0x1.fffffffffffffp-1;
                    P.f[d][i] = r;
                }
            } else {
                P.cell[i] = kOutside;
                for (int d = 0; d < 3; ++d) P.f[d][i] = (T)u[d];
            }
        } else {
            P.f[0][i] = (T)px; P.f[1][i] = (T)py; P.f[2][i] = (T)pz;
        }
        P.f[3][i] = (T)v[3 * i]; P.f[4][i] = (T)v[3 * i + 1]; P.f[5][i] = (T)v[3 * i + 2];
        const double wi = w[i];
        const T wc = (T)wi;
        P.f[6][i] = wc;
        if (w_lossy && !((double)wc == wi)) *w_lossy = 1u;   // the weight does not round-trip
        P.f[7][i] = (T)s[i];
        P.act[i] = a[i] ? 1 : 0;
    }
}

// Initial swarm electrons at the origin, weight 1, Maxwellian velocities (maxwellian_draw).
template <typename T>
__global__ void k_init_maxwellian(PopView<T> P, long long n, unsigned long long seed, double sigma) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double vx, vy, vz, s;
        maxwellian_draw(seed, (uint32_t)i, sigma, vx, vy, vz, s);
        P.f[0][i] = (T)0; P.f[1][i] = (T)0; P.f[2][i] = (T)0;
        P.f[3][i] = (T)vx; P.f[4][i] = (T)vy; P.f[5][i] = (T)vz;
        P.f[6][i] = (T)1;
        P.f[7][i] = (T)s;
        P.act[i] = 1;
    }
}

// Store absolute position (px, py, pz) of slot i in the population's layout: absolute, or
// (cell, in-cell offset) on a mesh (offsets clamped below 1; outside the mesh: kOutside and
// the position in cell units).
template <typename T>
__device__ __forceinline__ void put_position(const PopView<T>& P, const GridView& g, int mesh, long long i, double px,
                                             double py, double pz) {
    if (!mesh) {
        P.f[0][i] = (T)px; P.f[1][i] = (T)py; P.f[2][i] = (T)pz;
        return;
    }
    const double u[3] = {(px - g.x0) / g.h, (py - g.y0) / g.h, (pz - g.z0) / g.h};
    const int nc[3] = {g.nx, g.ny, g.nz};
    double fl[3];
    bool in = true;
    for (int d = 0; d < 3; ++d) {
        fl[d] = floor(u[d]);
        in = in && fl[d] >= 0.0 && fl[d] < (double)nc[d];
    }
    if (in) {
        P.cell[i] = (uint32_t)((long long)fl[0] + (long long)g.nx * ((long long)fl[1] + (long long)g.ny * (long long)fl[2]));
        for (int d = 0; d < 3; ++d) {
            T r = (T)(u[d] - fl[d]);
            if (r >= (T)1) r = sizeof(T) == 4 ? (T)0x1.fffffep-1f : (T)0x1.fffffffffffffp-1;
            P.f[d][i] = r;
        }
    } else {
        P.cell[i] = kOutside;
        for (int d = 0; d < 3; ++d) P.f[d][i] = (T)u[d];
    }
}

// A Gaussian cloud of electrons (the streamer workloads' initial condition): position
// centre + N(0, sigma^2) per axis, speed sqrt(2 E / m) in an isotropic direction, weight
// log-uniform on [wmin, wmax] (wmin when equal), s = -log(u).  Eight uniforms of the INIT
// stream of slot i: Box-Muller on (u0,u1), (u2,u3) for the offsets, (u4,u5) direction,
// u6 weight, u7 free flight.
template <typename T>
__global__ void k_init_cloud(PopView<T> P, GridView g, int mesh, long long n, unsigned long long seed, double cx,
                             double cy, double cz, double sigma, double vabs, double wmin, double wmax) {
    const double lw = log(wmax / wmin);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        Rng r;
        r.init(seed, (uint32_t)i, 0u, TAG_INIT);
        double u[8];
        for (int q = 0; q < 8; ++q) u[q] = r.u64();
        const double r0 = sqrt(-2.0 * log(u[0])), r1 = sqrt(-2.0 * log(u[2]));
        double s0, c0, s1, c1;
        sincos(6.283185307179586 * u[1], &s0, &c0);
        sincos(6.283185307179586 * u[3], &s1, &c1);
        put_position(P, g, mesh, i, cx + sigma * (r0 * c0), cy + sigma * (r0 * s0), cz + sigma * (r1 * c1));
        const double uz = 2.0 * u[4] - 1.0, st = sqrt(1.0 - uz * uz);
        double sp, cp;
        sincos(6.283185307179586 * u[5], &sp, &cp);
        P.f[3][i] = (T)(vabs * st * cp);
        P.f[4][i] = (T)(vabs * st * sp);
        P.f[5][i] = (T)(vabs * uz);
        P.f[6][i] = (T)(wmin == wmax ? wmin : wmin * exp(lw * u[6]));
        P.f[7][i] = (T)(-log(u[7]));
        P.act[i] = 1;
    }
}

int launch_init_cloud(mcs_pop* p, long long n, const double c[3], double sigma, double vabs, double wmin, double wmax) {
    mcs_ctx* ctx = p->ctx;
    const int gr = grid_for(ctx, n, 256);
    const GridView gv = grid_view(p->cells);
    const int mesh = p->cells != nullptr;
    if (p->precision == MCS_FP32)
        k_init_cloud<float><<<gr, 256, 0, ctx->stream>>>(pop_view<float>(p), gv, mesh, n, p->seed, c[0], c[1], c[2],
                                                          sigma, vabs, wmin, wmax);
    else
        k_init_cloud<double><<<gr, 256, 0, ctx->stream>>>(pop_view<double>(p), gv, mesh, n, p->seed, c[0], c[1], c[2],
                                                           sigma, vabs, wmin, wmax);
    MCS_CK_LAUNCH(ctx);
    return MCS_OK;
}

// Node field of a Gaussian charge rho = e * rho_peak * exp(-r^2 / 2 sigma^2) at c plus a
// uniform background: E = e_bg + Q(r) / (4 pi eps0 r^2) r_hat with
// Q(r) = e rho_peak (2 pi sigma^2)^(3/2) [erf(r / (sqrt2 sigma)) - sqrt(2/pi) (r/sigma) exp(-r^2/2sigma^2)]
// (Gauss's law for the spherical charge).  FP64 arithmetic; stored as the grid's precision.
__global__ void k_efield_gaussian(GridView g, float4* e32, double* e64, double cx, double cy, double cz, double sigma,
                                  double q0, double ebx, double eby, double ebz) {
    const long long nx1 = g.nx + 1, ny1 = g.ny + 1;
    const long long nn = nx1 * ny1 * (long long)(g.nz + 1);
    const double k4pe = 4.0 * 3.141592653589793 * 8.854187817620389e-12;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nn; q += (long long)gridDim.x * blockDim.x) {
        const long long i = q % nx1, j = (q / nx1) % ny1, k = q / (nx1 * ny1);
        const double dx = (g.x0 + g.h * (double)i) - cx, dy = (g.y0 + g.h * (double)j) - cy,
                     dz = (g.z0 + g.h * (double)k) - cz;
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const double rs = r / sigma;
        const double Q = q0 * (erf(rs / 1.4142135623730951) - 0.7978845608028654 * rs * exp(-0.5 * rs * rs));
        const double f = r > 0.0 ? Q / (k4pe * (r * r * r)) : 0.0;
        const double ex = ebx + f * dx, ey = eby + f * dy, ez = ebz + f * dz;
        if (e32) e32[q] = make_float4((float)ex, (float)ey, (float)ez, 0.0f);
        else { e64[3 * q] = ex; e64[3 * q + 1] = ey; e64[3 * q + 2] = ez; }
    }
}

int launch_efield_gaussian(mcs_grid* g, const double c[3], double sigma, double rho_peak, const double eb[3]) {
    mcs_ctx* ctx = g->ctx;
    const double q0 = kElementaryCharge * rho_peak * pow(2.0 * 3.141592653589793 * sigma * sigma, 1.5);
    const int gr = grid_for(ctx, (long long)g->nq, 256);
    k_efield_gaussian<<<gr, 256, 0, ctx->stream>>>(g->v, reinterpret_cast<float4*>(g->d_e32), g->d_e64, c[0], c[1],
                                                    c[2], sigma, q0, eb[0], eb[1], eb[2]);
    MCS_CK_LAUNCH(ctx);
    return MCS_OK;
}

int launch_init_maxwellian(mcs_pop* p, long long n, double sigma) {
    mcs_ctx* c = p->ctx;
    const int gr = grid_for(c, n, 256);
    if (p->precision == MCS_FP32)
        k_init_maxwellian<float><<<gr, 256, 0, c->stream>>>(pop_view<float>(p), n, p->seed, sigma);
    else
        k_init_maxwellian<double><<<gr, 256, 0, c->stream>>>(pop_view<double>(p), n, p->seed, sigma);
    MCS_CK_LAUNCH(c);
    return MCS_OK;
}

template <typename T>
__device__ __forceinline__ void abs_position(const PopView<T>& P, const GridView& g, int mesh, long long i, double& x,
                                             double& y, double& z) {
    if (!mesh) { x = P.f[0][i]; y = P.f[1][i]; z = P.f[2][i]; return; }
    const uint32_t c = P.cell[i];
    if (c == kOutside) {
        x = g.x0 + g.h * (double)P.f[0][i];
        y = g.y0 + g.h * (double)P.f[1][i];
        z = g.z0 + g.h * (double)P.f[2][i];
        return;
    }
    uint32_t ix, iy, iz;
    cell_split(g, c, ix, iy, iz);
    x = g.x0 + g.h * ((double)ix + (double)P.f[0][i]);
    y = g.y0 + g.h * ((double)iy + (double)P.f[1][i]);
    z = g.z0 + g.h * ((double)iz + (double)P.f[2][i]);
}

template <typename T>
__global__ void k_download(double* __restrict__ x, double* __restrict__ v, double* __restrict__ w, double* __restrict__ s,
                           uint8_t* __restrict__ a, PopView<T> P, GridView g, int mesh) {
    const long long n = *P.n_in;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double px, py, pz;
        abs_position(P, g, mesh, i, px, py, pz);
        x[3 * i] = px; x[3 * i + 1] = py; x[3 * i + 2] = pz;
        v[3 * i] = P.f[3][i]; v[3 * i + 1] = P.f[4][i]; v[3 * i + 2] = P.f[5][i];
        w[i] = P.f[6][i];
        s[i] = P.f[7][i];
        a[i] = P.act[i];
    }
}

// ---------------------------------------------------------------------------------------
// Device-wide exclusive scan of u32 counts, single pass (decoupled look-back over tiles
// handed out by an atomic ticket).  in == nullptr scans the active flags of the population.
// total (optional) receives the sum.
// ---------------------------------------------------------------------------------------
constexpr int SCAN_BLOCK = 256, SCAN_ITEMS = 16, SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

__global__ void __launch_bounds__(SCAN_BLOCK) k_scan(const uint32_t* __restrict__ in, const uint8_t* __restrict__ act,
                                                     uint32_t* __restrict__ out, const long long* n_ptr,
                                                     unsigned long long* tile_status, uint32_t* counters, uint32_t epoch,
                                                     uint32_t* status, long long* total) {
    __shared__ uint32_t s_tile, s_excl, s_warp[SCAN_BLOCK / 32];
    __shared__ int s_last;
    const long long n = *n_ptr;
    const long long ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    // vector accesses when the arrays start on 16-byte boundaries (allocation bases do)
    const bool vec = ((reinterpret_cast<uintptr_t>(out) | reinterpret_cast<uintptr_t>(in) |
                       reinterpret_cast<uintptr_t>(act)) & 15u) == 0;
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(&counters[0], 1u);
        __syncthreads();
        const long long tile = s_tile;
        if (tile >= ntiles) break;
        const long long base = tile * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
        const bool full = base + SCAN_ITEMS <= n;   // a thread's 16 items as four (flags: one) 16-byte accesses
        uint32_t c8[SCAN_ITEMS];
        if (full && vec) {
            if (in) {
#pragma unroll
                for (int r = 0; r < SCAN_ITEMS / 4; ++r) {
                    const uint4 a = *reinterpret_cast<const uint4*>(in + base + 4 * r);
                    c8[4 * r] = a.x; c8[4 * r + 1] = a.y; c8[4 * r + 2] = a.z; c8[4 * r + 3] = a.w;
                }
            } else {
                const uint4 a = *reinterpret_cast<const uint4*>(act + base);
                const uint32_t wv[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
                for (int r = 0; r < 4; ++r)
#pragma unroll
                    for (int q = 0; q < 4; ++q) c8[4 * r + q] = ((wv[r] >> (8 * q)) & 0xffu) != 0;
            }
        } else {
#pragma unroll
            for (int q = 0; q < SCAN_ITEMS; ++q) {
                const long long i = base + q;
                c8[q] = i < n ? (in ? in[i] : (uint32_t)(act[i] != 0)) : 0u;
            }
        }
        uint32_t v[SCAN_ITEMS];
        uint32_t tsum = 0;
#pragma unroll
        for (int q = 0; q < SCAN_ITEMS; ++q) {
            v[q] = tsum;
            tsum += c8[q];
        }
        uint32_t incl = tsum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) s_warp[wid] = incl;
        __syncthreads();
        if (wid == 0) {   // the tile's total, its warps' offsets, and the look-back by warp 0
            uint32_t t[SCAN_BLOCK / 32], acc = 0;
#pragma unroll
            for (int q = 0; q < SCAN_BLOCK / 32; ++q) t[q] = s_warp[q];
            __syncwarp();
#pragma unroll
            for (int q = 0; q < SCAN_BLOCK / 32; ++q) {
                if (lane == 0) s_warp[q] = acc;
                acc += t[q];
            }
            bool ok;
            const uint32_t ex = tile_lookback_from_warp(tile_status, 0u, (uint32_t)tile, epoch, acc, status, &ok);
            if (lane == 0) {
                s_excl = ex;
                if (tile == ntiles - 1 && total) *total = (long long)ex + acc;
            }
        }
        __syncthreads();
        const uint32_t off = s_excl + s_warp[wid] + incl - tsum;
        if (full && vec) {
#pragma unroll
            for (int r = 0; r < SCAN_ITEMS / 4; ++r)
                *reinterpret_cast<uint4*>(out + base + 4 * r) =
                    make_uint4(off + v[4 * r], off + v[4 * r + 1], off + v[4 * r + 2], off + v[4 * r + 3]);
        } else {
#pragma unroll
            for (int q = 0; q < SCAN_ITEMS; ++q) {
                const long long i = base + q;
                if (i < n) out[i] = off + v[q];
            }
        }
        __syncthreads();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t d = atomicAdd(&counters[1], 1u);
        s_last = d == gridDim.x - 1;
    }
    __syncthreads();
    if (s_last && threadIdx.x == 0) {
        if (ntiles == 0 && total) *total = 0;
        counters[0] = 0;
        counters[1] = 0;
    }
}

int launch_scan(mcs_pop* p, const uint32_t* in, uint32_t* out, const long long* n_dev, long long* total) {
    mcs_ctx* c = p->ctx;
    const long long max_tiles = (p->cap + SCAN_TILE - 1) / SCAN_TILE;
    const int grid = persistent_grid(c, k_scan, SCAN_BLOCK, max_tiles);
    c->epoch += 1;
    if ((c->epoch & 0x3fffffffu) == 0) c->epoch += 1;
    k_scan<<<grid, SCAN_BLOCK, 0, c->stream>>>(in, p->act, out, n_dev, p->tile_status, p->counters + 2, c->epoch,
                                                 c->d_status, total);
    MCS_CK_LAUNCH(c);
    return MCS_OK;
}

// ---------------------------------------------------------------------------------------
// Generic slot copy of every population array (dst <- src).
// ---------------------------------------------------------------------------------------
struct RawPop {
    char* f[8];
    uint32_t* cell;
    uint8_t* act;
    int esz;
};

__device__ __forceinline__ void copy_slot(const RawPop& r, long long dst, long long src) {
    if (r.esz == 8) {
#pragma unroll
        for (int q = 0; q < 8; ++q) reinterpret_cast<double*>(r.f[q])[dst] = reinterpret_cast<const double*>(r.f[q])[src];
    } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) reinterpret_cast<float*>(r.f[q])[dst] = reinterpret_cast<const float*>(r.f[q])[src];
    }
    if (r.cell) r.cell[dst] = r.cell[src];
    r.act[dst] = r.act[src];
}

RawPop raw_pop(mcs_pop* p) {
    RawPop r;
    for (int q = 0; q < 8; ++q) r.f[q] = static_cast<char*>(p->f[q]);
    r.cell = p->cell;
    r.act = p->act;
    r.esz = (int)p->esz;
    return r;
}

// repack!: hole k (k-th inactive slot below A, ascending) receives the k-th active slot at
// or above A counted from the end, which is the pairing of the reference's two-pointer loop.
__global__ void k_repack_holes(const uint8_t* __restrict__ act, const uint32_t* __restrict__ pre,
                               const long long* A_ptr, uint32_t* __restrict__ holepos) {
    const long long A = *A_ptr;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < A; i += (long long)gridDim.x * blockDim.x)
        if (!act[i]) holepos[i - pre[i]] = (uint32_t)i;
}

__global__ void k_repack_move(RawPop r, const uint32_t* __restrict__ pre, const long long* n_ptr, const long long* A_ptr,
                              const uint32_t* __restrict__ holepos, long long* n_out) {
    const long long n = *n_ptr, A = *A_ptr;
    for (long long i = A + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (!r.act[i]) continue;
        const long long q = A - 1 - (long long)pre[i];
        copy_slot(r, holepos[q], i);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *n_out = A;
}

int grid_for(mcs_ctx* c, long long n, int block) {
    long long g = (n + block - 1) / block;
    const long long gmax = (long long)c->num_sms * 8;
    if (g > gmax) g = gmax;
    if (g < 1) g = 1;
    return (int)g;
}

int launch_repack(mcs_pop* p) {
    mcs_ctx* c = p->ctx;
    long long* A = reinterpret_cast<long long*>(p->counters + 4);
    int st = launch_scan(p, nullptr, p->u32b, p->d_n + p->cur, A);
    if (st) return st;
    const int g = grid_for(c, p->cap, 256);
    k_repack_holes<<<g, 256, 0, c->stream>>>(p->act, p->u32b, A, p->u32a);
    MCS_CK_LAUNCH(c);
    k_repack_move<<<g, 256, 0, c->stream>>>(raw_pop(p), p->u32b, p->d_n + p->cur, A, p->u32a, p->d_n + (p->cur ^ 1));
    MCS_CK_LAUNCH(c);
    p->cur ^= 1;
    return MCS_OK;
}

// ---------------------------------------------------------------------------------------
// Swarm.resample!(popl, n0, tol): Swarm/src/Swarm.jl:193-223.
// ---------------------------------------------------------------------------------------
__global__ void k_sres_count(uint8_t* __restrict__ act, const long long* n_ptr, const long long* ncur_ptr, long long n0,
                             double tol, unsigned long long seed, uint32_t step, uint32_t* __restrict__ counts) {
    const long long n = *n_ptr, ncur = *ncur_ptr;
    const bool skip = ncur == 0 || fabs((double)(ncur - n0) / (double)n0) < tol;
    const bool drop = ncur > n0;
    const double pdrop = (double)(ncur - n0) / (double)ncur;
    const double lam = (double)(n0 - ncur) / (double)ncur;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        uint32_t c = 0;
        if (!skip && act[i]) {
            Rng r;
            r.init(seed, (uint32_t)i, step, TAG_SWARM_RESAMPLE);
            if (drop) {
                if (r.u64() < pdrop) act[i] = 0;
            } else {
                c = (uint32_t)poisson_draw(r, lam);
            }
        }
        counts[i] = c;
    }
}

__global__ void k_sres_write(RawPop r, const long long* n_ptr, const uint32_t* __restrict__ counts,
                             const uint32_t* __restrict__ off, const long long* total_ptr, long long cap,
                             long long* n_out, uint32_t* status) {
    const long long n = *n_ptr;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const uint32_t c = counts[i];
        for (uint32_t j = 0; j < c; ++j) {
            const long long d = n + (long long)off[i] + j;
            if (d >= cap) { atomicOr(status, ST_CAPACITY); break; }
            copy_slot(r, d, i);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        long long m = n + *total_ptr;
        if (m > cap) m = cap;
        *n_out = m;
    }
}

int launch_swarm_resample(mcs_pop* p, long long n0, double tol) {
    mcs_ctx* c = p->ctx;
    long long* ncur = reinterpret_cast<long long*>(p->counters + 4);
    long long* total = reinterpret_cast<long long*>(p->counters + 6);
    int st = launch_scan(p, nullptr, p->u32b, p->d_n + p->cur, ncur);  // nactives
    if (st) return st;
    const int g = grid_for(c, p->cap, 256);
    k_sres_count<<<g, 256, 0, c->stream>>>(p->act, p->d_n + p->cur, ncur, n0, tol, p->seed, p->step, p->u32a);
    MCS_CK_LAUNCH(c);
    st = launch_scan(p, p->u32a, p->u32b, p->d_n + p->cur, total);
    if (st) return st;
    k_sres_write<<<g, 256, 0, c->stream>>>(raw_pop(p), p->d_n + p->cur, p->u32a, p->u32b, total, p->cap,
                                           p->d_n + (p->cur ^ 1), c->d_status);
    MCS_CK_LAUNCH(c);
    p->cur ^= 1;
    return MCS_OK;
}

// ---------------------------------------------------------------------------------------
// Moments (layout MCS_M_*): per-block partials in fixed order, then a fixed-order finish.
// ---------------------------------------------------------------------------------------
constexpr int MOM_BLOCK = 256;
constexpr int MOM_MAX = MCS_MOMENTS_BASE + kMaxRows;

template <typename T>
__global__ void __launch_bounds__(MOM_BLOCK) k_moments(PopView<T> P, GridView g, int mesh, TableView tab, int use_tab,
                                                       int nm, double* __restrict__ partials) {
    __shared__ double red[MOM_BLOCK / 32][MOM_MAX];
    const long long n = *P.n_in;
    double acc[MOM_MAX];
    for (int q = 0; q < MOM_MAX; ++q) acc[q] = 0.0;
    acc[MCS_M_EMAX] = -INFINITY;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double vx = P.f[3][i], vy = P.f[4][i], vz = P.f[5][i];
        const double eng = 0.5 * kElectronMass * (vx * vx + vy * vy + vz * vz);
        acc[MCS_M_EMAX] = fmax(acc[MCS_M_EMAX], eng);
        if (!P.act[i]) continue;
        double x, y, z;
        abs_position(P, g, mesh, i, x, y, z);
        const double w = P.f[6][i];
        acc[MCS_M_COUNT] += 1.0;
        acc[MCS_M_W] += w;
        acc[MCS_M_X] += x; acc[MCS_M_X + 1] += y; acc[MCS_M_X + 2] += z;
        acc[MCS_M_X2] += x * x; acc[MCS_M_X2 + 1] += y * y; acc[MCS_M_X2 + 2] += z * z;
        acc[MCS_M_V] += vx; acc[MCS_M_V + 1] += vy; acc[MCS_M_V + 2] += vz;
        acc[MCS_M_E] += eng;
        acc[MCS_M_WE] += w * eng;
        acc[MCS_M_WX] += w * x; acc[MCS_M_WX + 1] += w * y; acc[MCS_M_WX + 2] += w * z;
        acc[MCS_M_WX2] += w * (x * x + y * y + z * z);
        if (use_tab) {
            const double u = (eng - tab.e0) / tab.step;
            double fk = floor(u);
            if (__fma_rn(fk, tab.step, -(eng - tab.e0)) > 0.0) fk -= 1.0;
            long long k;
            double wk;
            if (!(fk >= 0.0 && fk <= (double)(tab.neps - 2))) {
                const bool low = !(fk >= 0.0);
                k = low ? 0 : tab.neps - 2;
                wk = low ? 1.0 : 0.0;
            } else {
                k = (long long)fk;
                const double tt = (double)(k + 1) / (double)(tab.neps - 1);
                wk = (((1.0 - tt) * tab.e0 + tt * tab.emax) - eng) / tab.step;
            }
            for (int j = 0; j < tab.nrows; ++j)
                acc[MCS_MOMENTS_BASE + j] +=
                    wk * tab.rate64[k * tab.nrows + j] + (1.0 - wk) * tab.rate64[(k + 1) * tab.nrows + j];
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int q = 0; q < nm; ++q) {
        const double v = q == MCS_M_EMAX ? warp_max(acc[q]) : warp_sum(acc[q]);
        if (lane == 0) red[wid][q] = v;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nm; q += MOM_BLOCK) {
        double a = q == MCS_M_EMAX ? -INFINITY : 0.0;
        for (int wv = 0; wv < MOM_BLOCK / 32; ++wv) a = q == MCS_M_EMAX ? fmax(a, red[wv][q]) : a + red[wv][q];
        partials[(long long)blockIdx.x * nm + q] = a;
    }
}

__global__ void k_moments_finish(const double* __restrict__ partials, int nblocks, int nm, double* __restrict__ out) {
    for (int q = threadIdx.x; q < nm; q += blockDim.x) {
        double a = q == MCS_M_EMAX ? -INFINITY : 0.0, comp = 0.0;
        for (int b = 0; b < nblocks; ++b) {
            const double v = partials[(long long)b * nm + q];
            if (q == MCS_M_EMAX) { a = fmax(a, v); continue; }
            const double y = v - comp, s = a + y;
            comp = (s - a) - y;
            a = s;
        }
        out[q] = a;
    }
}

template <typename T>
int launch_moments_t(mcs_pop* p, const mcs_table* t, double* d_out, int nm) {
    mcs_ctx* c = p->ctx;
    int g = c->num_sms * 2;
    const long long need = (p->cap + MOM_BLOCK - 1) / MOM_BLOCK;
    if (g > need) g = (int)need;
    if (g > kMomentPartialsMin / nm) g = kMomentPartialsMin / nm;  // partials buffer bound
    if (g < 1) g = 1;
    double* partials = p->tile_partials;  // >= num_sms*2*MOM_MAX doubles, see pop create
    const GridView gv = grid_view(p->cells);
    TableView tv{};
    if (t) tv = t->v;
    k_moments<T><<<g, MOM_BLOCK, 0, c->stream>>>(pop_view<T>(p), gv, p->cells != nullptr, tv, t != nullptr, nm, partials);
    MCS_CK_LAUNCH(c);
    k_moments_finish<<<1, 64, 0, c->stream>>>(partials, g, nm, d_out);
    MCS_CK_LAUNCH(c);
    return MCS_OK;
}

int launch_moments(mcs_pop* p, const mcs_table* t, double* d_out, int nm) {
    return p->precision == MCS_FP32 ? launch_moments_t<float>(p, t, d_out, nm) : launch_moments_t<double>(p, t, d_out, nm);
}

// ---------------------------------------------------------------------------------------
// density!: MCStreamer/src/poisson.jl:65-84.  3-D mesh: CIC int64; cylinder: NGP int64 of
// w*val (density = q*2^-32/dV on read).
// ---------------------------------------------------------------------------------------
template <typename T>
__global__ void k_deposit(PopView<T> P, GridView g, int mesh, double val, long long* __restrict__ q,
                          uint32_t* status) {
    const long long n = *P.n_in;
    const long long stride = (long long)gridDim.x * blockDim.x;
    if (mesh) {
        // warp-uniform trip count: every lane takes part in the aggregated deposit
        for (long long i0 = (long long)blockIdx.x * blockDim.x; i0 < n; i0 += stride) {
            const long long i = i0 + threadIdx.x;
            bool valid = false;
            uint32_t cidx = kOutside;
            int ix = 0, iy = 0, iz = 0;
            double fx = 0.0, fy = 0.0, fz = 0.0, charge = 0.0;
            if (i < n && P.act[i]) {
                cidx = P.cell[i];
                if (cidx != kOutside) {
                    valid = true;
                    uint32_t ux, uy, uz;
                    cell_split(g, cidx, ux, uy, uz);
                    ix = (int)ux;
                    iy = (int)uy;
                    iz = (int)uz;
                    fx = (double)P.f[0][i]; fy = (double)P.f[1][i]; fz = (double)P.f[2][i];
                    charge = (double)P.f[6][i] * val;
                }
            }
            cic_fixed_warp(q, g.nx, g.ny, valid, cidx, ix, iy, iz, fx, fy, fz, charge, status);
        }
        return;
    }
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) {
        if (!P.act[i]) continue;
        const double charge = (double)P.f[6][i] * val;
        if (g.type == GRID_CART3D) {
            int ix, iy, iz;
            double fx, fy, fz;
            if (cart_locate(g, P.f[0][i], P.f[1][i], P.f[2][i], ix, iy, iz, fx, fy, fz))
                cic_fixed(q, g.nx, g.ny, ix, iy, iz, fx, fy, fz, charge, status);
        } else {
            cyl_track(g, q, P.f[0][i], P.f[1][i], P.f[2][i], charge, status);
        }
    }
}

int launch_deposit(mcs_pop* p, mcs_grid* g, double val) {
    mcs_ctx* c = p->ctx;
    const int gr = grid_for(c, p->cap, 256);
    const int mesh = p->cells != nullptr;
    if (p->precision == MCS_FP32)
        k_deposit<float><<<gr, 256, 0, c->stream>>>(pop_view<float>(p), g->v, mesh, val, g->d_q[MCS_Q_PART],
                                                     c->d_status);
    else
        k_deposit<double><<<gr, 256, 0, c->stream>>>(pop_view<double>(p), g->v, mesh, val, g->d_q[MCS_Q_PART],
                                                      c->d_status);
    MCS_CK_LAUNCH(c);
    return MCS_OK;
}

// ---------------------------------------------------------------------------------------
int launch_upload(mcs_pop* p, const double* dx, const double* dv, const double* dw, const double* ds, const uint8_t* da,
                  long long n, unsigned int* w_lossy) {
    mcs_ctx* c = p->ctx;
    const int gr = grid_for(c, n, 256);
    const GridView gv = grid_view(p->cells);
    const int mesh = p->cells != nullptr;
    if (p->precision == MCS_FP32)
        k_upload<float><<<gr, 256, 0, c->stream>>>(dx, dv, dw, ds, da, n, pop_view<float>(p), gv, mesh, w_lossy);
    else
        k_upload<double><<<gr, 256, 0, c->stream>>>(dx, dv, dw, ds, da, n, pop_view<double>(p), gv, mesh, w_lossy);
    MCS_CK_LAUNCH(c);
    return MCS_OK;
}

int launch_download(mcs_pop* p, double* dx, double* dv, double* dw, double* ds, uint8_t* da) {
    mcs_ctx* c = p->ctx;
    const int gr = grid_for(c, p->cap, 256);
    const GridView gv = grid_view(p->cells);
    const int mesh = p->cells != nullptr;
    if (p->precision == MCS_FP32)
        k_download<float><<<gr, 256, 0, c->stream>>>(dx, dv, dw, ds, da, pop_view<float>(p), gv, mesh);
    else
        k_download<double><<<gr, 256, 0, c->stream>>>(dx, dv, dw, ds, da, pop_view<double>(p), gv, mesh);
    MCS_CK_LAUNCH(c);
    return MCS_OK;
}

}  // namespace mcs
