// fluid.cu -- MCStreamer's electron fluid (MCStreamer/src/fluid.jl) on the device: the
// needle initial condition setneedle!, the Neumann ghosts setnebc!, the Koren-limited upwind
// flux divergence setdne! and the explicit update euler!, over the fields poisson! leaves on
// the grid's faces.  poisson!'s charge subtracts the fluid density (poisson.jl:24), which
// mcs_poisson_assemble reads from here.
//
// Compiled with -fmad=false: every flux and every accumulation is evaluated unfused in the
// reference's order, so the kernels reproduce the serial loops bit for bit.
//
// Layout: ne, dne are column-major (M+4)x(N+4), element (i, j), i in -1..M+2, j in -1..N+2,
// at (i+1) + (j+1)(M+4) (calloc_centers with two ghost layers).  The faces er, ez are the
// grid's (M+3)x(N+3) arrays (calloc_faces).
//
// One thread per padded cell.  setnebc! copies each ghost from the nearest interior cell
// (whole rows first, then whole columns: every ghost, corners included, ends as the value of
// the clamped interior index), so a flux reads ne at clamped indices and the ghosts are
// written by their own threads, never read.  A cell (i, j) assembles
//   dne = (((0 + Fz(i,j)/dz) - Fz(i,j+1)/dz) + Fr(i,j)/dr) - Fr(i+1,j)/dr,
// the order in which the reference's face loops add into it (z faces first, then r faces,
// ascending); the first ghost layer receives the boundary faces' single terms.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <new>

#include "../../include/mcs.h"
#include "host_util.h"
#include "mcs_internal.h"

namespace mcs {
namespace {

constexpr int BX = 64, BY = 8;

struct FluidArgs {
    const double* ne;   // read (interior only)
    double* ghost_out;  // receives the ghost values (ne itself, or the next buffer)
    double* ne_out;     // interior update ne + dt dne (STEP only)
    double* dne;
    const double* er;
    const double* ez;
    int M, N;
    double dr, dz, mob, dt;
};

__device__ __forceinline__ double koren(double theta) {   // fluid.jl:107-112
    if (theta >= 4.0) return 1.0;
    if (theta > 0.4) return 1.0 / 3.0 + theta / 6.0;
    if (theta > 0.0) return theta;
    return 0.0;
}

// The limiter of a nonzero slope ratio a / b and the quotient F / h live out of line: a
// call is a branch the compiler cannot turn into predicated code, so a face whose slope and
// flux are zero (most faces outside the fluid) executes no division.
__device__ __noinline__ double limiter(double a, double b) {
    if (b == 0.0 && !isnan(a)) return signbit(a) == signbit(b) ? 1.0 : 0.0;   // a / +-0 = +-inf
    return koren(a / b);
}

__device__ __noinline__ double quotient(double F, double h) { return F / h; }

// The flux F(n_u2, n_u, n_d) = v (n_u + koren((n_u - n_u2) / (n_d - n_u)) (n_d - n_u))
// (fluid.jl:57-64 and 75-82), over the cell size h > 0.  A zero slope a gives a ratio of
// +-0 or NaN (limiter 0), and a zero F over h keeps its sign: neither needs the division.
__device__ __forceinline__ double face_term(double v, double nu2, double nu, double nd, double h) {
    const double b = nd - nu, a = nu - nu2;
    const double k = a != 0.0 ? limiter(a, b) : 0.0;
    const double F = v * (nu + k * b);
    return F == 0.0 ? F : quotient(F, h);
}

// The upwind triple of a face between cells lo and hi = lo + 1 along one axis, from the
// densities of cells lo-1, lo, hi, hi+1: v >= 0 flows lo -> hi (upstream lo, twice-upstream
// lo-1, downstream hi), v < 0 (signbit, -0 included) the other way.
__device__ __forceinline__ double face(double v, double m1, double lo, double hi, double p1, double h) {
    const bool neg = signbit(v);
    return face_term(v, neg ? p1 : m1, neg ? hi : lo, neg ? lo : hi, h);
}

constexpr int HX = BX + 4, HY = BY + 4;   // ne tile with two cells of halo on each side

// setnebc! + setdne! (+ euler! into ne_out when STEP).  A BX x BY tile of cells stages ne
// over its cells and two on each side in shared memory, read at clamped indices (the values
// setnebc! gives the ghosts).  Every face is computed once, by the thread of the cell above
// it (z faces) or right of it (r faces); the tile's top row and right column also compute
// the faces beyond them, and each cell reads its four face terms from shared memory.
template <bool STEP>
__global__ void __launch_bounds__(BX * BY, 4) k_fluid(FluidArgs a) {
    __shared__ double sn[HY][HX];        // ne at (i0 - 2 + x, j0 - 2 + y) (tile indices, clamped)
    __shared__ double sz[BY + 1][BX];    // z face terms F/dz of faces j .. j+BY
    __shared__ double sr[BY][BX + 1];    // r face terms F/dr of faces i .. i+BX
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i0 = blockIdx.x * BX - 1, j0 = blockIdx.y * BY - 1;   // reference indices of the tile's corner
    const int ld = a.M + 4;
    const int i = i0 + tx, j = j0 + ty;
    const bool live = i + 1 < a.M + 4 && j + 1 < a.N + 4;
    const bool zrow = i >= 1 && i <= a.M, rrow = j >= 1 && j <= a.N;
    const int fl = a.M + 3;
    double vz = 0.0, vz1 = 0.0, vr = 0.0, vr1 = 0.0;
    const bool fz = live && zrow && j >= 1 && j <= a.N + 1;
    const bool fz1 = live && ty == BY - 1 && zrow && j + 1 <= a.N + 1 && j + 1 >= 1;
    const bool fr = live && rrow && i >= 1 && i <= a.M + 1;
    const bool fr1 = live && tx == BX - 1 && rrow && i + 1 <= a.M + 1 && i + 1 >= 1;
    if (fz) vz = -a.ez[i + j * fl] * a.mob;
    if (fz1) vz1 = -a.ez[i + (j + 1) * fl] * a.mob;
    if (fr) vr = -a.er[i + j * fl] * a.mob;
    if (fr1) vr1 = -a.er[(i + 1) + j * fl] * a.mob;
    // the staged tile: both passes' loads issued before either store
    {
        constexpr int T = BX * BY, NS = (HX * HY + T - 1) / T;
        double val[NS];
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            const int t = ty * BX + tx + q * T;
            if (t < HX * HY) {
                const int y = t / HX, x = t - y * HX;
                const int ic = min(max(i0 - 2 + x, 1), a.M), jc = min(max(j0 - 2 + y, 1), a.N);
                val[q] = a.ne[(ic + 1) + (jc + 1) * ld];
            }
        }
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            const int t = ty * BX + tx + q * T;
            if (t < HX * HY) sn[t / HX][t % HX] = val[q];
        }
    }
    __syncthreads();
    const int x = tx + 2, y = ty + 2;   // this cell in the staged tile
    // z face j lies between cells j-1 and j, r face i between cells i-1 and i.
    if (fz) sz[ty][tx] = face(vz, sn[y - 2][x], sn[y - 1][x], sn[y][x], sn[y + 1][x], a.dz);
    if (fz1) sz[BY][tx] = face(vz1, sn[y - 1][x], sn[y][x], sn[y + 1][x], sn[y + 2][x], a.dz);
    if (fr) sr[ty][tx] = face(vr, sn[y][x - 2], sn[y][x - 1], sn[y][x], sn[y][x + 1], a.dr);
    if (fr1) sr[ty][BX] = face(vr1, sn[y][x - 1], sn[y][x], sn[y][x + 1], sn[y][x + 2], a.dr);
    __syncthreads();
    if (!live) return;
    const int k = (i + 1) + (j + 1) * ld;
    double d = 0.0;
    if (zrow && rrow) {
        d += sz[ty][tx];
        d -= sz[ty + 1][tx];
        d += sr[ty][tx];
        d -= sr[ty][tx + 1];
        if (STEP) a.ne_out[k] = sn[y][x] + a.dt * d;
    } else {
        if (zrow && j == 0) d -= sz[ty + 1][tx];
        else if (zrow && j == a.N + 1) d += sz[ty][tx];
        else if (rrow && i == 0) d -= sr[ty][tx + 1];
        else if (rrow && i == a.M + 1) d += sr[ty][tx];
        a.ghost_out[k] = sn[y][x];
    }
    a.dne[k] = d;
}

// euler!: fluid.jl:100-111.
__global__ void __launch_bounds__(BX * BY) k_euler(double* ne, const double* dne, int M, int N, double dt) {
    const int i = blockIdx.x * BX + threadIdx.x + 1;
    if (i > M) return;
    for (int j = blockIdx.y * BY + threadIdx.y + 1; j <= N; j += gridDim.y * BY) {
        const long k = (long)(i + 1) + (long)(j + 1) * (M + 4);
        ne[k] += dt * dne[k];
    }
}

// setneedle!: fluid.jl:3-13, cell centres rc = (i - 1/2) dr, zc = (j - 1/2) dz.
__global__ void __launch_bounds__(BX * BY) k_needle(double* ne, double* qfd, int M, int N, double dr, double dz,
                                                   double sigma_z, double sigma_r, double position_z, double ne0) {
    const int i = blockIdx.x * BX + threadIdx.x + 1;
    if (i > M) return;
    for (int j = blockIdx.y * BY + threadIdx.y + 1; j <= N; j += gridDim.y * BY) {
        const long k = (long)(i + 1) + (long)(j + 1) * (M + 4);
        const double rc = ((double)(i - 1) + 0.5) * dr;
        const double zc = ((double)(j - 1) + 0.5) * dz;
        const double dzp = zc - position_z;
        const double z1 = dzp > 0.0 ? dzp : 0.0;
        const double e = -(rc * rc) / (sigma_r * sigma_r) - (z1 * z1) / (sigma_z * sigma_z);
        const double v = ne[k] + ne0 * exp(e);
        ne[k] = v;
        const long q = (long)i + (long)j * (M + 2);
        qfd[q] = qfd[q] + v;
    }
}

dim3 fluid_grid(const mcs_fluid* f, int rows) {
    const int gx = (f->M + 4 + BX - 1) / BX;
    const long want = ((long)rows + BY - 1) / BY;
    const long cap = std::max(1L, (long)f->ctx->num_sms * 16 / gx);
    return dim3(gx, (unsigned)std::max(1L, std::min(want, std::min(cap, 65535L))));
}

// One thread per padded cell, no row loop (k_fluid shares faces within a tile).
dim3 tile_grid(const mcs_fluid* f) {
    return dim3((f->M + 4 + BX - 1) / BX, (f->N + 4 + BY - 1) / BY);
}

int falloc(mcs_ctx* c, double** p, size_t count) {
    if (cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(count, 1) * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return set_err(c, MCS_ERR_NOMEM, "fluid: device allocation failed");
    }
    return MCS_OK;
}

size_t padded(const mcs_fluid* f) { return (size_t)(f->M + 4) * (f->N + 4); }

int use(mcs_fluid* f) {
    if (!f->g) return set_err(f->ctx, MCS_ERR_ARG, "fluid: its grid was destroyed");
    MCS_CK(f->ctx, cudaSetDevice(f->ctx->device));
    return MCS_OK;
}

FluidArgs args(mcs_fluid* f, double mob, double dt) {
    FluidArgs a{};
    a.ne = f->ne[f->cur];
    a.dne = f->dne;
    a.er = f->g->d_er;
    a.ez = f->g->d_ez;
    a.M = f->M;
    a.N = f->N;
    a.dr = f->g->v.dr;
    a.dz = f->g->v.dz;
    a.mob = mob;
    a.dt = dt;
    return a;
}

}  // namespace

double* grid_qfd(mcs_grid* g) {
    if (g->d_qfd) return g->d_qfd;
    const size_t n = (size_t)(g->v.M + 2) * (g->v.N + 2);
    if (falloc(g->ctx, &g->d_qfd, n)) return nullptr;
    if (cudaMemsetAsync(g->d_qfd, 0, n * sizeof(double), g->ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(g->ctx->stream) != cudaSuccess) {
        cudaFree(g->d_qfd);
        g->d_qfd = nullptr;
        set_err(g->ctx, MCS_ERR_CUDA, "qfixed density: device initialisation failed");
        return nullptr;
    }
    return g->d_qfd;
}

}  // namespace mcs

using namespace mcs;

extern "C" {

MCS_API int mcs_fluid_create(mcs_grid* g, mcs_fluid** out) {
    if (!g || !out) return MCS_ERR_ARG;
    mcs_ctx* c = g->ctx;
    if (g->v.type != GRID_CYL) return set_err(c, MCS_ERR_ARG, "fluid: needs a cylindrical grid");
    if (g->fluid) return set_err(c, MCS_ERR_ARG, "fluid: the grid has a fluid already");
    if ((long)(g->v.M + 4) * (g->v.N + 4) >= (1L << 31) || (g->v.N + 4 + BY - 1) / BY > 65535)
        return set_err(c, MCS_ERR_ARG, "fluid: grid above 2^31 cells or N above 524,000");
    MCS_CK(c, cudaSetDevice(c->device));
    mcs_fluid* f = new (std::nothrow) mcs_fluid();
    if (!f) return MCS_ERR_NOMEM;
    f->ctx = c;
    f->g = g;
    f->M = g->v.M;
    f->N = g->v.N;
    const size_t n = padded(f);
    int st = falloc(c, &f->ne[0], n);
    if (!st) st = falloc(c, &f->ne[1], n);
    if (!st) st = falloc(c, &f->dne, n);
    if (!st && !grid_qfd(g)) st = MCS_ERR_NOMEM;
    if (st) {
        cudaFree(f->ne[0]); cudaFree(f->ne[1]); cudaFree(f->dne);
        delete f;
        return st;
    }
    cudaMemsetAsync(f->ne[0], 0, n * sizeof(double), c->stream);
    cudaMemsetAsync(f->ne[1], 0, n * sizeof(double), c->stream);
    cudaMemsetAsync(f->dne, 0, n * sizeof(double), c->stream);
    MCS_CK(c, cudaStreamSynchronize(c->stream));
    g->fluid = f;
    *out = f;
    return MCS_OK;
}

MCS_API int mcs_fluid_destroy(mcs_fluid* f) {
    if (!f) return MCS_OK;
    cudaSetDevice(f->ctx->device);
    cudaStreamSynchronize(f->ctx->stream);
    if (f->g && f->g->fluid == f) f->g->fluid = nullptr;
    cudaFree(f->ne[0]); cudaFree(f->ne[1]); cudaFree(f->dne);
    delete f;
    return MCS_OK;
}

MCS_API int mcs_fluid_upload(mcs_fluid* f, const double* ne, const double* qfd) {
    if (!f) return MCS_ERR_ARG;
    if (int e = use(f)) return e;
    mcs_ctx* c = f->ctx;
    if (ne)
        MCS_CK(c, cudaMemcpyAsync(f->ne[f->cur], ne, padded(f) * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    if (qfd)
        MCS_CK(c, cudaMemcpyAsync(f->g->d_qfd, qfd, (size_t)(f->M + 2) * (f->N + 2) * sizeof(double),
                                  cudaMemcpyHostToDevice, c->stream));
    MCS_CK(c, cudaStreamSynchronize(c->stream));
    return MCS_OK;
}

MCS_API int mcs_fluid_download(mcs_fluid* f, double* ne, double* dne, double* qfd) {
    if (!f) return MCS_ERR_ARG;
    if (int e = use(f)) return e;
    mcs_ctx* c = f->ctx;
    if (ne)
        MCS_CK(c, cudaMemcpyAsync(ne, f->ne[f->cur], padded(f) * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (dne) MCS_CK(c, cudaMemcpyAsync(dne, f->dne, padded(f) * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (qfd)
        MCS_CK(c, cudaMemcpyAsync(qfd, f->g->d_qfd, (size_t)(f->M + 2) * (f->N + 2) * sizeof(double),
                                  cudaMemcpyDeviceToHost, c->stream));
    MCS_CK(c, cudaStreamSynchronize(c->stream));
    return MCS_OK;
}

MCS_API int mcs_fluid_set_needle(mcs_fluid* f, double sigma_z, double sigma_r, double position_z, double position_r,
                                 double ne0) {
    if (!f) return MCS_ERR_ARG;
    (void)position_r;   // taken and unused by setneedle!
    if (int e = use(f)) return e;
    ++f->launches;
    k_needle<<<fluid_grid(f, f->N), dim3(BX, BY), 0, f->ctx->stream>>>(f->ne[f->cur], f->g->d_qfd, f->M, f->N,
                                                                        f->g->v.dr, f->g->v.dz, sigma_z, sigma_r,
                                                                        position_z, ne0);
    MCS_CK(f->ctx, cudaGetLastError());
    return MCS_OK;
}

MCS_API int mcs_fluid_derivatives(mcs_fluid* f, double mobility) {
    if (!f) return MCS_ERR_ARG;
    if (int e = use(f)) return e;
    FluidArgs a = args(f, mobility, 0.0);
    a.ghost_out = f->ne[f->cur];
    ++f->launches;
    k_fluid<false><<<tile_grid(f), dim3(BX, BY), 0, f->ctx->stream>>>(a);
    MCS_CK(f->ctx, cudaGetLastError());
    return MCS_OK;
}

MCS_API int mcs_fluid_euler(mcs_fluid* f, double dt) {
    if (!f) return MCS_ERR_ARG;
    if (int e = use(f)) return e;
    ++f->launches;
    k_euler<<<fluid_grid(f, f->N), dim3(BX, BY), 0, f->ctx->stream>>>(f->ne[f->cur], f->dne, f->M, f->N, dt);
    MCS_CK(f->ctx, cudaGetLastError());
    return MCS_OK;
}

MCS_API int mcs_fluid_step(mcs_fluid* f, double mobility, double dt) {
    if (!f) return MCS_ERR_ARG;
    if (int e = use(f)) return e;
    FluidArgs a = args(f, mobility, dt);
    a.ne_out = f->ne[f->cur ^ 1];
    a.ghost_out = a.ne_out;
    ++f->launches;
    k_fluid<true><<<tile_grid(f), dim3(BX, BY), 0, f->ctx->stream>>>(a);
    MCS_CK(f->ctx, cudaGetLastError());
    f->cur ^= 1;
    return MCS_OK;
}

MCS_API int mcs_fluid_launches(mcs_fluid* f, int64_t* count) {
    if (!f || !count) return MCS_ERR_ARG;
    *count = f->launches;
    return MCS_OK;
}

}  // extern "C"
