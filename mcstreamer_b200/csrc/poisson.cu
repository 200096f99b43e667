// poisson.cu -- the electrostatic solve of MCStreamer's poisson! (MCStreamer/src/poisson.jl:
// 6-58) on the device: charge assembly from the int64 cell deposits, the cylindrical
// multigrid of Multigrid/src/Multigrid.jl with MCStreamer's configuration (main.jl:131-144),
// the free boundary condition of freebc.jl:4-36 and the face fields the push gathers.
//
// Compiled with -fmad=false: every operation is evaluated unfused and in the reference's
// order, so a kernel reproduces the FP64 restatement bit for bit; only the coarsest direct
// solve (an explicit inverse here), the residual norm and the sine transforms round
// differently.
//
// Layout: every level is a column-major (M+2)x(N+2) FP64 array, r fastest, ghosts at
// i = 0, M+1 and j = 0, N+1 (element (i, j) at i + j*(M+2)).  Level l has M >> l by N >> l
// cells.  Levels of at most kSmallCells cells run inside one CTA (their kernels would be
// launch-bound); the rest run one grid-wide kernel per operation.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/mcs.h"
#include "host_util.h"
#include "mcs_device.cuh"
#include "mcs_internal.h"
#include "pop_ops.h"

namespace mcs {
namespace {

constexpr int kMaxLevels = 16;
constexpr long kSmallCells = 32768;
constexpr long kTailSmemBytes = 200 * 1024;   // shared memory of the one-CTA tail
constexpr int kCtaThreads = 1024;
constexpr int kThreads = 256;
constexpr int kCoarsestSweeps = 50;   // mgv! at level == levels (Multigrid.jl:340-346)
constexpr int kMaxCoarse = 4096;      // cells of the coarsest level (dense inverse)
constexpr double kElementaryCharge = 1.6021766208e-19;
constexpr double kEpsilon0 = 8.854187817620389e-12;

struct LevelView {
    int M, N;
    double* res;    // right-hand side of this level (ws.res)
    double* res1;   // residual of the V-cycle (ws.res1)
    double* sol;    // solution / correction (ws.sol)
    const double* fp;   // connector factor toward +r, per row 0..M+1
    const double* fm;   // toward -r
};

struct MgView {
    int levels, smooth1, smooth2, small;
    int nc;
    const double* ainv;   // inverse of the coarsest Cartesian matrix, nc x nc row-major
    LevelView lv[kMaxLevels + 1];
};

// ---------------------------------------------------------------------------------------
// Operations over an index range [t0, n) with stride dt, so that one body serves the
// grid-wide kernels (t0 = global thread, dt = grid threads) and the one-CTA kernels.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ double dneg(double v) { return -v + 0.0; }   // coef -1, cons 0

// apply! (boundaries.jl:119-133) for bc = ((Left, Dirichlet), (Right, Dirichlet),
// (Top, Dirichlet), (Bottom, Neumann)).  Left/Right fill the inner rows; Top/Bottom then
// fill every column, so the corners take Top/Bottom of the Left/Right ghosts.  No thread
// reads a value that another one writes.
__device__ __forceinline__ void bc_range(double* a, int M, int N, int t0, int dt) {
    const long ld = M + 2;
    const int n = max(M + 1, N + 2);
    for (int t = t0; t < n; t += dt) {
        if (t >= 1 && t <= M) {
            a[t] = dneg(a[t + ld]);
            a[t + (N + 1) * ld] = dneg(a[t + N * ld]);
        }
        if (t <= N + 1) {
            double vt, vb;
            if (t == 0) {
                vt = dneg(a[M + ld]);
                vb = dneg(a[1 + ld]);
            } else if (t == N + 1) {
                vt = dneg(a[M + N * ld]);
                vb = dneg(a[1 + N * ld]);
            } else {
                vt = a[M + t * ld];
                vb = a[1 + t * ld];
            }
            a[M + 1 + t * ld] = dneg(vt);
            a[t * ld] = vb + 0.0;
        }
    }
}

// laplacian (Multigrid.jl:152-158) with CylindricalConnector{1}; stencil order +r, +z,
// -r, -z; neighbours addressed linearly like the reference's column-major arrays.
__device__ __forceinline__ double lap5(const double* u, long k, long ld, double fp, double fm) {
    double s = -4.0 * u[k];
    s += u[k + 1] * fp;
    s += u[k + ld];
    s += u[k - 1] * fm;
    s += u[k - ld];
    return s;
}

// One pass of gauss_seidel! (Multigrid.jl:168-178, redblack.jl:38-46): in column j the
// rows 1, 3, ... <= M shifted by parity xor (j even).  An odd M (possible on the coarsest
// level only) shifts into the ghost row M+1, which the reference updates too.
__device__ __forceinline__ void gs_range(double* u, const double* b, const double* fp, const double* fm, int M, int N,
                         int parity, int t0, int dt) {
    const long ld = M + 2;
    const int hm = (M + 1) >> 1;
    const int n = hm * N;
    for (int t = t0; t < n; t += dt) {
        const int j = 1 + t / hm;
        const int i = 1 + 2 * (t - (j - 1) * hm) + (parity ^ ((j & 1) == 0 ? 1 : 0));
        const long k = i + j * ld;
        const double l = lap5(u, k, ld, fp[i], fm[i]);
        u[k] += 1.0 * (l + b[k]) / 4.0;
    }
}

// residual! (Multigrid.jl:186-193): r = s b + L u on the inner cells.
__device__ __forceinline__ void residual_range(double* r, const double* u, const double* b, double s, const double* fp,
                               const double* fm, int M, int N, int t0, int dt) {
    const long ld = M + 2;
    const int n = M * N;
    for (int t = t0; t < n; t += dt) {
        const int j = 1 + t / M;
        const int i = 1 + (t - (j - 1) * M);
        const long k = i + j * ld;
        r[k] = s * b[k] + lap5(u, k, ld, fp[i], fm[i]);
    }
}

// restrict! (Multigrid.jl:213-226): coarse (I, J) = 4 * (sum of the children in the order
// (0,0), (0,1), (1,0), (1,1)) / 4.  M, N are the coarse sizes.
__device__ __forceinline__ void restrict_range(double* h, const double* f, int M, int N, int t0, int dt) {
    const long ldh = M + 2, ldf = 2 * M + 2;
    const int n = M * N;
    for (int t = t0; t < n; t += dt) {
        const int J = 1 + t / M;
        const int I = 1 + (t - (J - 1) * M);
        const long k = (2 * I - 1) + (2 * J - 1) * ldf;
        double s = 0.0;
        s += f[k];
        s += f[k + ldf];
        s += f[k + 1];
        s += f[k + 1 + ldf];
        h[I + J * ldh] = 4.0 * s / 4.0;
    }
}

// interpolate! (Multigrid.jl:232-258): fine child s of (I, J) = sum over sh of w(sh) *
// coarse[(I, J) + (2s - 1) .* sh], w = 9/16, 3/16, 3/16, 1/16; added or stored.
__device__ __forceinline__ void interp_range(double* f, const double* h, int M, int N, bool add, int t0, int dt) {
    const long ldh = M + 2, ldf = 2 * M + 2;
    const int n = M * N;
    for (int t = t0; t < n; t += dt) {
        const int J = 1 + t / M;
        const int I = 1 + (t - (J - 1) * M);
        const long kh = I + J * ldh;
#pragma unroll
        for (int si = 0; si < 2; ++si)
#pragma unroll
            for (int sj = 0; sj < 2; ++sj) {
                const long di = 2 * si - 1, dj = (2 * sj - 1) * ldh;
                double s = 0.0;
                s += (9.0 / 16.0) * h[kh];
                s += (3.0 / 16.0) * h[kh + dj];
                s += (3.0 / 16.0) * h[kh + di];
                s += (1.0 / 16.0) * h[kh + di + dj];
                const long kf = (2 * I - 1 + si) + (long)(2 * J - 1 + sj) * ldf;
                f[kf] = add ? f[kf] + s : s;
            }
    }
}

__device__ __forceinline__ void zero_range(double* a, int n, int t0, int dt) {
    for (int t = t0; t < n; t += dt) a[t] = 0.0;
}

// ---------------------------------------------------------------------------------------
// Grid-wide kernels, one per operation.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ int gtid() { return blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ int gthreads() { return gridDim.x * blockDim.x; }

__global__ void k_bc(double* a, int M, int N) { bc_range(a, M, N, gtid(), gthreads()); }
__global__ void k_gs(double* u, const double* b, const double* fp, const double* fm, int M, int N, int parity) {
    gs_range(u, b, fp, fm, M, N, parity, gtid(), gthreads());
}
__global__ void k_residual(double* r, const double* u, const double* b, double s, const double* fp,
                           const double* fm, int M, int N) {
    residual_range(r, u, b, s, fp, fm, M, N, gtid(), gthreads());
}
__global__ void k_restrict(double* h, const double* f, int M, int N) { restrict_range(h, f, M, N, gtid(), gthreads()); }
__global__ void k_interp(double* f, const double* h, int M, int N, int add) {
    interp_range(f, h, M, N, add != 0, gtid(), gthreads());
}
__global__ void k_add(double* x, const double* z, long n) {
    for (long t = gtid(); t < n; t += gthreads()) x[t] = x[t] + z[t];
}

// Block sum of per-thread values in a fixed tree order (deterministic for a fixed launch).
__device__ double block_sum(double v, double* sh) {
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int w = blockDim.x >> 1; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] = sh[threadIdx.x] + sh[threadIdx.x + w];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

// fmg!'s residual (Multigrid.jl:386-391) with the sum of squares of each block: a block
// takes columns blockIdx.x + 1, + gridDim.x, ..., its threads the rows.
__global__ void __launch_bounds__(kThreads) k_residual_norm(double* r, const double* u, const double* b, double s,
                                                           const double* fp, const double* fm, int M, int N,
                                                           double* partial) {
    __shared__ double sh[kThreads];
    const long ld = M + 2;
    double acc = 0.0;
    for (int j = 1 + blockIdx.x; j <= N; j += gridDim.x)
        for (int i = 1 + threadIdx.x; i <= M; i += kThreads) {
            const long k = i + j * ld;
            const double v = s * b[k] + lap5(u, k, ld, __ldg(fp + i), __ldg(fm + i));
            r[k] = v;
            acc = acc + v * v;
        }
    const double tot = block_sum(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

// eps = norm(res) / sqrt(M N); out = {eps, converged = (s * tolerance > eps)}.
__global__ void __launch_bounds__(kCtaThreads) k_norm_final(const double* partial, int np, double cells, double stol,
                                                            double* out) {
    __shared__ double sh[kCtaThreads];
    double acc = 0.0;
    for (int t = threadIdx.x; t < np; t += blockDim.x) acc = acc + partial[t];
    const double ss = block_sum(acc, sh);
    if (threadIdx.x == 0) {
        const double eps = sqrt(ss) / sqrt(cells);
        out[0] = eps;
        out[1] = (stol > eps) ? 1.0 : 0.0;
    }
}

// ---------------------------------------------------------------------------------------
// One-CTA kernels for the small levels.
// ---------------------------------------------------------------------------------------
__device__ void smooth_cta(const LevelView& L, const double* b, int n) {
    for (int it = 0; it < n; ++it) {
        bc_range(L.sol, L.M, L.N, threadIdx.x, blockDim.x);
        __syncthreads();
        gs_range(L.sol, b, L.fp, L.fm, L.M, L.N, 0, threadIdx.x, blockDim.x);
        __syncthreads();
        gs_range(L.sol, b, L.fp, L.fm, L.M, L.N, 1, threadIdx.x, blockDim.x);
        __syncthreads();
    }
}

// The same sweeps by warp 0 alone (levels of at most 1024 cells: a warp barrier is far
// cheaper than a block one, and the coarsest level runs 50 sweeps).
__device__ void smooth_warp(const LevelView& L, const double* b, int n) {
    const int lane = threadIdx.x & 31;
    for (int it = 0; it < n; ++it) {
        bc_range(L.sol, L.M, L.N, lane, 32);
        __syncwarp();
        gs_range(L.sol, b, L.fp, L.fm, L.M, L.N, 0, lane, 32);
        __syncwarp();
        gs_range(L.sol, b, L.fp, L.fm, L.M, L.N, 1, lane, 32);
        __syncwarp();
    }
}

__device__ void smooth_coarsest(const LevelView& C) {
    if ((long)(C.M + 2) * (C.N + 2) <= 1024) {
        if (threadIdx.x < 32) smooth_warp(C, C.res, kCoarsestSweeps);
        __syncthreads();
    } else {
        smooth_cta(C, C.res, kCoarsestSweeps);
    }
}

// mgv! (Multigrid.jl:334-377) from level l0 down to the coarsest and back, written as a
// loop: level l solves into sol[l] with right-hand side res[l].
__device__ void vcycle_cta(const MgView& V, int l0) {
    const int t0 = threadIdx.x, dt = blockDim.x;
    for (int l = l0; l < V.levels; ++l) {
        const LevelView& L = V.lv[l];
        const LevelView& H = V.lv[l + 1];
        smooth_cta(L, L.res, V.smooth1);
        bc_range(L.sol, L.M, L.N, t0, dt);
        __syncthreads();
        residual_range(L.res1, L.sol, L.res, 1.0, L.fp, L.fm, L.M, L.N, t0, dt);
        __syncthreads();
        restrict_range(H.res, L.res1, H.M, H.N, t0, dt);
        zero_range(H.sol, (long)(H.M + 2) * (H.N + 2), t0, dt);
        __syncthreads();
    }
    smooth_coarsest(V.lv[V.levels]);
    for (int l = V.levels - 1; l >= l0; --l) {
        const LevelView& L = V.lv[l];
        const LevelView& H = V.lv[l + 1];
        interp_range(L.sol, H.sol, H.M, H.N, true, t0, dt);
        __syncthreads();
        smooth_cta(L, L.res, V.smooth2);
    }
}

__global__ void __launch_bounds__(kCtaThreads) k_vcycle_cta(MgView V, int l0) { vcycle_cta(V, l0); }

// ---------------------------------------------------------------------------------------
// Fused smoothing on the grid-wide levels (even M).  One CTA owns kTileR x kTileZ inner
// cells and holds them in shared memory with a halo of H = 2 NS + 1 cells, enough for
// NS red-black sweeps (half-sweep h only updates the cells h or more away from the loaded
// edge, the ones whose result is still exact) plus the residual's stencil, so NS sweeps of
// the whole level cost one read and one write of it.  Every value a CTA writes depends
// only on cells inside its halo and is computed with the arithmetic of the per-operation
// kernels above, so the result is the same bit for bit.
//   TILE_PRE:     x = NS x (apply!, red, black); apply!; r = b + L x; rh = restrict(r);
//                 the next level's solution cleared (mgv! before its recursion).
//   TILE_PRE_SET: the same with x = interpolate(xh) first (an FMG stage entering mgv!).
//   TILE_POST:    x += interpolate(xh); NS x (apply!, red, black) (mgv! after it).
// In shared memory each column of the tile is split by row parity (local row ii = 2 m +
// parity at parity * PL + column * LH + m), so a colour pass reads every operand at unit
// stride; cp.async gathers the tile into that layout (zero outside the array).  A launch
// reads xin and writes xout (tiles read each other's halo, so not in place).
// ---------------------------------------------------------------------------------------
constexpr int kTileR = 96, kTileZ = 24, kTileThreads = 256, kTileWarps = kTileThreads / 32;
enum { TILE_PRE = 0, TILE_PRE_SET = 1, TILE_POST = 2 };

struct TileArgs {
    const double* xin;   // current solution of the level (unused by TILE_PRE_SET)
    double* xout;
    const double* b;     // right-hand side of the level
    const double* xh;    // next coarser solution (TILE_PRE_SET, TILE_POST)
    double* rh;          // next coarser right-hand side (TILE_PRE, TILE_PRE_SET)
    double* hzero;       // next coarser solution to clear (TILE_PRE)
    const double* fp;
    const double* fm;
    int M, N, tiles_r;
};

template <int NS>
struct TileShape {
    static constexpr int H = 2 * NS + 1;                 // halo
    static constexpr int LR = kTileR + 2 * H;            // loaded rows (even)
    static constexpr int LZ = kTileZ + 2 * H;            // loaded columns
    static constexpr int LH = LR / 2;                    // rows of one parity per column
    static constexpr int PL = LH * LZ;                   // doubles per parity plane
    static constexpr int CR = LR / 2 + 4;                // coarse rows for the interpolation
    static constexpr int CZ = LZ / 2 + 3;
    static constexpr int SX = (2 * PL + 15) & ~15;       // doubles per fine array
    static constexpr int SH = (CR * CZ + 15) & ~15;
    static constexpr int SF = (2 * LR + 15) & ~15;       // connector factors: fp even, odd, fm even, odd
    static constexpr size_t smem = sizeof(double) * (size_t)(2 * SX + SH + SF);
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// 8 bytes global -> shared without passing through registers; zeros when !valid.
__device__ __forceinline__ void cp_async8(void* dst, const void* src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" :: "r"(smem_u32(dst)), "l"(src), "r"(valid ? 8 : 0)
                 : "memory");
}

template <class S>
__device__ __forceinline__ int sidx(int ii, int jj) {
    return (ii & 1) * S::PL + jj * S::LH + (ii >> 1);
}

// apply! on the ghost cells of the array that lie in the tile: local (ii, jj) holds
// global (gr0 + ii, gc0 + jj), nr x nz local cells.
template <class S>
__device__ void tile_bc(double* xs, int nr, int nz, int gr0, int gc0, int M, int N) {
    auto at = [&](int i, int j) -> double& { return xs[sidx<S>(i - gr0, j - gc0)]; };
    auto has = [&](int i, int j) { return i >= gr0 && i < gr0 + nr && j >= gc0 && j < gc0 + nz; };
    for (int t = threadIdx.x; t < max(nr, nz); t += blockDim.x) {
        const int i = gr0 + t, j = gc0 + t;
        if (t < nr && i >= 1 && i <= M) {   // Left, Right (inner rows)
            if (has(i, 0) && has(i, 1)) at(i, 0) = dneg(at(i, 1));
            if (has(i, N + 1) && has(i, N)) at(i, N + 1) = dneg(at(i, N));
        }
        if (t < nz && j >= 0 && j <= N + 1) {   // Top, Bottom (every column)
            const int js = j == 0 ? 1 : (j == N + 1 ? N : j);
            const bool edge = (j == 0 || j == N + 1);
            if (has(M + 1, j) && has(M, js)) {
                const double v = edge ? dneg(at(M, js)) : at(M, js);
                at(M + 1, j) = dneg(v);
            }
            if (has(0, j) && has(1, js)) {
                const double v = edge ? dneg(at(1, js)) : at(1, js);
                at(0, j) = v + 0.0;
            }
        }
    }
}

// One colour of gauss_seidel! on the cells h or more away from the loaded edge.  The
// colour's cells of every other column lie in one parity plane at the same local rows, so a
// thread takes one row m across K columns jj0, jj0 + 2, ...: the right neighbour of one cell
// is the left neighbour of the next, and the row's connector factors are loaded once (lanes
// take consecutive m, so a warp reads consecutive doubles).  Each cell's arithmetic is the
// per-operation kernel's, in its order.
template <class S>
__device__ void tile_gs(double* xs, const double* bs, const double* ft, int nr, int nz, int gr0, int gc0, int M,
                        int N, int color, int h) {
    constexpr int LH = S::LH, PL = S::PL, K = 4;
    const int runs = (((nz + 1) >> 1) + K - 1) / K;      // runs of K columns per column parity
    const int n = 2 * runs * LH;
    for (int t = threadIdx.x; t < n; t += kTileThreads) {
        const int g = t / LH, m = t - g * LH;
        const int cls = g & 1, run = g >> 1;
        const int pp = (color ^ (gc0 + cls)) & 1;         // gr0 is even
        const int ii = 2 * m + pp, i = gr0 + ii;
        if (!(ii >= h && ii < nr - h && i >= 1 && i <= M)) continue;
        const double f1 = ft[pp * LH + m], f2 = ft[2 * LH + pp * LH + m];
        const int jj0 = cls + 2 * K * run;
        const int base = pp * PL + m, obase = (1 - pp) * PL + m + pp;   // row ii; row ii + 1
        double lf = jj0 >= 1 ? xs[base + (jj0 - 1) * LH] : 0.0;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int jj = jj0 + 2 * k;
            if (jj >= nz) break;
            const int d = base + jj * LH, o = obase + jj * LH;
            const double rt = jj + 1 < nz ? xs[d + LH] : 0.0;
            const int j = gc0 + jj;
            if (jj >= h && jj < nz - h && j >= 1 && j <= N) {
                const double c = xs[d], up = xs[o], dn = xs[o - 1], bb = bs[d];
                double s = -4.0 * c;
                s += up * f1;
                s += rt;
                s += dn * f2;
                s += lf;
                xs[d] = c + 1.0 * (s + bb) / 4.0;
            }
            lf = rt;
        }
    }
}

template <int NS, int MODE>
__global__ void __launch_bounds__(kTileThreads, 3) k_smooth_tile(TileArgs a) {
    using S = TileShape<NS>;
    constexpr int H = S::H, LR = S::LR, LH = S::LH, PL = S::PL, CR = S::CR, CZ = S::CZ;
    extern __shared__ __align__(16) double smem[];
    double* xs = smem;
    double* bs = smem + S::SX;
    double* hs = bs + S::SX;
    double* ft = hs + S::SH;
    const int M = a.M, N = a.N;
    const long ld = M + 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ti = blockIdx.x % a.tiles_r, tj = blockIdx.x / a.tiles_r;
    const int r0 = 1 + ti * kTileR, c0 = 1 + tj * kTileZ;
    const int r1 = min(r0 + kTileR, M + 1), c1 = min(c0 + kTileZ, N + 1);
    const int gr0 = r0 - H, gc0 = c0 - H;   // gr0 even: local and global row parities agree
    const int nr = (r1 - r0) + 2 * H, nz = (c1 - c0) + 2 * H;
    const int Mh = M / 2, Nh = N / 2;
    const long ldh = Mh + 2;
    const int Ilo = (gr0 >> 1) - 2, Jlo = (gc0 >> 1) - 1;

    // gather x, b, the coarse neighbourhood and the rows' connector factors
    for (int t = threadIdx.x; t < LR * nz; t += kTileThreads) {
        const int jj = t / LR, ii = t - jj * LR;
        const int i = gr0 + ii, j = gc0 + jj;
        const bool in = ii < nr && i >= 0 && i <= M + 1 && j >= 0 && j <= N + 1;
        const long k = in ? i + j * ld : 0;
        const int d = sidx<S>(ii, jj);
        cp_async8(bs + d, a.b + k, in);
        if (MODE != TILE_PRE_SET) cp_async8(xs + d, a.xin + k, in);
    }
    if (MODE != TILE_PRE) {
        for (int t = threadIdx.x; t < CR * CZ; t += kTileThreads) {
            const int jj = t / CR, ii = t - jj * CR;
            const int I = Ilo + ii, J = Jlo + jj;
            const bool in = I >= 0 && I <= Mh + 1 && J >= 0 && J <= Nh + 1;
            cp_async8(hs + t, a.xh + (in ? I + J * ldh : 0), in);
        }
    }
    for (int t = threadIdx.x; t < LR; t += kTileThreads) {
        const int i = gr0 + t;
        const bool in = i >= 0 && i <= M + 1;
        const int d = (t & 1) * LH + (t >> 1);
        cp_async8(ft + d, a.fp + (in ? i : 0), in);
        cp_async8(ft + 2 * LH + d, a.fm + (in ? i : 0), in);
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();

    if (MODE != TILE_PRE) {
        // interpolate! (Multigrid.jl:232-258) into (TILE_PRE_SET) or onto (TILE_POST) x
        for (int par = 0; par < 2; ++par)
            for (int t = threadIdx.x; t < LH * nz; t += kTileThreads) {
                const int jj = t / LH, m = t - jj * LH;
                const int ii = 2 * m + par;
                if (ii >= nr) continue;
                const int i = gr0 + ii, j = gc0 + jj;
                const int d = par * PL + jj * LH + m;
                if (i >= 1 && i <= M && j >= 1 && j <= N) {
                    const int I = (i + 1) >> 1, J = (j + 1) >> 1;
                    const int di = 2 * ((i + 1) & 1) - 1, dj = (2 * ((j + 1) & 1) - 1) * CR;
                    const int kh = (I - Ilo) + (J - Jlo) * CR;
                    double s = 0.0;
                    s += (9.0 / 16.0) * hs[kh];
                    s += (3.0 / 16.0) * hs[kh + dj];
                    s += (3.0 / 16.0) * hs[kh + di];
                    s += (1.0 / 16.0) * hs[kh + di + dj];
                    xs[d] = (MODE == TILE_POST) ? xs[d] + s : s;
                } else if (MODE == TILE_PRE_SET) {
                    xs[d] = 0.0;
                }
            }
        __syncthreads();
    }
    for (int sw = 0; sw < NS; ++sw) {
        tile_bc<S>(xs, nr, nz, gr0, gc0, M, N);
        __syncthreads();
        tile_gs<S>(xs, bs, ft, nr, nz, gr0, gc0, M, N, 0, 2 * sw + 1);
        __syncthreads();
        tile_gs<S>(xs, bs, ft, nr, nz, gr0, gc0, M, N, 1, 2 * sw + 2);
        __syncthreads();
    }
    if (MODE != TILE_POST) {
        tile_bc<S>(xs, nr, nz, gr0, gc0, M, N);
        __syncthreads();
        // residual! (s = 1) and restrict! over the owned coarse cells
        auto X = [&](int ii, int jj) { return xs[sidx<S>(ii, jj)]; };
        const int hr = (r1 - r0) >> 1, hz = (c1 - c0) >> 1;
        const int I0 = (r0 + 1) >> 1, J0 = (c0 + 1) >> 1;
        for (int q = warp; q < hz; q += kTileWarps) {
            const int J = J0 + q;
            for (int p = lane; p < hr; p += 32) {
                const int I = I0 + p;
                double s = 0.0;
#pragma unroll
                for (int c = 0; c < 4; ++c) {   // children (0,0), (0,1), (1,0), (1,1)
                    const int ii = 2 * I - 1 + (c >> 1) - gr0, jj = 2 * J - 1 + (c & 1) - gc0;
                    const int f = (ii & 1) * LH + (ii >> 1);
                    double l = -4.0 * X(ii, jj);
                    l += X(ii + 1, jj) * ft[f];
                    l += X(ii, jj + 1);
                    l += X(ii - 1, jj) * ft[2 * LH + f];
                    l += X(ii, jj - 1);
                    const double r = 1.0 * bs[sidx<S>(ii, jj)] + l;
                    s += r;
                }
                a.rh[I + (long)J * ldh] = 4.0 * s / 4.0;
            }
        }
        if (MODE == TILE_PRE) {
            // xh .= 0 over the owned coarse cells, coarse ghosts by the edge tiles
            const int ia = (ti == 0) ? 0 : I0, ib = (r1 == M + 1) ? Mh + 2 : I0 + hr;
            const int ja = (tj == 0) ? 0 : J0, jb = (c1 == N + 1) ? Nh + 2 : J0 + hz;
            for (int J = ja + warp; J < jb; J += kTileWarps)
                for (int I = ia + lane; I < ib; I += 32) a.hzero[I + (long)J * ldh] = 0.0;
        }
    }
    // the owned cells, with the array's ghosts by the edge tiles
    const int ia = (ti == 0) ? 0 : r0, ib = (r1 == M + 1) ? M + 2 : r1;
    const int ja = (tj == 0) ? 0 : c0, jb = (c1 == N + 1) ? N + 2 : c1;
    for (int j = ja + warp; j < jb; j += kTileWarps)
        for (int i = ia + lane; i < ib; i += 32) a.xout[i + (long)j * ld] = xs[sidx<S>(i - gr0, j - gc0)];
}

// The coarse end of fmg! (Multigrid.jl:400-428): the restrictions below level `small`,
// the direct solve ws.mat \ btop on the coarsest level, and the FMG stages down to level
// `small`.
__device__ void fmg_tail_body(const MgView& V) {
    const int t0 = threadIdx.x, dt = blockDim.x;
    for (int k = V.small; k < V.levels; ++k) {
        restrict_range(V.lv[k + 1].res, V.lv[k].res, V.lv[k + 1].M, V.lv[k + 1].N, t0, dt);
        __syncthreads();
    }
    {
        const LevelView& C = V.lv[V.levels];
        const long ld = C.M + 2;
        for (long p = t0; p < V.nc; p += dt) {
            double acc = 0.0;
            for (int q = 0; q < V.nc; ++q) {
                const int qi = 1 + q % C.M, qj = 1 + q / C.M;
                acc = acc + V.ainv[p * V.nc + q] * C.res[qi + qj * ld];
            }
            const int pi = 1 + (int)(p % C.M), pj = 1 + (int)(p / C.M);
            C.sol[pi + pj * ld] = acc;
        }
        __syncthreads();
    }
    for (int l = V.levels - 1; l >= V.small; --l) {
        const LevelView& L = V.lv[l];
        const LevelView& H = V.lv[l + 1];
        zero_range(L.sol, (long)(L.M + 2) * (L.N + 2), t0, dt);
        bc_range(H.sol, H.M, H.N, t0, dt);
        __syncthreads();
        interp_range(L.sol, H.sol, H.M, H.N, false, t0, dt);
        __syncthreads();
        vcycle_cta(V, l);
    }
}

__global__ void __launch_bounds__(kCtaThreads) k_fmg_tail(MgView V) { fmg_tail_body(V); }

// The same two tails with the levels from `small` down held in shared memory: the
// connector factors of level `small` (those of a coarser level are their first rows: the
// factor depends on the row index alone), then per level its res, res1 and sol arrays
// (each padded to an even number of doubles).  Every address is the shared base plus an
// offset computed here, so the accesses compile to shared-memory instructions; only level
// `small`'s arrays travel to and from HBM.
__host__ __device__ inline int tail_cells(int M, int N) { return ((M + 2) * (N + 2) + 1) & ~1; }
__host__ __device__ inline int tail_tables(int M) { return 2 * ((M + 2 + 1) & ~1); }

struct TailArgs {
    int M0, N0, K;           // level `small` sizes, levels below it
    int s1, s2, nc, total;   // sweeps, coarsest unknowns, shared doubles
    const double* ainv;
    const double* gres;      // level `small` right-hand side (HBM)
    double* gsol;            // level `small` solution (HBM)
    const double* gfp;       // its connector factors
    const double* gfm;
};

struct TailLevel {
    int M, N;
    double* res;
    double* res1;
    double* sol;
};

__device__ __forceinline__ TailLevel tail_level(double* sm, const TailArgs& A, int k) {
    int off = tail_tables(A.M0), M = A.M0, N = A.N0;
    for (int q = 0; q < k; ++q) {
        off += 3 * tail_cells(M, N);
        M >>= 1;
        N >>= 1;
    }
    const int cp = tail_cells(M, N);
    TailLevel L;
    L.M = M;
    L.N = N;
    L.res = sm + off;
    L.res1 = sm + off + cp;
    L.sol = sm + off + 2 * cp;
    return L;
}

__device__ __forceinline__ void tail_smooth(const TailLevel& L, const double* fp, const double* fm, int n, int t0,
                                            int dt, bool warp_only) {
    for (int it = 0; it < n; ++it) {
        bc_range(L.sol, L.M, L.N, t0, dt);
        if (warp_only) __syncwarp(); else __syncthreads();
        gs_range(L.sol, L.res, fp, fm, L.M, L.N, 0, t0, dt);
        if (warp_only) __syncwarp(); else __syncthreads();
        gs_range(L.sol, L.res, fp, fm, L.M, L.N, 1, t0, dt);
        if (warp_only) __syncwarp(); else __syncthreads();
    }
}

// mgv! from tail level k0 (level small + k0) down to the coarsest and back.
__device__ __forceinline__ void tail_vcycle(double* sm, const TailArgs& A, int k0) {
    const double* fp = sm;
    const double* fm = sm + tail_tables(A.M0) / 2;
    const int t0 = threadIdx.x, dt = blockDim.x;
    for (int k = k0; k < A.K; ++k) {
        const TailLevel L = tail_level(sm, A, k), H = tail_level(sm, A, k + 1);
        tail_smooth(L, fp, fm, A.s1, t0, dt, false);
        bc_range(L.sol, L.M, L.N, t0, dt);
        __syncthreads();
        residual_range(L.res1, L.sol, L.res, 1.0, fp, fm, L.M, L.N, t0, dt);
        __syncthreads();
        restrict_range(H.res, L.res1, H.M, H.N, t0, dt);
        zero_range(H.sol, (H.M + 2) * (H.N + 2), t0, dt);
        __syncthreads();
    }
    const TailLevel C = tail_level(sm, A, A.K);
    if ((C.M + 2) * (C.N + 2) <= 1024) {   // the coarsest sweeps by one warp
        if (threadIdx.x < 32) tail_smooth(C, fp, fm, kCoarsestSweeps, threadIdx.x, 32, true);
        __syncthreads();
    } else {
        tail_smooth(C, fp, fm, kCoarsestSweeps, t0, dt, false);
    }
    for (int k = A.K - 1; k >= k0; --k) {
        const TailLevel L = tail_level(sm, A, k), H = tail_level(sm, A, k + 1);
        interp_range(L.sol, H.sol, H.M, H.N, true, t0, dt);
        __syncthreads();
        tail_smooth(L, fp, fm, A.s2, t0, dt, false);
    }
}

__device__ __forceinline__ void tail_load(double* sm, const TailArgs& A, bool with_sol) {
    zero_range(sm, A.total, threadIdx.x, blockDim.x);
    __syncthreads();
    const int m2 = A.M0 + 2;
    for (int t = threadIdx.x; t < m2; t += blockDim.x) {
        sm[t] = A.gfp[t];
        sm[tail_tables(A.M0) / 2 + t] = A.gfm[t];
    }
    const TailLevel G = tail_level(sm, A, 0);
    const int n = (G.M + 2) * (G.N + 2);
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        G.res[t] = A.gres[t];
        if (with_sol) G.sol[t] = A.gsol[t];
    }
    __syncthreads();
}

__device__ __forceinline__ void tail_store(double* sm, const TailArgs& A) {
    __syncthreads();
    const TailLevel G = tail_level(sm, A, 0);
    const int n = (G.M + 2) * (G.N + 2);
    for (int t = threadIdx.x; t < n; t += blockDim.x) A.gsol[t] = G.sol[t];
}

__global__ void __launch_bounds__(kCtaThreads) k_vcycle_tail_smem(TailArgs A) {
    extern __shared__ __align__(16) double sm[];
    tail_load(sm, A, true);
    tail_vcycle(sm, A, 0);
    tail_store(sm, A);
}

// fmg_tail_body on the shared-memory levels.
__global__ void __launch_bounds__(kCtaThreads) k_fmg_tail_smem(TailArgs A) {
    extern __shared__ __align__(16) double sm[];
    const int t0 = threadIdx.x, dt = blockDim.x;
    tail_load(sm, A, false);
    for (int k = 0; k < A.K; ++k) {
        const TailLevel L = tail_level(sm, A, k), H = tail_level(sm, A, k + 1);
        restrict_range(H.res, L.res, H.M, H.N, t0, dt);
        __syncthreads();
    }
    {
        const TailLevel C = tail_level(sm, A, A.K);
        const int ld = C.M + 2;
        for (int p = t0; p < A.nc; p += dt) {
            double acc = 0.0;
            for (int q = 0; q < A.nc; ++q) {
                const int qi = 1 + q % C.M, qj = 1 + q / C.M;
                acc = acc + A.ainv[(long)p * A.nc + q] * C.res[qi + qj * ld];
            }
            C.sol[(1 + p % C.M) + (1 + p / C.M) * ld] = acc;
        }
        __syncthreads();
    }
    for (int k = A.K - 1; k >= 0; --k) {
        const TailLevel L = tail_level(sm, A, k), H = tail_level(sm, A, k + 1);
        zero_range(L.sol, (L.M + 2) * (L.N + 2), t0, dt);
        bc_range(H.sol, H.M, H.N, t0, dt);
        __syncthreads();
        interp_range(L.sol, H.sol, H.M, H.N, false, t0, dt);
        __syncthreads();
        tail_vcycle(sm, A, k);
    }
    tail_store(sm, A);
}

// ---------------------------------------------------------------------------------------
// Free boundary condition (freebc.jl:12-35) and the steps of poisson! around the solve.
// ---------------------------------------------------------------------------------------
// grad[j-1] = (u[M+1, j] - u[M, j]) / dr, j = 1..N.
__global__ void k_top_grad(const double* u, int M, int N, double dr, double* grad) {
    const long ld = M + 2;
    for (long j = 1 + gtid(); j <= N; j += gthreads()) grad[j - 1] = (u[M + 1 + j * ld] - u[M + j * ld]) / dr;
}

// sin(pi m / (2n)) for any m >= 0 from the quarter-wave table q[0..n].
__device__ __forceinline__ double sin_quarter(const double* q, uint32_t m, uint32_t n) {
    const uint32_t two = 2u * n;
    const bool neg = (m % (2u * two)) >= two;
    uint32_t r = m % two;
    if (r > n) r = two - r;
    const double v = __ldg(q + r);
    return neg ? -v : v;
}

// am[k] = (-(dr/2) * RODFT10(grad)[k]) / f[k], one warp per k.  RODFT10:
// Y_k = 2 sum_j X_j sin(pi (2j+1)(k+1) / (2n)).
__global__ void k_dst2_am(const double* grad, const double* qsin, const double* f, int n, double dr, double* am) {
    const int lane = threadIdx.x & 31;
    const long warp = gtid() >> 5, warps = gthreads() >> 5;
    const uint32_t mod = 4u * (uint32_t)n;
    for (long k = warp; k < n; k += warps) {
        const uint32_t kk = (uint32_t)k + 1u;
        const uint32_t step = (uint32_t)((64ull * kk) % mod);
        uint32_t m = (uint32_t)(((2ull * lane + 1ull) * kk) % mod);
        double acc = 0.0;
        for (int j = lane; j < n; j += 32) {
            acc = acc + grad[j] * sin_quarter(qsin, m, (uint32_t)n);
            m += step;
            if (m >= mod) m -= mod;
        }
        for (int o = 16; o > 0; o >>= 1) acc = acc + __shfl_down_sync(0xffffffffu, acc, o);
        if (lane == 0) am[k] = (-(dr / 2.0) * (2.0 * acc)) / f[k];
    }
}

// bcond[k+1] = RODFT01(am)[k] / 2 + RODFT01(am1)[k], am1 = am's last entry alone, i.e.
// RODFT01(am1)[k] = (-1)^k am[n-1].  RODFT01:
// Y_k = (-1)^k X_{n-1} + 2 sum_{j<n-1} X_j sin(pi (j+1)(2k+1) / (2n)).
__global__ void k_dst3_bcond(const double* am, const double* qsin, int n, double* bcond) {
    const int lane = threadIdx.x & 31;
    const long warp = gtid() >> 5, warps = gthreads() >> 5;
    const uint32_t mod = 4u * (uint32_t)n;
    for (long k = warp; k < n; k += warps) {
        const uint32_t kk = 2u * (uint32_t)k + 1u;
        const uint32_t step = (uint32_t)((32ull * kk) % mod);
        uint32_t m = (uint32_t)(((uint64_t)lane + 1ull) * kk % mod);
        double acc = 0.0;
        for (int j = lane; j < n - 1; j += 32) {
            acc = acc + am[j] * sin_quarter(qsin, m, (uint32_t)n);
            m += step;
            if (m >= mod) m -= mod;
        }
        for (int o = 16; o > 0; o >>= 1) acc = acc + __shfl_down_sync(0xffffffffu, acc, o);
        if (lane == 0) {
            const double last = (k & 1) ? -am[n - 1] : am[n - 1];
            const double y = last + 2.0 * acc;
            bcond[k + 1] = y / 2.0 + last;
        }
    }
}

// setinhom!(mg, b, TopBnd(), bcond) (boundaries.jl:141-153): b[M, j] += c * bcond[j].
__global__ void k_set_inhom_top(double* b, int M, int N, double c, const double* bcond) {
    const long ld = M + 2;
    for (long j = gtid(); j <= N + 1; j += gthreads()) b[M + j * ld] = b[M + j * ld] + c * bcond[j];
}

// u[M+1, :] .+= 2 .* bcond (freebc.jl:35).
__global__ void k_top_ghost(double* u, int M, int N, const double* bcond) {
    const long ld = M + 2;
    for (long j = gtid(); j <= N + 1; j += gthreads()) u[M + 1 + j * ld] = u[M + 1 + j * ld] + 2.0 * bcond[j];
}

// q of poisson! (poisson.jl:17-34) from the int64 cell charges: densities q * 2^-32 / dV,
// q0 = (qfixed + qpart - ne) e through the NullDenoiser's Float32 copy.  qfixed is the int64
// deposit plus qfd, its FP64 density part (setneedle!, initfromfiles!), and ne the fluid
// density ((M+4)x(N+4)); either is zero when absent (null pointer).  Ghost cells are zero.
__global__ void k_assemble(double* b, const long long* qf, const long long* qp, const double* qfd,
                           const double* ne, int M, int N, double dr, double dz, uint32_t* status) {
    const long ld = M + 2;
    const long n = (long)(M + 2) * (N + 2);
    for (long t = gtid(); t < n; t += gthreads()) {
        const int j = (int)(t / ld);
        const int i = (int)(t - (long)j * ld);
        double v = 0.0;
        // a cell sum within a factor 2 of where the int64 2^-32 e sums would wrap
        const unsigned long long uf = (unsigned long long)qf[t], up = (unsigned long long)qp[t];
        const unsigned long long af = qf[t] < 0 ? 0ull - uf : uf, ap = qp[t] < 0 ? 0ull - up : up;
        if (af >= (unsigned long long)kMaxNodeCharge || ap >= (unsigned long long)kMaxNodeCharge)
            atomicOr(status, ST_CHARGE);
        if (i >= 1 && i <= M && j >= 1 && j <= N) {
            const double rc = ((double)(i - 1) + 0.5) * dr;
            const double dv = 2.0 * M_PI * rc * dr * dz;
            const double df = (double)qf[t] * 0x1p-32 / dv;
            const double dp = (double)qp[t] * 0x1p-32 / dv;
            double q0 = df;
            if (qfd) q0 = q0 + qfd[t];
            q0 = q0 + dp;
            q0 = q0 - (ne ? ne[(long)(i + 1) + (long)(j + 1) * (M + 4)] : 0.0);
            q0 = q0 * kElementaryCharge;
            v = (double)__double2float_rn(q0);
        }
        b[t] = v;
    }
}

// poisson.jl:47-52: er[i,j] = (u[i-1,j] - u[i,j]) / dr, ez[i,j] = eb + (u[i,j-1] - u[i,j]) / dz
// for i = 1..M+1, j = 1..N+1 on the (M+3)x(N+3) face arrays.
__global__ void k_faces(double* er, double* ez, const double* u, double eb, double dr, double dz, int M, int N) {
    const long ld = M + 2, lf = M + 3;
    const long n = (long)(M + 1) * (N + 1);
    for (long t = gtid(); t < n; t += gthreads()) {
        const int j = 1 + (int)(t / (M + 1));
        const int i = 1 + (int)(t - (long)(j - 1) * (M + 1));
        const long k = i + j * ld;
        er[i + j * lf] = (u[k - 1] - u[k]) / dr;
        ez[i + j * lf] = eb + (u[k - ld] - u[k]) / dz;
    }
}

// poisson.jl:54-57: ez[0,:] = ez[1,:], ez[M+1,:] = ez[M,:], er[:,0] = er[:,1],
// er[:,N+1] = er[:,N] (independent copies for M, N >= 2).
__global__ void k_faces_edges(double* er, double* ez, int M, int N) {
    const long lf = M + 3;
    for (long t = gtid(); t <= (long)max(M, N) + 2; t += gthreads()) {
        if (t <= N + 2) {
            ez[0 + t * lf] = ez[1 + t * lf];
            ez[M + 1 + t * lf] = ez[M + t * lf];
        }
        if (t <= M + 2) {
            er[t] = er[t + lf];
            er[t + (N + 1) * lf] = er[t + N * lf];
        }
    }
}

// FP32 copies of the face fields (the FP32 push gathers them).
__global__ void k_faces32(const double* er, const double* ez, float* er32, float* ez32, long n) {
    for (long t = gtid(); t < n; t += gthreads()) {
        er32[t] = (float)er[t];
        ez32[t] = (float)ez[t];
    }
}

// ---------------------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------------------
// I1/I0 and K1/K0 at x > 0 (the exponential scalings of besselix/besselkx cancel).
// Small x: the power series of I0, I1 and the K's from libstdc++; large x: the Hankel
// asymptotic expansions (Abramowitz & Stegun 9.7.1, 9.7.2), summed while the terms fall.
void bessel_ratios(double x, double* ri, double* rk) {
    if (x < 30.0) {
        long double i0 = 0, i1 = 0, t0 = 1, t1 = x / 2.0L;
        const long double q = (long double)x * x / 4.0L;
        for (int k = 0; k < 200; ++k) {
            i0 += t0;
            i1 += t1;
            t0 *= q / ((k + 1.0L) * (k + 1.0L));
            t1 *= q / ((k + 1.0L) * (k + 2.0L));
            if (t0 < 1e-22L * i0 && t1 < 1e-22L * i1) break;
        }
        *ri = (double)(i1 / i0);
        *rk = (double)(std::cyl_bessel_k(1.0L, (long double)x) / std::cyl_bessel_k(0.0L, (long double)x));
        return;
    }
    // a_k(nu) = prod_{m=1..k} (4 nu^2 - (2m-1)^2) / (k! 8^k)
    long double si0 = 1, si1 = 1, sk0 = 1, sk1 = 1, a0 = 1, a1 = 1;
    const long double z = 8.0L * x;
    for (int k = 1; k < 200; ++k) {
        const long double o = (2.0L * k - 1.0L) * (2.0L * k - 1.0L);
        const long double n0 = a0 * (0.0L - o) / (k * z), n1 = a1 * (4.0L - o) / (k * z);
        if (std::fabs(n0) >= std::fabs(a0) && k > 1) break;   // the terms stopped falling
        a0 = n0;
        a1 = n1;
        const long double sg = (k & 1) ? -1.0L : 1.0L;
        si0 += sg * a0;
        si1 += sg * a1;
        sk0 += a0;
        sk1 += a1;
        if (std::fabs(a0) < 1e-22L && std::fabs(a1) < 1e-22L) break;
    }
    *ri = (double)(si1 / si0);
    *rk = (double)(sk1 / sk0);
}

}  // namespace
}  // namespace mcs

using namespace mcs;

struct mcs_poisson {
    mcs_ctx* ctx = nullptr;
    mcs_grid* g = nullptr;
    int M = 0, N = 0, levels = 0, smooth1 = 2, smooth2 = 2, maxiter = 50, small = 0;
    double s = 1.0, tol = 0.0, dr = 0.0, dz = 0.0, R = 0.0, L = 0.0;
    int nblocks_norm = 0;
    MgView V{};
    std::vector<void*> allocs;
    double* u = nullptr;       // potential (fields.u)
    double* b = nullptr;       // right-hand side (fields.q)
    double* fvec = nullptr;    // freebc coefficients f_n, n = 1..N
    double* qsin = nullptr;    // sin(pi m / (2N)), m = 0..N
    double* grad = nullptr;    // N
    double* am = nullptr;      // N
    double* bcond = nullptr;   // N + 2
    double* partial = nullptr;
    double* dnorm = nullptr;   // {eps, converged}
    double* hnorm = nullptr;   // pinned copy
    double* sol2[kMaxLevels + 1] = {};   // second solution buffer of the grid-wide levels
    int tail_smem = 0;                            // bytes of the shared-memory tail (0: in HBM)
    bool fused = false;                   // smooth1, smooth2 in {1, 2}: fused tile kernels
    long long launches = 0;    // kernels launched by this workspace
    cudaGraphExec_t x_check = nullptr, x_work = nullptr;   // the two halves of fmg!
    long long n_check = 0, n_work = 0;                     // kernels per replay
    int last_iters[2] = {0, 0};
    double last_eps = 0.0;
};

namespace {

int palloc(mcs_poisson* p, double** out, size_t count) {
    void* d = nullptr;
    if (cudaMalloc(&d, count * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return set_err(p->ctx, MCS_ERR_NOMEM, "poisson: device allocation failed");
    }
    p->allocs.push_back(d);
    *out = static_cast<double*>(d);
    return cudaMemset(d, 0, count * sizeof(double)) == cudaSuccess ? MCS_OK : MCS_ERR_CUDA;
}

template <int NS>
int tile_attr(mcs_poisson* p) {
    using S = TileShape<NS>;
    const void* fns[3] = {(const void*)k_smooth_tile<NS, TILE_PRE>, (const void*)k_smooth_tile<NS, TILE_PRE_SET>,
                          (const void*)k_smooth_tile<NS, TILE_POST>};
    for (const void* f : fns)
        if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::smem) != cudaSuccess)
            return set_err(p->ctx, MCS_ERR_CUDA, "poisson: shared memory attribute failed");
    return MCS_OK;
}

int tile_setup(mcs_poisson* p) {
    if (int e = tile_attr<1>(p)) return e;
    return tile_attr<2>(p);
}

int use_dev(mcs_poisson* p) {
    MCS_CK(p->ctx, cudaSetDevice(p->ctx->device));
    return MCS_OK;
}

int grid_blocks(mcs_poisson* p, long work) {
    const long b = (work + kThreads - 1) / kThreads;
    const long cap = (long)p->ctx->num_sms * 8;
    return (int)std::max(1L, std::min(b, cap));
}

size_t cells_of(int M, int N) { return (size_t)(M + 2) * (N + 2); }

// Gauss-Jordan inverse with partial pivoting of buildmat's Cartesian matrix
// (Multigrid.jl:261-295) on the coarsest level.
void coarse_inverse(int Mc, int Nc, std::vector<double>& inv) {
    const int n = Mc * Nc;
    std::vector<long double> a((size_t)n * 2 * n, 0.0L);
    auto A = [&](int r, int c) -> long double& { return a[(size_t)r * 2 * n + c]; };
    const int di[4] = {1, 0, -1, 0}, dj[4] = {0, 1, 0, -1};
    for (int j = 1; j <= Nc; ++j)
        for (int i = 1; i <= Mc; ++i) {
            const int p = (i - 1) + (j - 1) * Mc;
            A(p, p) -= 4.0L;
            A(p, n + p) = 1.0L;
            for (int d = 0; d < 4; ++d) {
                int ni = i + di[d], nj = j + dj[d];
                long double m = 1.0L;
                if (nj == 0) { nj = 1; m = -1.0L; }
                else if (nj == Nc + 1) { nj = Nc; m = -1.0L; }
                else if (ni == Mc + 1) { ni = Mc; m = -1.0L; }
                else if (ni == 0) { ni = 1; m = 1.0L; }
                A(p, (ni - 1) + (nj - 1) * Mc) += m;
            }
        }
    for (int k = 0; k < n; ++k) {
        int best = k;
        for (int r = k + 1; r < n; ++r)
            if (std::fabs(A(r, k)) > std::fabs(A(best, k))) best = r;
        if (best != k)
            for (int c = 0; c < 2 * n; ++c) std::swap(A(k, c), A(best, c));
        const long double piv = A(k, k);
        for (int c = 0; c < 2 * n; ++c) A(k, c) /= piv;
        for (int r = 0; r < n; ++r) {
            if (r == k) continue;
            const long double f = A(r, k);
            if (f == 0.0L) continue;
            for (int c = 0; c < 2 * n; ++c) A(r, c) -= f * A(k, c);
        }
    }
    inv.resize((size_t)n * n);
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) inv[(size_t)r * n + c] = (double)A(r, n + c);
}

#define PSN_LAUNCH(p) MCS_CK((p)->ctx, cudaGetLastError())

// The one-CTA tails: mgv! from level `small`, and the coarse end of fmg!.
TailArgs tail_args(mcs_poisson* p) {
    const LevelView& G = p->V.lv[p->small];
    TailArgs A{};
    A.M0 = G.M;
    A.N0 = G.N;
    A.K = p->levels - p->small;
    A.s1 = p->smooth1;
    A.s2 = p->smooth2;
    A.nc = p->V.nc;
    A.total = p->tail_smem / (int)sizeof(double);
    A.ainv = p->V.ainv;
    A.gres = G.res;
    A.gsol = G.sol;
    A.gfp = G.fp;
    A.gfm = G.fm;
    return A;
}

void launch_vtail(mcs_poisson* p, cudaStream_t st) {
    ++p->launches;
    if (p->tail_smem)
        k_vcycle_tail_smem<<<1, kCtaThreads, p->tail_smem, st>>>(tail_args(p));
    else
        k_vcycle_cta<<<1, kCtaThreads, 0, st>>>(p->V, p->small);
}

void launch_ftail(mcs_poisson* p, cudaStream_t st) {
    ++p->launches;
    if (p->tail_smem)
        k_fmg_tail_smem<<<1, kCtaThreads, p->tail_smem, st>>>(tail_args(p));
    else
        k_fmg_tail<<<1, kCtaThreads, 0, st>>>(p->V);
}

int smooth_grid(mcs_poisson* p, const LevelView& L, const double* b, int n, cudaStream_t st) {
    const long hm = (long)((L.M + 1) >> 1) * L.N;
    for (int it = 0; it < n; ++it) {
        ++p->launches;
        k_bc<<<grid_blocks(p, std::max(L.M + 1, L.N + 2)), kThreads, 0, st>>>(L.sol, L.M, L.N);
        ++p->launches;
        k_gs<<<grid_blocks(p, hm), kThreads, 0, st>>>(L.sol, b, L.fp, L.fm, L.M, L.N, 0);
        ++p->launches;
        k_gs<<<grid_blocks(p, hm), kThreads, 0, st>>>(L.sol, b, L.fp, L.fm, L.M, L.N, 1);
    }
    PSN_LAUNCH(p);
    return MCS_OK;
}

// mgv! from level l0 (< small) down: grid-wide kernels above `small`, the one-CTA
// V-cycle from `small` on.
int vcycle(mcs_poisson* p, int l0, cudaStream_t st) {
    const MgView& V = p->V;
    for (int l = l0; l < p->small; ++l) {
        const LevelView& L = V.lv[l];
        const LevelView& H = V.lv[l + 1];
        if (int e = smooth_grid(p, L, L.res, V.smooth1, st)) return e;
        ++p->launches;
        k_bc<<<grid_blocks(p, std::max(L.M + 1, L.N + 2)), kThreads, 0, st>>>(L.sol, L.M, L.N);
        ++p->launches;
        k_residual<<<grid_blocks(p, (long)L.M * L.N), kThreads, 0, st>>>(L.res1, L.sol, L.res, 1.0, L.fp, L.fm,
                                                                           L.M, L.N);
        ++p->launches;
        k_restrict<<<grid_blocks(p, (long)H.M * H.N), kThreads, 0, st>>>(H.res, L.res1, H.M, H.N);
        MCS_CK(p->ctx, cudaMemsetAsync(H.sol, 0, cells_of(H.M, H.N) * sizeof(double), st));
    }
    launch_vtail(p, st);
    for (int l = p->small - 1; l >= l0; --l) {
        const LevelView& L = V.lv[l];
        const LevelView& H = V.lv[l + 1];
        ++p->launches;
        k_interp<<<grid_blocks(p, (long)H.M * H.N), kThreads, 0, st>>>(L.sol, H.sol, H.M, H.N, 1);
        if (int e = smooth_grid(p, L, L.res, V.smooth2, st)) return e;
    }
    PSN_LAUNCH(p);
    return MCS_OK;
}

// Which buffer holds each grid-wide level's solution while a graph is recorded; the
// recorded pointers then follow the same hand-offs on every replay.
struct Buffers {
    int cur[kMaxLevels + 1] = {};
};

double* sol_buf(mcs_poisson* p, const Buffers& B, int l) {
    return (l < p->small && B.cur[l]) ? p->sol2[l] : p->V.lv[l].sol;
}

template <int NS, int MODE>
void launch_tile(mcs_poisson* p, const TileArgs& a, cudaStream_t st) {
    using S = TileShape<NS>;
    const int tr = (a.M + kTileR - 1) / kTileR, tz = (a.N + kTileZ - 1) / kTileZ;
    TileArgs b = a;
    b.tiles_r = tr;
    ++p->launches;
    k_smooth_tile<NS, MODE><<<tr * tz, kTileThreads, S::smem, st>>>(b);
}

// One fused step at level l: TILE_PRE / TILE_PRE_SET (smooth1 sweeps) or TILE_POST
// (smooth2 sweeps); hands level l's solution to its other buffer.
void tile_step(mcs_poisson* p, Buffers& B, int l, int mode, cudaStream_t st) {
    const LevelView& L = p->V.lv[l];
    TileArgs a{};
    a.xin = sol_buf(p, B, l);
    B.cur[l] ^= 1;
    a.xout = sol_buf(p, B, l);
    a.b = L.res;
    a.xh = sol_buf(p, B, l + 1);
    a.rh = p->V.lv[l + 1].res;
    a.hzero = sol_buf(p, B, l + 1);
    a.fp = L.fp;
    a.fm = L.fm;
    a.M = L.M;
    a.N = L.N;
    const int ns = mode == TILE_POST ? p->smooth2 : p->smooth1;
    if (ns == 1) {
        if (mode == TILE_PRE) launch_tile<1, TILE_PRE>(p, a, st);
        else if (mode == TILE_PRE_SET) launch_tile<1, TILE_PRE_SET>(p, a, st);
        else launch_tile<1, TILE_POST>(p, a, st);
    } else {
        if (mode == TILE_PRE) launch_tile<2, TILE_PRE>(p, a, st);
        else if (mode == TILE_PRE_SET) launch_tile<2, TILE_PRE_SET>(p, a, st);
        else launch_tile<2, TILE_POST>(p, a, st);
    }
}

// mgv! from level l0 (< small) with the fused kernels; `set` = the FMG stage entry, whose
// level-l0 solution starts as the interpolation of the next coarser one.
int vcycle_fused(mcs_poisson* p, Buffers& B, int l0, bool set, cudaStream_t st) {
    for (int l = l0; l < p->small; ++l) {
        const bool first_set = set && l == l0;
        tile_step(p, B, l, first_set ? TILE_PRE_SET : TILE_PRE, st);
        if (first_set) {
            const LevelView& H = p->V.lv[l + 1];
            MCS_CK(p->ctx, cudaMemsetAsync(sol_buf(p, B, l + 1), 0, cells_of(H.M, H.N) * sizeof(double), st));
        }
    }
    launch_vtail(p, st);
    for (int l = p->small - 1; l >= l0; --l) tile_step(p, B, l, TILE_POST, st);
    PSN_LAUNCH(p);
    return MCS_OK;
}

int fmg_work_fused(mcs_poisson* p, cudaStream_t st) {
    const MgView& V = p->V;
    Buffers B;
    for (int k = 0; k < p->small; ++k) {
        ++p->launches;
        k_restrict<<<grid_blocks(p, (long)V.lv[k + 1].M * V.lv[k + 1].N), kThreads, 0, st>>>(
            V.lv[k + 1].res, V.lv[k].res, V.lv[k + 1].M, V.lv[k + 1].N);
    }
    launch_ftail(p, st);
    for (int l = p->small - 1; l >= 0; --l) {
        const LevelView& H = V.lv[l + 1];
        ++p->launches;
        k_bc<<<grid_blocks(p, std::max(H.M + 1, H.N + 2)), kThreads, 0, st>>>(sol_buf(p, B, l + 1), H.M, H.N);
        if (int e = vcycle_fused(p, B, l, true, st)) return e;
    }
    const long n = (long)cells_of(p->M, p->N);
    ++p->launches;
    k_add<<<grid_blocks(p, n), kThreads, 0, st>>>(p->u, sol_buf(p, B, 0), n);
    ++p->launches;
    k_bc<<<grid_blocks(p, std::max(p->M + 1, p->N + 2)), kThreads, 0, st>>>(p->u, p->M, p->N);
    PSN_LAUNCH(p);
    return MCS_OK;
}

// The test at the top of fmg! (Multigrid.jl:384-398): apply!, the residual s b + L u and
// its RMS, copied to the pinned {eps, converged} pair.
int fmg_check(mcs_poisson* p, cudaStream_t st) {
    const LevelView& F = p->V.lv[0];
    ++p->launches;
    k_bc<<<grid_blocks(p, std::max(p->M + 1, p->N + 2)), kThreads, 0, st>>>(p->u, p->M, p->N);
    ++p->launches;
    k_residual_norm<<<p->nblocks_norm, kThreads, 0, st>>>(F.res, p->u, p->b, p->s, F.fp, F.fm, p->M, p->N,
                                                          p->partial);
    ++p->launches;
    k_norm_final<<<1, kCtaThreads, 0, st>>>(p->partial, p->nblocks_norm, (double)((long long)p->M * p->N),
                                            p->s * p->tol, p->dnorm);
    PSN_LAUNCH(p);
    MCS_CK(p->ctx, cudaMemcpyAsync(p->hnorm, p->dnorm, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    return MCS_OK;
}

// The rest of fmg! (Multigrid.jl:400-433): restrictions, the coarsest direct solve, the
// FMG stages with their V-cycles, u += correction, apply!.
int fmg_work(mcs_poisson* p, cudaStream_t st) {
    const MgView& V = p->V;
    const LevelView& F = V.lv[0];
    for (int k = 0; k < p->small; ++k) {
        ++p->launches;
        k_restrict<<<grid_blocks(p, (long)V.lv[k + 1].M * V.lv[k + 1].N), kThreads, 0, st>>>(
            V.lv[k + 1].res, V.lv[k].res, V.lv[k + 1].M, V.lv[k + 1].N);
    }
    launch_ftail(p, st);
    for (int l = p->small - 1; l >= 0; --l) {
        const LevelView& L = V.lv[l];
        const LevelView& H = V.lv[l + 1];
        MCS_CK(p->ctx, cudaMemsetAsync(L.sol, 0, cells_of(L.M, L.N) * sizeof(double), st));
        ++p->launches;
        k_bc<<<grid_blocks(p, std::max(H.M + 1, H.N + 2)), kThreads, 0, st>>>(H.sol, H.M, H.N);
        ++p->launches;
        k_interp<<<grid_blocks(p, (long)H.M * H.N), kThreads, 0, st>>>(L.sol, H.sol, H.M, H.N, 0);
        if (int e = vcycle(p, l, st)) return e;
    }
    const long n = (long)cells_of(p->M, p->N);
    ++p->launches;
    k_add<<<grid_blocks(p, n), kThreads, 0, st>>>(p->u, F.sol, n);
    ++p->launches;
    k_bc<<<grid_blocks(p, std::max(p->M + 1, p->N + 2)), kThreads, 0, st>>>(p->u, p->M, p->N);
    PSN_LAUNCH(p);
    return MCS_OK;
}

// Records `fn` into a graph (on a private stream: the context's stream may be the legacy
// one, which cannot be captured) and counts the kernels one replay launches.
template <typename Fn>
int capture(mcs_poisson* p, Fn fn, cudaGraphExec_t* exec, long long* nlaunch) {
    cudaStream_t cs;
    MCS_CK(p->ctx, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    const long long before = p->launches;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    int st = e == cudaSuccess ? fn(cs) : MCS_ERR_CUDA;
    cudaGraph_t g = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    *nlaunch = p->launches - before;
    p->launches = before;
    if (st || e != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return st ? st : set_err(p->ctx, MCS_ERR_CUDA, "poisson: graph capture failed");
    }
    e = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return set_err(p->ctx, MCS_ERR_CUDA, "poisson: graph instantiate failed");
    return MCS_OK;
}

int replay(mcs_poisson* p, cudaGraphExec_t exec, long long nlaunch) {
    p->launches += nlaunch;
    MCS_CK(p->ctx, cudaGraphLaunch(exec, p->ctx->stream));
    return MCS_OK;
}

// fmg! (Multigrid.jl:380-434) on u, b.  *cont = false once the residual is below
// s * tolerance (nothing else is done then).  Both halves replay CUDA graphs.
int fmg(mcs_poisson* p, bool* cont) {
    if (!p->x_check) {
        if (int e = capture(p, [&](cudaStream_t s) { return fmg_check(p, s); }, &p->x_check, &p->n_check)) return e;
        if (int e = capture(p, [&](cudaStream_t s) { return p->fused ? fmg_work_fused(p, s) : fmg_work(p, s); },
                            &p->x_work, &p->n_work))
            return e;
    }
    if (int e = replay(p, p->x_check, p->n_check)) return e;
    MCS_CK(p->ctx, cudaStreamSynchronize(p->ctx->stream));
    p->last_eps = p->hnorm[0];
    if (p->hnorm[1] != 0.0) {
        *cont = false;
        return MCS_OK;
    }
    *cont = true;
    return replay(p, p->x_work, p->n_work);
}

// Multigrid.solve (Multigrid.jl:449-467): fmg! while it reports work and iter <= maxiter.
int mg_solve(mcs_poisson* p, int* iters) {
    bool cont = true;
    int iter = 0;
    while (cont && iter <= p->maxiter) {
        if (int e = fmg(p, &cont)) return e;
        ++iter;
    }
    if (iters) *iters = iter;
    return MCS_OK;
}

int freebc(mcs_poisson* p, int* it) {
    cudaStream_t st = p->ctx->stream;
    if (int e = mg_solve(p, &it[0])) return e;
    const int n = p->N;
    ++p->launches;
    k_top_grad<<<grid_blocks(p, n), kThreads, 0, st>>>(p->u, p->M, n, p->dr, p->grad);
    const int wblocks = (int)std::min<long>(((long)n * 32 + kThreads - 1) / kThreads, (long)p->ctx->num_sms * 16);
    ++p->launches;
    k_dst2_am<<<wblocks, kThreads, 0, st>>>(p->grad, p->qsin, p->fvec, n, p->dr, p->am);
    ++p->launches;
    k_dst3_bcond<<<wblocks, kThreads, 0, st>>>(p->am, p->qsin, n, p->bcond);
    const double c = (2.0 / p->s) * (1.0 + 1.0 / (double)(2 * p->M - 1));
    ++p->launches;
    k_set_inhom_top<<<grid_blocks(p, n + 2), kThreads, 0, st>>>(p->b, p->M, n, c, p->bcond);
    PSN_LAUNCH(p);
    if (int e = mg_solve(p, &it[1])) return e;
    ++p->launches;
    k_top_ghost<<<grid_blocks(p, n + 2), kThreads, 0, st>>>(p->u, p->M, n, p->bcond);
    PSN_LAUNCH(p);
    return MCS_OK;
}

}  // namespace

extern "C" {

MCS_API int mcs_freebc_coefficients(double L, double R, int N, double* f) {
    if (!(L > 0) || !(R > 0) || N < 1 || !f) return MCS_ERR_ARG;
    const double kk = M_PI / L;
    for (int n = 1; n <= N; ++n) {
        const double k = kk * (double)n;
        const double x = k * R;
        double ri, rk;
        bessel_ratios(x, &ri, &rk);
        f[n - 1] = L * k * (ri + rk) / 2.0;
    }
    return MCS_OK;
}

MCS_API int mcs_poisson_create(mcs_grid* g, int levels, int smooth1, int smooth2, int maxiter, double tolerance,
                               double s, mcs_poisson** out) {
    if (!g || !out) return MCS_ERR_ARG;
    mcs_ctx* c = g->ctx;
    const GridView& gv = g->v;
    if (gv.type != GRID_CYL) return set_err(c, MCS_ERR_ARG, "poisson: needs a cylindrical grid");
    const int M = gv.M, N = gv.N;
    if (levels < 0 || levels > kMaxLevels || smooth1 < 0 || smooth2 < 0 || maxiter < 0 || !(tolerance >= 0))
        return set_err(c, MCS_ERR_ARG, "poisson: bad multigrid configuration");
    if ((long)(M + 3) * (N + 3) >= (1L << 31))
        return set_err(c, MCS_ERR_ARG, "poisson: grid above 2^31 cells");
    if (M < 2 || N < 2 || ((M >> levels) << levels) != M || ((N >> levels) << levels) != N)
        return set_err(c, MCS_ERR_ARG, "poisson: M and N must be multiples of 2^levels (and >= 2)");
    const int Mc = M >> levels, Nc = N >> levels;
    if ((long)Mc * Nc > kMaxCoarse) return set_err(c, MCS_ERR_ARG, "poisson: coarsest level above 4096 cells");
    MCS_CK(c, cudaSetDevice(c->device));
    mcs_poisson* p = new (std::nothrow) mcs_poisson();
    if (!p) return MCS_ERR_NOMEM;
    p->ctx = c;
    p->g = g;
    p->M = M;
    p->N = N;
    p->levels = levels;
    p->smooth1 = smooth1;
    p->smooth2 = smooth2;
    p->maxiter = maxiter;
    p->tol = tolerance;
    p->dr = gv.dr;
    p->dz = gv.dz;
    p->R = gv.R;
    p->L = gv.L;
    p->s = (s > 0) ? s : gv.dz * gv.dz / kEpsilon0;   // main.jl:138
    p->nblocks_norm = c->num_sms * 4;
    auto fail = [&](int e) {
        mcs_poisson_destroy(p);
        return e;
    };
    int e = MCS_OK;
    p->V.levels = levels;
    p->V.smooth1 = smooth1;
    p->V.smooth2 = smooth2;
    // The tail (levels small..levels) runs in one CTA: from shared memory when the three
    // arrays of all its levels fit (the finest such split), else from HBM for the levels
    // of at most kSmallCells cells.
    p->small = levels;
    p->tail_smem = 0;
    for (int l = 0; l <= levels; ++l) {
        long tot = tail_tables(M >> l);
        for (int k = l; k <= levels; ++k) tot += 3 * tail_cells(M >> k, N >> k);
        if (tot * (long)sizeof(double) <= kTailSmemBytes) {
            p->small = l;
            p->tail_smem = (int)(tot * sizeof(double));
            break;
        }
    }
    if (!p->tail_smem)
        for (int l = 0; l <= levels; ++l)
            if ((long)(M >> l) * (N >> l) <= kSmallCells) { p->small = l; break; }
    p->V.small = p->small;
    if (p->tail_smem &&
        (cudaFuncSetAttribute(k_vcycle_tail_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, p->tail_smem) !=
             cudaSuccess ||
         cudaFuncSetAttribute(k_fmg_tail_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, p->tail_smem) !=
             cudaSuccess)) {
        delete p;
        return set_err(c, MCS_ERR_CUDA, "poisson: shared memory attribute failed");
    }
    std::vector<double> tab;
    for (int l = 0; l <= levels; ++l) {
        LevelView& Lv = p->V.lv[l];
        Lv.M = M >> l;
        Lv.N = N >> l;
        const size_t n = cells_of(Lv.M, Lv.N);
        double *res, *res1, *sol, *fpm;
        if ((e = palloc(p, &res, n)) || (e = palloc(p, &res1, n)) || (e = palloc(p, &sol, n)) ||
            (e = palloc(p, &fpm, 2 * (size_t)(Lv.M + 2))))
            return fail(e);
        Lv.res = res;
        Lv.res1 = res1;
        Lv.sol = sol;
        // CylindricalConnector{1} (Multigrid.jl:37-39): 1 + d / (2 i - 1) for storage row i.
        tab.assign(2 * (size_t)(Lv.M + 2), 0.0);
        for (int i = 1; i <= Lv.M + 1; ++i) {
            tab[i] = 1.0 + 1.0 / (double)(2 * i - 1);
            tab[Lv.M + 2 + i] = 1.0 + (-1.0) / (double)(2 * i - 1);
        }
        if (cudaMemcpy(fpm, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
            return fail(set_err(c, MCS_ERR_CUDA, "poisson: upload failed"));
        Lv.fp = fpm;
        Lv.fm = fpm + Lv.M + 2;
    }
    p->fused = smooth1 >= 1 && smooth1 <= 2 && smooth2 >= 1 && smooth2 <= 2;
    if (p->fused) {
        for (int l = 0; l < p->small; ++l)
            if ((e = palloc(p, &p->sol2[l], cells_of(M >> l, N >> l)))) return fail(e);
        if ((e = tile_setup(p))) return fail(e);
    }
    std::vector<double> inv;
    coarse_inverse(Mc, Nc, inv);
    double* ainv;
    if ((e = palloc(p, &ainv, inv.size()))) return fail(e);
    if (cudaMemcpy(ainv, inv.data(), inv.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(set_err(c, MCS_ERR_CUDA, "poisson: upload failed"));
    p->V.ainv = ainv;
    p->V.nc = Mc * Nc;
    const size_t ncell = cells_of(M, N);
    if ((e = palloc(p, &p->u, ncell)) || (e = palloc(p, &p->b, ncell)) || (e = palloc(p, &p->fvec, N)) ||
        (e = palloc(p, &p->qsin, (size_t)N + 1)) || (e = palloc(p, &p->grad, N)) || (e = palloc(p, &p->am, N)) ||
        (e = palloc(p, &p->bcond, (size_t)N + 2)) || (e = palloc(p, &p->partial, p->nblocks_norm)) ||
        (e = palloc(p, &p->dnorm, 2)))
        return fail(e);
    if (cudaMallocHost(&p->hnorm, 2 * sizeof(double)) != cudaSuccess)
        return fail(set_err(c, MCS_ERR_NOMEM, "poisson: pinned allocation failed"));
    std::vector<double> f(N), q(N + 1);
    mcs_freebc_coefficients(p->L, p->R, N, f.data());
    for (int m = 0; m <= N; ++m) q[m] = (double)std::sin(3.14159265358979323846264338327950288L * m / (2.0L * N));
    if (cudaMemcpy(p->fvec, f.data(), N * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(p->qsin, q.data(), (N + 1) * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(set_err(c, MCS_ERR_CUDA, "poisson: upload failed"));
    // the zero fills and uploads ran on the legacy stream; the context's stream does not
    // wait for it
    if (cudaDeviceSynchronize() != cudaSuccess) return fail(set_err(c, MCS_ERR_CUDA, "poisson: init failed"));
    *out = p;
    return MCS_OK;
}

MCS_API int mcs_poisson_destroy(mcs_poisson* p) {
    if (!p) return MCS_ERR_ARG;
    if (p->ctx && p->ctx->stream) cudaStreamSynchronize(p->ctx->stream);
    if (p->x_check) cudaGraphExecDestroy(p->x_check);
    if (p->x_work) cudaGraphExecDestroy(p->x_work);
    for (void* a : p->allocs) cudaFree(a);
    if (p->hnorm) cudaFreeHost(p->hnorm);
    delete p;
    return MCS_OK;
}

MCS_API int mcs_poisson_upload(mcs_poisson* p, int which, const double* host) {
    if (!p || !host) return MCS_ERR_ARG;
    if (int e = use_dev(p)) return e;
    double* d = which == MCS_PSN_U ? p->u : which == MCS_PSN_B ? p->b : nullptr;
    if (!d) return MCS_ERR_ARG;
    MCS_CK(p->ctx, cudaMemcpyAsync(d, host, cells_of(p->M, p->N) * sizeof(double), cudaMemcpyHostToDevice,
                                   p->ctx->stream));
    MCS_CK(p->ctx, cudaStreamSynchronize(p->ctx->stream));
    return MCS_OK;
}

MCS_API int mcs_poisson_download(mcs_poisson* p, int which, double* host) {
    if (!p || !host) return MCS_ERR_ARG;
    if (int e = use_dev(p)) return e;
    const double* d = nullptr;
    size_t n = cells_of(p->M, p->N);
    if (which == MCS_PSN_U) d = p->u;
    else if (which == MCS_PSN_B) d = p->b;
    else if (which == MCS_PSN_BCOND) { d = p->bcond; n = (size_t)p->N + 2; }
    else if (which == MCS_PSN_FREEBC_F) { d = p->fvec; n = (size_t)p->N; }
    if (!d) return MCS_ERR_ARG;
    MCS_CK(p->ctx, cudaMemcpyAsync(host, d, n * sizeof(double), cudaMemcpyDeviceToHost, p->ctx->stream));
    MCS_CK(p->ctx, cudaStreamSynchronize(p->ctx->stream));
    return MCS_OK;
}

MCS_API int mcs_poisson_launches(mcs_poisson* p, int64_t* count) {
    if (!p || !count) return MCS_ERR_ARG;
    *count = p->launches;
    return MCS_OK;
}

MCS_API int mcs_poisson_zero(mcs_poisson* p, int which) {
    if (!p) return MCS_ERR_ARG;
    if (int e = use_dev(p)) return e;
    double* d = which == MCS_PSN_U ? p->u : which == MCS_PSN_B ? p->b : nullptr;
    if (!d) return MCS_ERR_ARG;
    MCS_CK(p->ctx, cudaMemsetAsync(d, 0, cells_of(p->M, p->N) * sizeof(double), p->ctx->stream));
    return MCS_OK;
}

// Mean duration of one finest-level red-black pass and one finest-level residual, each
// launched `reps` times back to back between CUDA events on the context's stream.  They
// run on the workspace's scratch levels, so u and b are untouched.
MCS_API int mcs_poisson_profile(mcs_poisson* p, int reps, float* gs_ms, float* residual_ms, float* tile_ms) {
    if (!p || reps < 1) return MCS_ERR_ARG;
    if (int e = use_dev(p)) return e;
    cudaStream_t st = p->ctx->stream;
    const LevelView& F = p->V.lv[0];
    const long hm = (long)((F.M + 1) >> 1) * F.N;
    cudaEvent_t e0, e1;
    MCS_CK(p->ctx, cudaEventCreate(&e0));
    MCS_CK(p->ctx, cudaEventCreate(&e1));
    float ms = 0.0f;
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps; ++r) {
        ++p->launches;
        k_gs<<<grid_blocks(p, hm), kThreads, 0, st>>>(F.sol, F.res, F.fp, F.fm, F.M, F.N, r & 1);
    }
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    if (gs_ms) *gs_ms = ms / reps;
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps; ++r) {
        ++p->launches;
        k_residual<<<grid_blocks(p, (long)F.M * F.N), kThreads, 0, st>>>(F.res1, F.sol, F.res, 1.0, F.fp, F.fm,
                                                                           F.M, F.N);
    }
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    if (residual_ms) *residual_ms = ms / reps;
    if (tile_ms) *tile_ms = 0.0f;
    if (tile_ms && p->fused && p->small > 0) {
        // the fused post-smoothing of the finest level: sol -> sol2 with the next level's
        // solution interpolated on
        const LevelView& H = p->V.lv[1];
        TileArgs a{};
        a.xin = F.sol;
        a.xout = p->sol2[0];
        a.b = F.res;
        a.xh = H.sol;
        a.fp = F.fp;
        a.fm = F.fm;
        a.M = F.M;
        a.N = F.N;
        cudaEventRecord(e0, st);
        for (int r = 0; r < reps; ++r) {
            if (p->smooth2 == 1) launch_tile<1, TILE_POST>(p, a, st);
            else launch_tile<2, TILE_POST>(p, a, st);
        }
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        *tile_ms = ms / reps;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    PSN_LAUNCH(p);
    return MCS_OK;
}

MCS_API int mcs_poisson_mg_solve(mcs_poisson* p, int* iters, double* eps_last) {
    if (!p) return MCS_ERR_ARG;
    if (int e = use_dev(p)) return e;
    int it = 0;
    if (int e = mg_solve(p, &it)) return e;
    if (int e = sync_status(p->ctx)) return e;
    if (iters) *iters = it;
    if (eps_last) *eps_last = p->last_eps;
    return MCS_OK;
}

MCS_API int mcs_poisson_solve_freebc(mcs_poisson* p, int* iters) {
    if (!p) return MCS_ERR_ARG;
    if (int e = use_dev(p)) return e;
    int it[2] = {0, 0};
    if (int e = freebc(p, it)) return e;
    if (int e = sync_status(p->ctx)) return e;
    if (iters) { iters[0] = it[0]; iters[1] = it[1]; }
    return MCS_OK;
}

MCS_API int mcs_poisson_assemble(mcs_poisson* p) {
    if (!p) return MCS_ERR_ARG;
    if (int e = use_dev(p)) return e;
    const long n = (long)cells_of(p->M, p->N);
    ++p->launches;
    const mcs_fluid* fl = p->g->fluid;
    k_assemble<<<grid_blocks(p, n), kThreads, 0, p->ctx->stream>>>(
        p->b, p->g->d_q[MCS_Q_FIXED], p->g->d_q[MCS_Q_PART], p->g->d_qfd, fl ? fl->ne[fl->cur] : nullptr,
        p->M, p->N, p->dr, p->dz, p->ctx->d_status);
    PSN_LAUNCH(p);
    return MCS_OK;
}

MCS_API int mcs_poisson_fields(mcs_poisson* p, double eb) {
    if (!p) return MCS_ERR_ARG;
    if (int e = use_dev(p)) return e;
    cudaStream_t st = p->ctx->stream;
    ++p->launches;
    k_faces<<<grid_blocks(p, (long)(p->M + 1) * (p->N + 1)), kThreads, 0, st>>>(p->g->d_er, p->g->d_ez, p->u, eb,
                                                                                p->dr, p->dz, p->M, p->N);
    ++p->launches;
    k_faces_edges<<<grid_blocks(p, std::max(p->M, p->N) + 3), kThreads, 0, st>>>(p->g->d_er, p->g->d_ez, p->M, p->N);
    const long nf = (long)(p->M + 3) * (p->N + 3);
    ++p->launches;
    k_faces32<<<grid_blocks(p, nf), kThreads, 0, st>>>(p->g->d_er, p->g->d_ez, p->g->d_erz32, p->g->d_erz32 + nf, nf);
    PSN_LAUNCH(p);
    return MCS_OK;
}

MCS_API int mcs_poisson_run(mcs_poisson* p, double eb, int* iters) {
    if (!p) return MCS_ERR_ARG;
    if (int e = mcs_poisson_assemble(p)) return e;
    if (int e = mcs_poisson_solve_freebc(p, iters)) return e;
    if (int e = mcs_poisson_fields(p, eb)) return e;
    return sync_status(p->ctx);
}

}  // extern "C"
