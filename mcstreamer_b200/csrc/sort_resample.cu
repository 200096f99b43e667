// sort_resample.cu -- cell-key radix sort of the population and the per-cell Russian
// roulette / splitting of MCStreamer's resample! (MCStreamer/src/resample.jl:7-84).
//
// mcs_sort_cells: stable LSD radix sort of (cell key, slot) with 8-bit digits; only as many
// passes as the key range needs (keys are cell indices; inactive or out-of-grid particles
// get the key `ncells` and go last).  Each pass: per-tile digit histograms, one device-wide
// scan of the (digit, tile) table, and a stable scatter ranked with warp match-any.  A
// final gather permutes every population array.  Stability keeps the particles of a cell
// in ascending original slot order: the order in which the reference's serial passes
// visit them.
//
// mcs_resample_cells: after the sort every cell is a contiguous segment.  A count pass
// finds each cell's clones -- a thread per splitting cell, a warp per merging cell, which
// records its clone sources and total weight -- and, after a scan of the counts gives each
// cell its place, a write pass appends them.  The decisions are those of resample.jl's
// serial passes in slot order: the merging cells' weight sums are the serial FP64 sums bit
// for bit (exact warp sums where the weights allow, else the serial loop).  Clones are
// appended in cell order, which is the slot order of the sorted population (the serial
// reference's append order).  Uniforms: one Philox stream per cell, ctr = {cell, call,
// k/4, tag}.  ntarget > nmax or ntarget > 128 takes a thread-per-cell form of both passes.
#include <algorithm>

#include "host_util.h"
#include "pop_ops.h"
#include "step.cuh"

namespace mcs {

namespace {

constexpr int SB = 256;            // threads per block
constexpr int SI = 16;             // keys per thread per tile
constexpr int STILE = SB * SI;     // 4096 keys per tile
constexpr int RADIX = 256;

// ---- keys ----
template <typename T>
__global__ void k_keys(PopView<T> P, GridView g, int mesh, uint32_t ncells, uint32_t* __restrict__ key,
                       uint32_t* __restrict__ val) {
    const long long n = *P.n_in;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        uint32_t k = ncells;
        if (P.act[i]) {
            if (mesh) {
                const uint32_t c = P.cell[i];
                k = c == 0xffffffffu ? ncells : c;
            } else if (g.type == GRID_CART3D) {
                int ix, iy, iz;
                double fx, fy, fz;
                if (cart_locate(g, P.f[0][i], P.f[1][i], P.f[2][i], ix, iy, iz, fx, fy, fz))
                    k = (uint32_t)ix + (uint32_t)g.nx * ((uint32_t)iy + (uint32_t)g.ny * (uint32_t)iz);
            } else {
                // cellindex, MCStreamer/src/grid.jl:84-90, over p's (0:M+1, 0:N+1)
                const double x = P.f[0][i], y = P.f[1][i], z = P.f[2][i];
                const double rho = sqrt(x * x + y * y);
                double fi = floor(rho / g.dr);
                if (__fma_rn(fi, g.dr, -rho) > 0.0) fi -= 1.0;
                double fj = floor(z / g.dz);
                if (__fma_rn(fj, g.dz, -z) > 0.0) fj -= 1.0;
                fi += 1.0; fj += 1.0;
                if (fi >= 0.0 && fi <= g.M + 1.0 && fj >= 0.0 && fj <= g.N + 1.0)
                    k = (uint32_t)fi + (uint32_t)(g.M + 2) * (uint32_t)fj;
            }
        }
        key[i] = k;
        val[i] = (uint32_t)i;
    }
}

// ---- radix pass: histogram ----
// The (digit, tile) table is digit-major over the tiles the keys fill (ntiles of n keys),
// so that its scan covers those tiles only.
__global__ void __launch_bounds__(SB) k_hist(const uint32_t* __restrict__ key, const long long* n_ptr, int shift,
                                             uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[RADIX];
    const long long n = *n_ptr;
    const long long ntiles = (n + STILE - 1) / STILE;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        for (int d = threadIdx.x; d < RADIX; d += SB) h[d] = 0;
        __syncthreads();
        const long long base = tile * STILE;
        for (int it = 0; it < SI; ++it) {
            const long long i = base + (long long)it * SB + threadIdx.x;
            if (i < n) atomicAdd(&h[(key[i] >> shift) & 0xffu], 1u);
        }
        __syncthreads();
        for (int d = threadIdx.x; d < RADIX; d += SB) hist[(long long)d * ntiles + tile] = h[d];
        __syncthreads();
    }
}

// Entries of the (digit, tile) table of n keys.
__global__ void k_hist_entries(const long long* n_ptr, long long* out) {
    *out = (long long)RADIX * ((*n_ptr + STILE - 1) / STILE);
}

// ---- radix pass: stable scatter.  Each warp takes a contiguous 32*SI-key share of the
// tile and counts its keys per digit (warp match-any, the digit group's first lane adds),
// keeping each key's rank among the warp's keys of its digit; a block prefix of those
// counts gives every key its place in the tile sorted by digit (stable), where it is put in
// shared memory; the tile then goes out in that order, so that consecutive threads write
// consecutive slots of each digit's run.  Six barriers per tile.  At most 64 registers (4
// blocks of 256 per SM, a few bytes spilled): the occupancy is worth more than the spill.
__global__ void __launch_bounds__(SB, 4) k_scatter(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                uint32_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                const long long* n_ptr, int shift, const uint32_t* __restrict__ offs) {
    constexpr int NW = SB / 32;
    __shared__ uint32_t wc[NW][RADIX];   // per-warp digit counts -> the warp's first tile-local slot per digit
    __shared__ uint32_t loc[RADIX];      // first tile-local slot of each digit
    __shared__ uint32_t gofs[RADIX];     // the digit's first slot of this tile in the output
    __shared__ uint32_t skey[STILE], sval[STILE];
    const long long n = *n_ptr;
    const long long ntiles = (n + STILE - 1) / STILE;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        for (int d = threadIdx.x; d < NW * RADIX; d += SB) (&wc[0][0])[d] = 0;
        __syncthreads();
        const long long base = tile * STILE + (long long)wid * (32 * SI);
        uint32_t k[SI];
        uint32_t rk[SI / 2];   // each key's rank among the warp's keys of its digit (< 32 SI), two per word
#pragma unroll
        for (int r = 0; r < SI; ++r) {
            const long long i = base + (long long)r * 32 + lane;
            k[r] = i < n ? kin[i] : 0u;
            const uint32_t dg = i < n ? ((k[r] >> shift) & 0xffu) : 0x100u;
            const unsigned peers = __match_any_sync(0xffffffffu, dg);
            const uint32_t before = dg < RADIX ? wc[wid][dg] : 0u;
            __syncwarp();
            const uint32_t rank = before + __popc(peers & lt);
            if (r & 1) rk[r >> 1] |= rank << 16;
            else rk[r >> 1] = rank;
            if (dg < RADIX && (peers & lt) == 0) wc[wid][dg] = before + __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        // per digit: the warps' counts prefixed in warp order; the digit's tile total
        for (int d = threadIdx.x; d < RADIX; d += SB) {
            uint32_t acc = 0;
            for (int w2 = 0; w2 < NW; ++w2) { const uint32_t c = wc[w2][d]; wc[w2][d] = acc; acc += c; }
            loc[d] = acc;   // the total for now
            gofs[d] = offs[(long long)d * ntiles + tile];
        }
        __syncthreads();
        if (threadIdx.x < 32) {   // exclusive prefix of the 256 digit totals by one warp
            uint32_t t[RADIX / 32], sum = 0;
#pragma unroll
            for (int q = 0; q < RADIX / 32; ++q) { t[q] = loc[lane * (RADIX / 32) + q]; sum += t[q]; }
            uint32_t incl = sum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            uint32_t run = incl - sum;
#pragma unroll
            for (int q = 0; q < RADIX / 32; ++q) { loc[lane * (RADIX / 32) + q] = run; run += t[q]; }
        }
        __syncthreads();
        uint32_t cnt_tile = 0;   // keys of the tile (all threads)
        {
            const long long rest = n - tile * STILE;
            cnt_tile = rest < STILE ? (uint32_t)rest : (uint32_t)STILE;
        }
        // wc[wid][d] is now the warp's first place among the tile's keys of digit d
#pragma unroll
        for (int r = 0; r < SI; ++r) {
            const long long i = base + (long long)r * 32 + lane;
            if (i < n) {
                const uint32_t dg = (k[r] >> shift) & 0xffu;
                const uint32_t pos = loc[dg] + wc[wid][dg] + ((rk[r >> 1] >> (16 * (r & 1))) & 0xffffu);
                skey[pos] = k[r];
                sval[pos] = vin[i];
            }
        }
        __syncthreads();
        for (uint32_t j = threadIdx.x; j < cnt_tile; j += SB) {
            const uint32_t kk = skey[j];
            const uint32_t dg = (kk >> shift) & 0xffu;
            const uint32_t pos = gofs[dg] + (j - loc[dg]);
            kout[pos] = kk;
            vout[pos] = sval[j];
        }
        __syncthreads();
    }
}

struct DstArrays {
    void* f[8];
    uint32_t* cell;
    uint8_t* act;
};

// One state array at a time.  A stable sort by cell keeps every particle within a few
// z-planes of its old place, so the sources that a stretch of destinations reads lie in a
// window of the old order; one array's share of that window stays in L2 while the stretch
// is written, all eight arrays' share does not.
// A sorted key other than ncells belongs to an active particle, and on a mesh population
// it is the particle's cell: only the particles keyed ncells (inactive, or outside the
// mesh) read their flag and cell through the permutation.
template <typename T>
__global__ void k_gather(PopView<T> P, const uint32_t* __restrict__ perm, const uint32_t* __restrict__ key,
                         uint32_t ncells, DstArrays d) {
    const long long n = *P.n_in;
    const long long j0 = blockIdx.x * (long long)blockDim.x + threadIdx.x, js = (long long)gridDim.x * blockDim.x;
    for (int q = 0; q < 8; ++q) {
        const T* __restrict__ src = P.f[q];
        T* __restrict__ dst = static_cast<T*>(d.f[q]);
        for (long long j = j0; j < n; j += js) dst[j] = src[perm[j]];
    }
    for (long long j = j0; j < n; j += js) {
        const uint32_t k = key[j];
        if (k != ncells) {
            if (d.cell) d.cell[j] = k;
            d.act[j] = 1;
        } else {
            const uint32_t s = perm[j];
            if (d.cell) d.cell[j] = P.cell[s];
            d.act[j] = P.act[s];
        }
    }
}

uint32_t grid_cells(const mcs_grid* g) {
    if (g->v.type == GRID_CART3D) return (uint32_t)((long long)g->v.nx * g->v.ny * g->v.nz);
    return (uint32_t)((g->v.M + 2) * (g->v.N + 2));
}

template <typename P>
int ensure(mcs_ctx* c, P** p, size_t n) {
    if (*p) return MCS_OK;
    if (cudaMalloc(reinterpret_cast<void**>(p), (n ? n : 1) * sizeof(P)) != cudaSuccess) {
        *p = nullptr;
        return set_err(c, MCS_ERR_NOMEM, "sort / resample scratch allocation failed");
    }
    return MCS_OK;
}

// ---------------------------------------------------------------------------------------
// Per-cell resampling: resample.jl:16-76 restated for one segment (cell) per thread.
// ---------------------------------------------------------------------------------------
// Segment starts: seg_start[s] = first sorted slot of cell s (keys < ncells only).
__global__ void k_seg_flags(const uint32_t* __restrict__ key, const long long* n_ptr, uint32_t ncells,
                            uint32_t* __restrict__ flag) {
    const long long n = *n_ptr;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
        const uint32_t k = key[j];
        flag[j] = (k < ncells && (j == 0 || key[j - 1] != k)) ? 1u : 0u;
    }
}

__global__ void k_seg_starts(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ pos,
                             const long long* n_ptr, uint32_t* __restrict__ start) {
    const long long n = *n_ptr;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x)
        if (flag[j]) start[pos[j]] = (uint32_t)j;
}

struct ResampleArgs {
    const uint32_t* key;     // sorted keys
    const uint32_t* start;   // segment starts
    const long long* nseg;   // number of segments
    const long long* n;      // particles (sorted)
    uint32_t ncells;
    int ntarget, nmax;
    unsigned long long seed;
    uint32_t call;
};

// One segment: pass 1 then pass 2 of resample!.  WRITE=false only counts the clones.
template <typename T, bool WRITE>
__device__ uint32_t resample_segment(const ResampleArgs& a, PopView<T>& P, long long s, long long clone_base,
                                     long long cap, uint32_t* status) {
    const long long n = *a.n;
    const long long b = a.start[s];
    const uint32_t cell = a.key[b];
    long long e;
    if (s + 1 < *a.nseg) {
        e = a.start[s + 1];   // segments are consecutive: no dependent walk over the keys
    } else {
        e = b;
        while (e < n && a.key[e] == cell) ++e;
    }
    Rng rng;
    rng.init(a.seed, cell, a.call, TAG_CELL_RESAMPLE);
    // pass 1 (resample.jl:16-29): count, total weight, first sample when p reaches nmax
    long long p = 0;
    double wtotal = 0.0, x = 0.0;
    for (long long j = b; j < e; ++j) {
        p += 1;
        wtotal += (double)P.f[6][j];
        if (p == a.nmax) x = 1.0 - pow(1.0 - rng.u64(), 1.0 / (double)a.ntarget);   // samplemin(ntarget)
    }
    // pass 2 (resample.jl:31-76)
    long long pk = 0;
    double wcum = 0.0;
    uint32_t ncl = 0;
    for (long long j = b; j < e; ++j) {
        const double wj = (double)P.f[6][j];
        if (p > a.nmax) {
            while (wtotal * x < wcum + wj && pk < a.ntarget) {
                pk += 1;
                if (WRITE) {
                    const long long d = clone_base + ncl;
                    if (d < cap) {
#pragma unroll
                        for (int q = 0; q < 8; ++q) P.f[q][d] = P.f[q][j];
                        if (P.cell) P.cell[d] = P.cell[j];
                        P.act[d] = P.act[j];
                        P.f[6][d] = (T)(wtotal / (double)a.ntarget);
                    } else {
                        atomicOr(status, ST_CAPACITY);
                    }
                }
                ++ncl;
                if (pk < a.ntarget) x += (1.0 - pow(1.0 - rng.u64(), 1.0 / (double)(a.ntarget - pk))) * (1.0 - x);
            }
            wcum += wj;
            if (WRITE) P.act[j] = 0;   // remove_particle!
        } else if (p < a.ntarget && wj > 2) {
            const double wnew = rint(wj / 2.0);   // Julia round: nearest, ties to even
            if (WRITE) {
                const long long d = clone_base + ncl;
                if (d < cap) {
#pragma unroll
                    for (int q = 0; q < 8; ++q) P.f[q][d] = P.f[q][j];
                    if (P.cell) P.cell[d] = P.cell[j];
                    P.act[d] = P.act[j];
                    P.f[6][d] = (T)wnew;
                } else {
                    atomicOr(status, ST_CAPACITY);
                }
                P.f[6][j] = (T)(wj - wnew);
            }
            ++ncl;
            p += 1;
        }
    }
    return ncl;
}

// ---------------------------------------------------------------------------------------
// Warp per segment.  The decisions are those of resample_segment; the work is spread so
// that the warp's memory accesses are coalesced:
//  * split cells (p < ntarget): the first ntarget - p particles with w > 2, in index order,
//    split -- a ballot rank over the cell's particles (no arithmetic order involved);
//  * merge cells (p > nmax): the count pass selects the clone sources and records them with
//    the cell's total weight; the write pass copies the clones to consecutive slots and
//    removes the originals.
// ---------------------------------------------------------------------------------------
constexpr int RS_WARPS = 8;       // warps per block
constexpr int RS_BUF = 256;       // staged weights per warp (a cell is streamed in chunks)
constexpr int RS_SRC = 128;       // clone sources a merge can record (ntarget above: serial path)

struct RsShared {
    double w[RS_WARPS][RS_BUF];
    double f[RS_WARPS][RS_SRC];      // merge: f_k = samplemin(ntarget - k), then the positions t_k
    uint32_t src[RS_WARPS][RS_SRC];
};

// End of segment s (exclusive): the next segment's start, or for the last segment the first
// slot whose key differs (found 32 slots at a time).
__device__ __forceinline__ long long segment_end(const ResampleArgs& a, long long s, long long nseg, long long b,
                                                 uint32_t cell) {
    if (s + 1 < nseg) return (long long)a.start[s + 1];
    const long long n = *a.n;
    const int lane = threadIdx.x & 31;
    for (long long j0 = b; j0 < n; j0 += 32) {
        const long long j = j0 + lane;
        const unsigned diff = __ballot_sync(0xffffffffu, j < n && a.key[j] != cell);
        const unsigned past = __ballot_sync(0xffffffffu, j >= n);
        const unsigned stop = diff | past;
        if (stop) return j0 + __ffs(stop) - 1;
    }
    return n;
}

template <typename T>
__device__ __forceinline__ void copy_clone(PopView<T>& P, long long d, long long j, T w) {
#pragma unroll
    for (int q = 0; q < 8; ++q) P.f[q][d] = P.f[q][j];
    if (P.cell) P.cell[d] = P.cell[j];
    P.act[d] = 1;
    P.f[6][d] = w;
}

// Folds w into the exponent bounds of a cell's weights: emax = the largest exponent, lmin =
// the exponent of the lowest set bit over all weights.  False for a weight that is
// negative, -0, subnormal, infinite or NaN.
__device__ __forceinline__ bool weight_bits(double w, int& emax, int& lmin) {
    const unsigned long long u = (unsigned long long)__double_as_longlong(w);
    if (u == 0ull) return true;
    const int ex = (int)(u >> 52);   // sign bit included: a negative weight gives ex >= 0x800
    if (ex == 0 || ex >= 0x7ff) return false;
    const unsigned long long m = (u & ((1ull << 52) - 1ull)) | (1ull << 52);
    emax = max(emax, ex - 1023);
    lmin = min(lmin, ex - 1075 + (__ffsll((long long)m) - 1));
    return true;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// f_k = samplemin(ntarget - k) = 1 - (1 - U_k)^(1/(ntarget - k)) of the cell's draws U_k,
// k < ntarget, into fk (the lanes side by side).
__device__ __forceinline__ void merge_factors(const ResampleArgs& a, uint32_t cell, double* fk) {
    const int lane = threadIdx.x & 31;
    const uint32_t k0 = (uint32_t)a.seed, k1 = (uint32_t)(a.seed >> 32);
    for (int k = lane; k < a.ntarget; k += 32) {
        // word k of the cell's stream {cell, call, k/4, TAG_CELL_RESAMPLE}
        const U4 blk = philox10(U4{cell, a.call, (uint32_t)k >> 2, TAG_CELL_RESAMPLE}, k0, k1);
        const uint32_t q = (uint32_t)k & 3u;
        const uint32_t w = q == 0 ? blk.x : q == 1 ? blk.y : q == 2 ? blk.z : blk.w;
        fk[k] = 1.0 - pow(1.0 - uni64(w), 1.0 / (double)(a.ntarget - k));
    }
}

// A merging cell (p > nmax) by one warp: the clone sources of resample.jl:31-76 and the
// cell's total weight, recorded in sel[0, ncl) and *wt; returns ncl.
//
// The sample positions follow x_1 = samplemin(ntarget) and x_(k+1) = x_k + samplemin(ntarget
// - k) (1 - x_k), where samplemin draws the cell's k-th uniform: every factor f_k = 1 - (1 -
// U_k)^(1/(ntarget - k)) depends on the draw alone, so the lanes compute them side by side
// (the pows).  Clone k is the first particle j whose running weight A_j = w_1 + ... + w_j
// (summed in index order) exceeds t_k = wtotal x_k.
//
// Exact form: when every weight is a non-negative multiple of 2^lmin below 2^(emax+1) and
// p 2^(emax+1) <= 2^(lmin+53), every partial sum of the cell's weights is an integer
// multiple of 2^lmin below 2^53 of them, so FP64 adds it without rounding, in any order:
// the warp's prefix sums are then the serial pass's running sums bit for bit.  The x_k
// recurrence stays serial on lane 0 (unfused, the reference's order); with the t_k
// non-decreasing, each lane finds its clones' sources by binary search over the running
// sums staged in shared memory.  Otherwise lane 0 runs both serial passes over the weights
// staged in shared memory.
template <typename T>
__device__ uint32_t merge_select_warp(const ResampleArgs& a, const PopView<T>& P, long long b, long long e,
                                      uint32_t cell, RsShared& sh, int wid, uint32_t* __restrict__ sel,
                                      double* __restrict__ wt) {
    const int lane = threadIdx.x & 31;
    double* wb = sh.w[wid];
    double* fk = sh.f[wid];
    uint32_t* src = sh.src[wid];
    const int nt = a.ntarget;
    merge_factors(a, cell, fk);
    const long long p0 = e - b;
    // pass 1: the exponent bounds and (exact when they allow) the total
    int emax = -4096, lmin = 4096;
    bool ok = true;
    double part = 0.0;
    for (long long j = b + lane; j < e; j += 32) {
        const double w = (double)P.f[6][j];
        ok = weight_bits(w, emax, lmin) && ok;
        part += w;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        emax = max(emax, __shfl_xor_sync(0xffffffffu, emax, o));
        lmin = min(lmin, __shfl_xor_sync(0xffffffffu, lmin, o));
    }
    const int lg = 64 - __clzll((unsigned long long)(p0 - 1));   // ceil(log2 p0), p0 >= 2
    ok = __all_sync(0xffffffffu, ok) && (emax < -4000 || lg + emax + 1 <= lmin + 53);
    double wtotal = warp_sum_d(part);
    __syncwarp();   // fk visible
    bool refill = false;   // fk overwritten by the t_k
    if (ok) {
        refill = true;
        // t_k = wtotal x_k, serially; a decreasing t (x past 1) would break the search
        if (lane == 0) {
            double x = fk[0], tp = 0.0;
            for (int k = 0; k < nt; ++k) {
                if (k > 0) x = __dadd_rn(x, __dmul_rn(fk[k], __dadd_rn(1.0, -x)));
                const double t = __dmul_rn(wtotal, x);
                if (k > 0 && t < tp) ok = false;
                fk[k] = t;
                tp = t;
            }
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        __syncwarp();
    }
    if (ok) {
        // pass 2: running sums by warp scans, a chunk of RS_BUF particles at a time
        constexpr int KPL = RS_SRC / 32;
        int jk[KPL];
#pragma unroll
        for (int i = 0; i < KPL; ++i) jk[i] = -1;
        double carry = 0.0;
        for (long long c0 = b; c0 < e; c0 += RS_BUF) {
            const int m = (int)((e - c0) < RS_BUF ? (e - c0) : RS_BUF);
            for (int r = 0; r < m; r += 32) {
                const int idx = r + lane;
                double v = idx < m ? (double)P.f[6][c0 + idx] : 0.0;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const double y = __shfl_up_sync(0xffffffffu, v, o);
                    if (lane >= o) v += y;
                }
                const double A = carry + v;
                if (idx < m) wb[idx] = A;
                carry = __shfl_sync(0xffffffffu, A, 31);
            }
            __syncwarp();
            const double alast = wb[m - 1];
#pragma unroll
            for (int i = 0; i < KPL; ++i) {
                const int k = lane + 32 * i;
                if (k < nt && jk[i] < 0) {
                    const double t = fk[k];
                    if (t < alast) {
                        int lo = 0, hi = m - 1;   // the first idx with t < wb[idx]
                        while (lo < hi) {
                            const int mid = (lo + hi) >> 1;
                            if (t < wb[mid]) hi = mid; else lo = mid + 1;
                        }
                        jk[i] = (int)(c0 - b) + lo;
                    }
                }
            }
            __syncwarp();
        }
        // the selected k form a prefix 0..ncl-1 (t_k non-decreasing)
        uint32_t cnt = 0;
#pragma unroll
        for (int i = 0; i < KPL; ++i) {
            const int k = lane + 32 * i;
            if (k < nt && jk[i] >= 0) {
                sel[k] = (uint32_t)jk[i];
                ++cnt;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        if (lane == 0) *wt = wtotal;
        return cnt;
    }
    // serial form: both passes on lane 0 over staged weights, in index order
    if (refill) {
        __syncwarp();
        merge_factors(a, cell, fk);
    }
    wtotal = 0.0;
    double x = 0.0;
    for (long long c0 = b; c0 < e; c0 += RS_BUF) {
        const long long m = (e - c0) < RS_BUF ? (e - c0) : RS_BUF;
        __syncwarp();
        for (int q = lane; q < m; q += 32) wb[q] = (double)P.f[6][c0 + q];
        __syncwarp();
        if (lane == 0) {
            for (int q = 0; q < m; ++q) {
                wtotal = __dadd_rn(wtotal, wb[q]);
                if (c0 - b + q + 1 == a.nmax) x = fk[0];   // pass 1: samplemin(ntarget)
            }
        }
    }
    uint32_t ncl = 0;
    long long pk = 0;
    double wcum = 0.0;
    for (long long c0 = b; c0 < e; c0 += RS_BUF) {
        const long long m = (e - c0) < RS_BUF ? (e - c0) : RS_BUF;
        __syncwarp();
        for (int q = lane; q < m; q += 32) wb[q] = (double)P.f[6][c0 + q];
        __syncwarp();
        if (lane == 0) {
            for (int q = 0; q < m; ++q) {
                const double wj = wb[q];
                while (__dmul_rn(wtotal, x) < __dadd_rn(wcum, wj) && pk < nt) {
                    pk += 1;
                    src[ncl++] = (uint32_t)(c0 - b + q);
                    if (pk < nt) x = __dadd_rn(x, __dmul_rn(fk[pk], __dadd_rn(1.0, -x)));
                }
                wcum = __dadd_rn(wcum, wj);
            }
        }
    }
    __syncwarp();
    ncl = __shfl_sync(0xffffffffu, ncl, 0);
    for (uint32_t k = lane; k < ncl; k += 32) sel[k] = src[k];
    if (lane == 0) *wt = wtotal;
    __syncwarp();
    return ncl;
}

// Counting is latency-bound over millions of small segments: a thread per segment keeps 32
// segments' loads in flight per warp.
// Only merging cells need the weight sums and the clone positions; their segments go to a
// worklist for the warp kernel below.  A splitting cell (p < ntarget) clones its first ntarget - p particles with
// w > 2 (resample.jl:62-70); a cell with ntarget <= p <= nmax is left alone.
template <typename T>
__global__ void __launch_bounds__(128) k_resample_count(ResampleArgs a, PopView<T> P, uint32_t* __restrict__ counts,
                                                        uint32_t* __restrict__ merge_list,
                                                        unsigned long long* merge_n) {
    const long long nseg = *a.nseg;
    const long long n = *a.n;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < nseg; s += (long long)gridDim.x * blockDim.x) {
        const long long b = a.start[s];
        long long e;
        if (s + 1 < nseg) {
            e = a.start[s + 1];
        } else {
            const uint32_t cell = a.key[b];
            e = b;
            while (e < n && a.key[e] == cell) ++e;
        }
        const long long p0 = e - b;
        uint32_t cnt = 0;
        if (p0 > a.nmax) {
            merge_list[atomicAdd(merge_n, 1ull)] = (uint32_t)s;
        } else if (p0 < a.ntarget) {
            const long long K = a.ntarget - p0;
            for (long long j = b; j < e && cnt < K; ++j)
                if ((double)P.f[6][j] > 2) ++cnt;
        }
        counts[s] = cnt;
    }
}

// The merging cells of the worklist, a warp each: their clone counts, sources (sel, ntarget
// entries per listed cell) and total weights (wt).
template <typename T>
__global__ void __launch_bounds__(RS_WARPS * 32, 4) k_resample_merge_count(ResampleArgs a, PopView<T> P,
                                                                         uint32_t* __restrict__ counts,
                                                                         const uint32_t* __restrict__ merge_list,
                                                                         const unsigned long long* merge_n,
                                                                         uint32_t* __restrict__ sel,
                                                                         double* __restrict__ wt) {
    __shared__ RsShared sh;
    const long long nm = (long long)*merge_n;
    const long long nseg = *a.nseg;
    const int wid = threadIdx.x >> 5;
    const long long w0 = (long long)blockIdx.x * RS_WARPS + wid, ws = (long long)gridDim.x * RS_WARPS;
    for (long long q = w0; q < nm; q += ws) {
        const long long s = merge_list[q];
        const long long b = a.start[s];
        const uint32_t cell = a.key[b];
        const long long e = segment_end(a, s, nseg, b, cell);
        const uint32_t c = merge_select_warp<T>(a, P, b, e, cell, sh, wid, sel + q * a.ntarget, wt + q);
        if ((threadIdx.x & 31) == 0) counts[s] = c;
    }
}

// The serial form's count, a thread per segment (ntarget > nmax or ntarget > RS_SRC).
template <typename T>
__global__ void __launch_bounds__(128) k_resample_count_serial(ResampleArgs a, PopView<T> P,
                                                               uint32_t* __restrict__ counts, uint32_t* status) {
    const long long nseg = *a.nseg;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < nseg; s += (long long)gridDim.x * blockDim.x)
        counts[s] = resample_segment<T, false>(a, P, s, 0, 0, status);
}

// The serial form, a thread per segment: for ntarget > nmax or ntarget > RS_SRC.
template <typename T>
__global__ void __launch_bounds__(128) k_resample_write_serial(ResampleArgs a, PopView<T> P,
                                                               const uint32_t* __restrict__ offs,
                                                               const long long* total, uint32_t* status) {
    const long long nseg = *a.nseg;
    const long long n = *a.n;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < nseg; s += (long long)gridDim.x * blockDim.x)
        resample_segment<T, true>(a, P, s, n + (long long)offs[s], P.cap, status);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        long long m = n + *total;
        if (m > P.cap) { m = P.cap; atomicOr(status, ST_CAPACITY); }
        *P.n_out = m;
    }
}

// The write pass.  Split cells (segments with clones that are not on the merge worklist)
// take SPLIT_LANES lanes each, a warp four of them side by side: they are many and small
// (p < ntarget), and a group's loads and clone stores cover consecutive slots.  Then the
// merging cells, a warp each: their clones from the recorded sources, each with weight
// wtotal / ntarget, and the removal of the originals.
constexpr int SPLIT_LANES = 8;

template <typename T>
__global__ void __launch_bounds__(RS_WARPS * 32, 4) k_resample_write(ResampleArgs a, PopView<T> P,
                                                                   const uint32_t* __restrict__ counts,
                                                                   const uint32_t* __restrict__ offs,
                                                                   const uint32_t* __restrict__ merge_list,
                                                                   const unsigned long long* merge_n,
                                                                   const uint32_t* __restrict__ sel,
                                                                   const double* __restrict__ wt,
                                                                   const long long* total, uint32_t* status) {
    constexpr int GPW = 32 / SPLIT_LANES;   // split cells per warp
    const long long nseg = *a.nseg;
    const long long n = *a.n;
    const int lane = threadIdx.x & 31;
    const int g = lane / SPLIT_LANES, gl = lane % SPLIT_LANES;
    const long long w0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long ws = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long s0 = w0 * GPW; s0 < nseg; s0 += ws * GPW) {
        const long long s = s0 + g;
        long long b = 0, e = 0, d0 = 0;
        uint32_t K = 0;   // clones of this group's cell: the first K particles with w > 2 split
        if (s < nseg) {
            const uint32_t cnt = counts[s];   // 0: a full cell, or a split cell of light particles
            if (cnt) {
                b = a.start[s];
                if (s + 1 < nseg) {
                    e = a.start[s + 1];
                } else {
                    const uint32_t cell = a.key[b];
                    e = b;
                    while (e < n && a.key[e] == cell) ++e;
                }
                if (e - b < a.ntarget) {   // merging cells (p > nmax) are written below
                    K = cnt;
                    d0 = n + (long long)offs[s];
                }
            }
        }
        // resample.jl:62-70 by rank among the cell's w > 2 particles in index order
        uint32_t ranked = 0;
        for (long long j0 = b; __any_sync(0xffffffffu, ranked < K && j0 < e); j0 += SPLIT_LANES) {
            const long long j = j0 + gl;
            double wj = 0.0;
            bool q = false;
            if (ranked < K && j < e) {
                wj = (double)P.f[6][j];
                q = wj > 2;
            }
            const unsigned bg = (__ballot_sync(0xffffffffu, q) >> (g * SPLIT_LANES)) & ((1u << SPLIT_LANES) - 1u);
            const uint32_t r = ranked + __popc(bg & ((1u << gl) - 1u));
            if (q && r < K) {
                const double wnew = rint(wj / 2.0);   // Julia round: nearest, ties to even
                const long long d = d0 + r;
                if (d < P.cap) copy_clone<T>(P, d, j, (T)wnew);
                else atomicOr(status, ST_CAPACITY);
                P.f[6][j] = (T)(wj - wnew);
            }
            ranked += __popc(bg);
        }
    }
    const long long nm = (long long)*merge_n;
    for (long long q = w0; q < nm; q += ws) {
        const long long s = merge_list[q];
        const long long b = a.start[s];
        const uint32_t cell = a.key[b];
        const long long e = segment_end(a, s, nseg, b, cell);
        const uint32_t ncl = counts[s];
        const long long base = n + (long long)offs[s];
        const T wc = (T)(wt[q] / (double)a.ntarget);
        const uint32_t* sq = sel + q * a.ntarget;
        for (uint32_t k = lane; k < ncl; k += 32) {
            const long long d = base + k;
            if (d < P.cap) copy_clone<T>(P, d, b + sq[k], wc);
            else atomicOr(status, ST_CAPACITY);
        }
        for (long long j = b + lane; j < e; j += 32) P.act[j] = 0;   // remove_particle!
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        long long m = n + *total;
        if (m > P.cap) { m = P.cap; atomicOr(status, ST_CAPACITY); }
        *P.n_out = m;
    }
}

}  // namespace

// The second set of population arrays (cap slots): the sort's permutation target and the
// mesh step's secondary pool.
int reserve_alt(mcs_pop* p) {
    mcs_ctx* c = p->ctx;
    const size_t cap = (size_t)p->cap;
    for (int q = 0; q < 8; ++q)
        if (!p->alt[q] && cudaMalloc(&p->alt[q], cap * p->esz) != cudaSuccess)
            return set_err(c, MCS_ERR_NOMEM, "second population arrays");
    if (int st = ensure(c, &p->alt_act, cap)) return st;
    if (p->cell)
        if (int st = ensure(c, &p->alt_cell, cap)) return st;
    return MCS_OK;
}

// The mesh step's secondary pool (the second set of arrays) and its per-tile tables.
int reserve_mesh_pool(mcs_pop* p) {
    mcs_ctx* c = p->ctx;
    if (int st = reserve_alt(p)) return st;
    const size_t nt = (size_t)p->max_tiles;
    if (int st = ensure(c, &p->app_cnt, nt)) return st;
    if (int st = ensure(c, &p->app_off, nt)) return st;
    if (int st = ensure(c, &p->app_excl, nt)) return st;
    return MCS_OK;
}

// Scratch of the sort (keys, slots, digit tables and the second set of population arrays)
// and, with `resample`, of the per-cell resampling, sized for the population's capacity.
// Allocated once, on first use or by mcs_resample_reserve.
int reserve_sort_scratch(mcs_pop* p, bool resample) {
    mcs_ctx* c = p->ctx;
    const size_t cap = (size_t)p->cap;
    const long long ntiles_max = (p->cap + STILE - 1) / STILE;
    for (int q = 0; q < 2; ++q) {
        if (int st = ensure(c, &p->sort_key[q], cap)) return st;
        if (int st = ensure(c, &p->sort_val[q], cap)) return st;
    }
    if (int st = ensure(c, &p->sort_hist, (size_t)RADIX * ntiles_max)) return st;
    if (int st = ensure(c, &p->sort_hoff, (size_t)RADIX * ntiles_max)) return st;
    if (int st = reserve_alt(p)) return st;
    if (resample) {
        if (int st = ensure(c, &p->seg_a, cap)) return st;
        if (int st = ensure(c, &p->seg_b, cap)) return st;
    }
    return MCS_OK;
}

// Sort the population by cell key; on return the sorted keys are in *keys_out (device).
template <typename T>
int sort_cells_t(mcs_pop* p, mcs_grid* g, uint32_t** keys_out) {
    mcs_ctx* c = p->ctx;
    const long long ntiles_max = (p->cap + STILE - 1) / STILE;
    if (int st = reserve_sort_scratch(p, false)) return st;
    const uint32_t ncells = grid_cells(g);
    int nbits = 1;
    while (nbits < 32 && ((1ull << nbits) <= (unsigned long long)ncells)) ++nbits;
    const int passes = (nbits + 7) / 8;
    const int mesh = p->cells != nullptr;
    const long long* n_dev = p->d_n + p->cur;
    const int gr = grid_for(c, p->cap, 256);
    k_keys<T><<<gr, 256, 0, c->stream>>>(pop_view<T>(p), g->v, mesh, ncells, p->sort_key[0], p->sort_val[0]);
    MCS_CK_LAUNCH(c);
    long long* nhist = reinterpret_cast<long long*>(p->counters + 8);
    k_hist_entries<<<1, 1, 0, c->stream>>>(n_dev, nhist);
    MCS_CK_LAUNCH(c);
    int cur = 0;
    long long gs = ntiles_max;
    if (gs > (long long)c->num_sms * 8) gs = (long long)c->num_sms * 8;
    for (int ps = 0; ps < passes; ++ps) {
        const int shift = 8 * ps;
        k_hist<<<(int)gs, SB, 0, c->stream>>>(p->sort_key[cur], n_dev, shift, p->sort_hist);
        MCS_CK_LAUNCH(c);
        if (int st = launch_scan(p, p->sort_hist, p->sort_hoff, nhist, nullptr)) return st;
        k_scatter<<<(int)gs, SB, 0, c->stream>>>(p->sort_key[cur], p->sort_val[cur], p->sort_key[cur ^ 1],
                                                 p->sort_val[cur ^ 1], n_dev, shift, p->sort_hoff);
        MCS_CK_LAUNCH(c);
        cur ^= 1;
    }
    // permute every population array into the second buffer set, then swap the sets
    DstArrays d;
    for (int q = 0; q < 8; ++q) d.f[q] = p->alt[q];
    d.cell = p->cell ? p->alt_cell : nullptr;
    d.act = p->alt_act;
    k_gather<T><<<gr, 256, 0, c->stream>>>(pop_view<T>(p), p->sort_val[cur], p->sort_key[cur], ncells, d);
    MCS_CK_LAUNCH(c);
    for (int q = 0; q < 8; ++q) std::swap(p->f[q], p->alt[q]);
    std::swap(p->act, p->alt_act);
    if (p->cell) std::swap(p->cell, p->alt_cell);
    if (keys_out) *keys_out = p->sort_key[cur];
    return MCS_OK;
}

template <typename T>
int resample_cells_t(mcs_pop* p, mcs_grid* g, int ntarget, int nmax) {
    mcs_ctx* c = p->ctx;
    uint32_t* keys = nullptr;
    if (int st = reserve_sort_scratch(p, true)) return st;
    if (int st = sort_cells_t<T>(p, g, &keys)) return st;
    const uint32_t ncells = grid_cells(g);
    const long long* n_dev = p->d_n + p->cur;
    long long* nseg = reinterpret_cast<long long*>(p->counters + 10);
    long long* total = reinterpret_cast<long long*>(p->counters + 12);
    const int gr = grid_for(c, p->cap, 256);
    // segments: flags -> positions -> starts
    k_seg_flags<<<gr, 256, 0, c->stream>>>(keys, n_dev, ncells, p->seg_a);
    MCS_CK_LAUNCH(c);
    if (int st = launch_scan(p, p->seg_a, p->seg_b, n_dev, nseg)) return st;
    k_seg_starts<<<gr, 256, 0, c->stream>>>(p->seg_a, p->seg_b, n_dev, p->u32a);
    MCS_CK_LAUNCH(c);
    ResampleArgs a;
    a.key = keys;
    a.start = p->u32a;
    a.nseg = nseg;
    a.n = n_dev;
    a.ncells = ncells;
    a.ntarget = ntarget;
    a.nmax = nmax;
    a.seed = p->seed;
    a.call = p->resample_calls++;
    const bool serial = ntarget > nmax || ntarget > RS_SRC;
    // merging cells hold more than nmax particles each: at most n / (nmax + 1) of them, so
    // their recorded sources (ntarget each, ntarget <= nmax) fit in one cap-slot array (the
    // sort's permutation, consumed by the gather) and their FP64 totals in another (the
    // sort's free key buffer, cap 32-bit words)
    unsigned long long* merge_n = reinterpret_cast<unsigned long long*>(p->counters + 14);
    const int cur = keys == p->sort_key[1];
    uint32_t* sel = p->sort_val[cur];
    double* wt = reinterpret_cast<double*>(p->sort_key[cur ^ 1]);
    if (serial) {
        k_resample_count_serial<T><<<gr, 128, 0, c->stream>>>(a, pop_view<T>(p), p->seg_a, c->d_status);
        MCS_CK_LAUNCH(c);
    } else {
        MCS_CK(c, cudaMemsetAsync(merge_n, 0, sizeof(unsigned long long), c->stream));
        k_resample_count<T><<<gr, 128, 0, c->stream>>>(a, pop_view<T>(p), p->seg_a, p->u32b, merge_n);
        MCS_CK_LAUNCH(c);
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_resample_merge_count<T>, RS_WARPS * 32, 0);
        k_resample_merge_count<T><<<std::max(occ, 1) * c->num_sms, RS_WARPS * 32, 0, c->stream>>>(
            a, pop_view<T>(p), p->seg_a, p->u32b, merge_n, sel, wt);
        MCS_CK_LAUNCH(c);
    }
    if (int st = launch_scan(p, p->seg_a, p->seg_b, nseg, total)) return st;
    PopView<T> P = pop_view<T>(p);
    if (serial) {
        k_resample_write_serial<T><<<gr, 128, 0, c->stream>>>(a, P, p->seg_b, total, c->d_status);
    } else {
        int occ = 0;   // the warp-per-cell write pass: all blocks resident, grid-stride over cells
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_resample_write<T>, RS_WARPS * 32, 0);
        k_resample_write<T><<<std::max(occ, 1) * c->num_sms, RS_WARPS * 32, 0, c->stream>>>(
            a, P, p->seg_a, p->seg_b, p->u32b, merge_n, sel, wt, total, c->d_status);
    }
    MCS_CK_LAUNCH(c);
    p->cur ^= 1;
    return MCS_OK;
}

}  // namespace mcs

using namespace mcs;

extern "C" {

MCS_API int mcs_sort_cells(mcs_pop* p, mcs_grid* g) {
    if (!p || !g) return MCS_ERR_ARG;
    if (p->cells && p->cells != g) return set_err(p->ctx, MCS_ERR_UNSUPPORTED, "sort by another mesh");
    if (cudaSetDevice(p->ctx->device) != cudaSuccess) return MCS_ERR_CUDA;
    return p->precision == MCS_FP32 ? sort_cells_t<float>(p, g, nullptr) : sort_cells_t<double>(p, g, nullptr);
}

MCS_API int mcs_resample_reserve(mcs_pop* p) {
    if (!p) return MCS_ERR_ARG;
    if (cudaSetDevice(p->ctx->device) != cudaSuccess) return MCS_ERR_CUDA;
    return reserve_sort_scratch(p, true);
}

MCS_API int mcs_resample_cells(mcs_pop* p, mcs_grid* g, int ntarget, int nmax) {
    if (!p || !g || ntarget < 1 || nmax < 1) return MCS_ERR_ARG;
    if (p->cells && p->cells != g) return set_err(p->ctx, MCS_ERR_UNSUPPORTED, "resample on another mesh");
    if (cudaSetDevice(p->ctx->device) != cudaSuccess) return MCS_ERR_CUDA;
    return p->precision == MCS_FP32 ? resample_cells_t<float>(p, g, ntarget, nmax)
                                    : resample_cells_t<double>(p, g, ntarget, nmax);
}

}  // extern "C"
