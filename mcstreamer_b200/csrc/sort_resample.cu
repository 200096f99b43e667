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
// mcs_resample_cells: after the sort every cell is a contiguous segment.  One thread per
// segment restates resample.jl's two passes serially in slot order (so the weight sums and
// the roulette sequence are the reference's), first only counting the clones, then -- after
// a scan of the counts gives each cell its place -- writing them.  Clones are appended in
// cell order, which is the slot order of the sorted population (the serial reference's
// append order).  Uniforms: one Philox stream per cell, ctr = {cell, call, k/4, tag}.
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
// tile and counts its keys per digit (warp match-any, the digit group's first lane adds);
// a block prefix of those counts gives every key its place in the tile sorted by digit
// (stable), where it is put in shared memory; the tile then goes out in that order, so that
// consecutive threads write consecutive slots of each digit's run.  Four barriers per tile.
__global__ void __launch_bounds__(SB) k_scatter(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
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
#pragma unroll
        for (int r = 0; r < SI; ++r) {
            const long long i = base + (long long)r * 32 + lane;
            k[r] = i < n ? kin[i] : 0u;
            const uint32_t dg = i < n ? ((k[r] >> shift) & 0xffu) : 0x100u;
            const unsigned peers = __match_any_sync(0xffffffffu, dg);
            if (dg < RADIX && (peers & lt) == 0) wc[wid][dg] += __popc(peers);
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
#pragma unroll
        for (int r = 0; r < SI; ++r) {
            const long long i = base + (long long)r * 32 + lane;
            const uint32_t dg = i < n ? ((k[r] >> shift) & 0xffu) : 0x100u;
            const unsigned peers = __match_any_sync(0xffffffffu, dg);
            uint32_t pos = 0;
            if (dg < RADIX) pos = loc[dg] + wc[wid][dg] + __popc(peers & lt);
            __syncwarp();
            if (dg < RADIX) {
                if ((peers & lt) == 0) wc[wid][dg] += __popc(peers);
                skey[pos] = k[r];
                sval[pos] = vin[i];
            }
            __syncwarp();
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

template <typename T>
__global__ void k_gather(PopView<T> P, const uint32_t* __restrict__ perm, DstArrays d) {
    const long long n = *P.n_in;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
        const uint32_t s = perm[j];
#pragma unroll
        for (int q = 0; q < 8; ++q) static_cast<T*>(d.f[q])[j] = P.f[q][s];
        if (d.cell) d.cell[j] = P.cell[s];
        d.act[j] = P.act[s];
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
//  * merge cells (p > nmax): the serial pass (FP64 weight sums in index order, the clone
//    positions x) runs on lane 0 over the cell's weights staged in shared memory, and
//    records the clone sources; the warp then writes the clones to consecutive slots and
//    removes the originals.
// ---------------------------------------------------------------------------------------
constexpr int RS_WARPS = 8;       // warps per block
constexpr int RS_BUF = 256;       // staged weights per warp (a cell is streamed in chunks)
constexpr int RS_SRC = 128;       // clone sources a merge can record (ntarget above: serial path)

struct RsShared {
    double w[RS_WARPS][RS_BUF];
    double f[RS_WARPS][RS_SRC];      // merge: f_k = samplemin(ntarget - k) of the cell's draw k
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

// A merging cell (p > nmax) by one warp.  The sample positions of resample.jl:48-52 follow
// x_1 = samplemin(ntarget) and x_(k+1) = x_k + samplemin(ntarget - k) (1 - x_k), where
// samplemin draws the cell's k-th uniform: every factor f_k = 1 - (1 - U_k)^(1/(ntarget - k))
// depends on the draw alone, so the lanes compute them side by side (the pows), and lane 0
// runs the two serial passes over the staged weights with additions and products only --
// unfused, in the reference's order -- recording the clone sources.  The warp then writes
// the clones to consecutive slots and removes the originals.
template <typename T, bool WRITE>
__device__ uint32_t merge_segment_warp(const ResampleArgs& a, PopView<T>& P, long long b, long long e, uint32_t cell,
                                       long long clone_base, long long cap, uint32_t* status, RsShared& sh,
                                       int wid) {
    const int lane = threadIdx.x & 31;
    double* wb = sh.w[wid];
    double* fk = sh.f[wid];
    uint32_t* src = sh.src[wid];
    const uint32_t k0 = (uint32_t)a.seed, k1 = (uint32_t)(a.seed >> 32);
    for (int k = lane; k < a.ntarget; k += 32) {
        // word k of the cell's stream {cell, call, k/4, TAG_CELL_RESAMPLE}
        const U4 blk = philox10(U4{cell, a.call, (uint32_t)k >> 2, TAG_CELL_RESAMPLE}, k0, k1);
        const uint32_t q = (uint32_t)k & 3u;
        const uint32_t w = q == 0 ? blk.x : q == 1 ? blk.y : q == 2 ? blk.z : blk.w;
        fk[k] = 1.0 - pow(1.0 - uni64(w), 1.0 / (double)(a.ntarget - k));
    }
    double wtotal = 0.0, x = 0.0;
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
                while (__dmul_rn(wtotal, x) < __dadd_rn(wcum, wj) && pk < a.ntarget) {
                    pk += 1;
                    src[ncl++] = (uint32_t)(c0 - b + q);
                    if (pk < a.ntarget) x = __dadd_rn(x, __dmul_rn(fk[pk], __dadd_rn(1.0, -x)));
                }
                wcum = __dadd_rn(wcum, wj);
            }
        }
    }
    __syncwarp();
    ncl = __shfl_sync(0xffffffffu, ncl, 0);
    if (WRITE) {
        wtotal = __shfl_sync(0xffffffffu, wtotal, 0);
        const T wc = (T)(wtotal / (double)a.ntarget);
        for (uint32_t k = lane; k < ncl; k += 32) {
            const long long d = clone_base + k;
            if (d < cap) copy_clone<T>(P, d, b + src[k], wc);
            else atomicOr(status, ST_CAPACITY);
        }
        for (long long j = b + lane; j < e; j += 32) P.act[j] = 0;   // remove_particle!
    }
    __syncwarp();
    return ncl;
}

// Returns the number of clones of segment s (the same on every lane).
template <typename T, bool WRITE>
__device__ uint32_t resample_segment_warp(const ResampleArgs& a, PopView<T>& P, long long s, long long nseg,
                                          long long clone_base, long long cap, uint32_t* status, RsShared& sh,
                                          int wid) {
    const int lane = threadIdx.x & 31;
    const long long b = a.start[s];
    const uint32_t cell = a.key[b];
    const long long e = segment_end(a, s, nseg, b, cell);
    const long long p0 = e - b;
    // (the host takes the serial form when ntarget > nmax or ntarget > RS_SRC)
    if (p0 < a.ntarget) {
        // split: rank the particles with w > 2 in index order
        const uint32_t K = (uint32_t)(a.ntarget - p0);
        uint32_t ranked = 0;
        for (long long j0 = b; j0 < e && ranked < K; j0 += 32) {
            const long long j = j0 + lane;
            double wj = 0.0;
            bool q = false;
            if (j < e) {
                wj = (double)P.f[6][j];
                q = wj > 2;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, q);
            const uint32_t r = ranked + __popc(bal & ((1u << lane) - 1u));
            if (WRITE && q && r < K) {
                const double wnew = rint(wj / 2.0);   // Julia round: nearest, ties to even
                const long long d = clone_base + r;
                if (d < cap) copy_clone<T>(P, d, j, (T)wnew);
                else atomicOr(status, ST_CAPACITY);
                P.f[6][j] = (T)(wj - wnew);
            }
            ranked += __popc(bal);
        }
        return ranked < K ? ranked : K;
    }
    if (p0 <= a.nmax) return 0;
    return merge_segment_warp<T, WRITE>(a, P, b, e, cell, clone_base, cap, status, sh, wid);
}

// Counting is latency-bound over millions of small segments: a thread per segment keeps 32
// segments' loads in flight per warp.
// Only merging cells need the serial pass; their segments go to a worklist for the warp
// kernel below.  A splitting cell (p < ntarget) clones its first ntarget - p particles with
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

template <typename T>
__global__ void __launch_bounds__(RS_WARPS * 32, 4) k_resample_merge_count(ResampleArgs a, PopView<T> P,
                                                                         uint32_t* __restrict__ counts,
                                                                         const uint32_t* __restrict__ merge_list,
                                                                         const unsigned long long* merge_n) {
    __shared__ RsShared sh;
    const long long nm = (long long)*merge_n;
    const long long n = *a.n;
    const long long nseg = *a.nseg;
    const int wid = threadIdx.x >> 5;
    const long long w0 = (long long)blockIdx.x * RS_WARPS + wid, ws = (long long)gridDim.x * RS_WARPS;
    for (long long q = w0; q < nm; q += ws) {
        const long long s = merge_list[q];
        const long long b = a.start[s];
        const uint32_t cell = a.key[b];
        const long long e = segment_end(a, s, nseg, b, cell);
        (void)n;
        const uint32_t c = merge_segment_warp<T, false>(a, P, b, e, cell, 0, 0, nullptr, sh, wid);
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

template <typename T>
__global__ void __launch_bounds__(RS_WARPS * 32, 4) k_resample_write(ResampleArgs a, PopView<T> P,
                                                                   const uint32_t* __restrict__ offs,
                                                                   const long long* total, uint32_t* status) {
    __shared__ RsShared sh;
    const long long nseg = *a.nseg;
    const long long n = *a.n;
    const int wid = threadIdx.x >> 5;
    const long long w0 = (long long)blockIdx.x * RS_WARPS + wid, ws = (long long)gridDim.x * RS_WARPS;
    for (long long s = w0; s < nseg; s += ws)
        resample_segment_warp<T, true>(a, P, s, nseg, n + (long long)offs[s], P.cap, status, sh, wid);
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
    k_gather<T><<<gr, 256, 0, c->stream>>>(pop_view<T>(p), p->sort_val[cur], d);
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
    if (ntarget > nmax || ntarget > RS_SRC) {
        k_resample_count_serial<T><<<gr, 128, 0, c->stream>>>(a, pop_view<T>(p), p->seg_a, c->d_status);
        MCS_CK_LAUNCH(c);
    } else {
        // merging cells hold more than nmax particles each: at most n / (nmax + 1) of them
        unsigned long long* merge_n = reinterpret_cast<unsigned long long*>(p->counters + 14);
        MCS_CK(c, cudaMemsetAsync(merge_n, 0, sizeof(unsigned long long), c->stream));
        k_resample_count<T><<<gr, 128, 0, c->stream>>>(a, pop_view<T>(p), p->seg_a, p->u32b, merge_n);
        MCS_CK_LAUNCH(c);
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_resample_merge_count<T>, RS_WARPS * 32, 0);
        k_resample_merge_count<T><<<std::max(occ, 1) * c->num_sms, RS_WARPS * 32, 0, c->stream>>>(
            a, pop_view<T>(p), p->seg_a, p->u32b, merge_n);
        MCS_CK_LAUNCH(c);
    }
    if (int st = launch_scan(p, p->seg_a, p->seg_b, nseg, total)) return st;
    PopView<T> P = pop_view<T>(p);
    if (ntarget > nmax || ntarget > RS_SRC) {
        k_resample_write_serial<T><<<gr, 128, 0, c->stream>>>(a, P, p->seg_b, total, c->d_status);
    } else {
        int occ = 0;   // the warp-per-segment write pass: all blocks resident, grid-stride over segments
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_resample_write<T>, RS_WARPS * 32, 0);
        k_resample_write<T><<<std::max(occ, 1) * c->num_sms, RS_WARPS * 32, 0, c->stream>>>(a, P, p->seg_b, total,
                                                                                              c->d_status);
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
