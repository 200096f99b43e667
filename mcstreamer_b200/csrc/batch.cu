// batch.cu -- many swarm solves on one GPU: the Swarm.swarm time loop (Swarm/src/Swarm.jl:
// 124-142) of every instance advanced together by persistent kernels.
//
// All instances live in one FP32 structure-of-arrays population, each in its own slot
// region [base, base + cap).  Descriptors (gas table, field, seed, resampling target),
// counts, step counters and per-step moments are device-resident, so a whole batched step
// -- plan, advance!, Swarm.resample!, repack! -- is a fixed kernel sequence that is
// captured once into a CUDA graph and replayed; instances join and leave between steps by
// editing descriptors (continuous batching).
//
// Every pass walks one global list of tiles: a plan kernel prefixes the per-instance tile
// counts, and a CTA maps its ticket to (instance, local tile) by binary search.  Ordered
// appends (secondaries, clones) and the compaction scan use decoupled look-back bounded to
// the instance's first tile, and random streams are keyed by the instance seed and the
// instance-local slot, so each instance evolves exactly as it does alone through
// mcs_swarm_run with repack_every = 1.
#include <algorithm>
#include <cstring>
#include <vector>

#include "host_util.h"
#include "pop_ops.h"
#include "step_kernel.cuh"

namespace mcs {

constexpr int kMaxGases = 16;
constexpr int kBatchLog = MCS_BATCH_LOG;  // per-instance ring of per-step sums
constexpr int kBM = MCS_BATCH_MOMENTS;  // the 12 step sums + sum nu_ion, sum nu_ion^2
constexpr int kRBlock = 256;        // threads of the resample / repack passes
constexpr int kRItems = 16;         // contiguous slots per thread (one 16-byte load of flags)
constexpr int kRTile = kRBlock * kRItems;
constexpr int kSlotAlign = 16;      // instance regions start on 16-slot boundaries

// Passes of a batched step (what the plan tiles over, per instance):
//   PASS_STEP      advance! over [0, n)
//   PASS_RESAMPLE  Swarm.resample! decisions + clone append over [0, n), survivors counted
//   PASS_HOLES     repack!: inactive slots below A (A = actives) -> hole list
//   PASS_MOVE      repack!: actives at or above A, from the end, -> holes
enum : int { PASS_STEP = 0, PASS_RESAMPLE = 1, PASS_HOLES = 2, PASS_MOVE = 3 };
enum : int { MODE_SKIP = 0, MODE_DROP = 1, MODE_CLONE = 2 };

struct Inst {
    long long base, cap;
    unsigned long long seed;
    float ax, ay, az;
    int table;
    int live;
    int sel_row;                    // table row whose rate is averaged (ionization), -1 = none
    long long n0;
    double tol;
};

struct BatchDev {
    float* f[8];
    uint8_t* act;
    Inst* inst;
    long long* n0buf;               // n[0][k]
    long long* n1buf;               // n[1][k]
    uint32_t* step;
    long long* tstart;              // [K + 1]
    uint32_t* done;
    double* tpart;                  // [tiles][kBM]
    double* curm;                   // [K][kBM] moments of the last step
    double* log;                    // [K][kBatchLog][kBM]
    uint32_t* logpos;
    unsigned long long* tstatus;
    uint32_t* counters;             // [0] ticket, [1] CTA done, [2] epoch
    uint32_t* status;
    const TableView* tabs;
    uint32_t* holes;                // repack hole list (region-local slots), per slot
    uint32_t* tile_inst;            // instance of each tile of the current pass
    long long* rlo;                 // [K] first slot of the pass's range per instance
    long long* tot;                 // [K] clones appended by Swarm.resample!
    long long* actives;             // [K] actives after Swarm.resample! (A of repack!)
    uint8_t* mode;                  // [K] MODE_* of this step's Swarm.resample!
    int K;
    uint32_t flags;
    char* stage;
    unsigned long long stage_stride;
    uint32_t stage_cap;
    double dt;
};

// ---------------------------------------------------------------------------------------
// Plan of one pass: per instance a slot range [lo, hi) (see PASS_*), its tiles prefixed
// over instances (tstart), the tile -> instance map, and the pass's per-instance setup;
// advances the ordered-append epoch.  One block of 1024 threads.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ int resample_mode(const Inst& I, double ncur_d) {
    const long long ncur = (long long)ncur_d;
    if (I.n0 <= 0 || ncur == 0 || fabs((double)(ncur - I.n0) / (double)I.n0) < I.tol) return MODE_SKIP;
    return ncur > I.n0 ? MODE_DROP : MODE_CLONE;
}

// Slot range of instance k in a pass (after the pass's setup in k_bplan).
__device__ __forceinline__ void pass_range(const BatchDev& B, int pass, int k, long long& lo, long long& hi) {
    const int live = B.inst[k].live;
    lo = 0;
    if (pass == PASS_STEP) { hi = live ? B.n0buf[k] : 0; return; }
    if (pass == PASS_RESAMPLE) { hi = live ? B.n1buf[k] : 0; return; }
    const long long A = B.actives[k], n = B.n0buf[k];
    const bool need = live && A < n;
    if (pass == PASS_HOLES) { hi = need ? A : 0; return; }
    lo = A;
    hi = need ? n : A;
}

__global__ void __launch_bounds__(1024) k_bplan(BatchDev B, int pass, int tile) {
    __shared__ long long wsum[32];
    const int per = (B.K + 1023) / 1024;
    long long loc = 0;
    for (int q = 0; q < per; ++q) {
        const int k = threadIdx.x * per + q;
        if (k >= B.K) break;
        if (pass == PASS_STEP) {
            B.n1buf[k] = B.n0buf[k];
            B.done[k] = 0;
        } else if (pass == PASS_RESAMPLE) {
            const Inst I = B.inst[k];
            B.n0buf[k] = B.n1buf[k];
            B.tot[k] = 0;
            B.actives[k] = 0;
            B.mode[k] = (uint8_t)(I.live ? resample_mode(I, B.curm[(long long)k * kBM + SM_COUNT]) : MODE_SKIP);
        }
        long long lo, hi;
        pass_range(B, pass, k, lo, hi);
        B.rlo[k] = lo;
        loc += (hi - lo + tile - 1) / tile;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    long long incl = loc;
    for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long a = 0;
        for (int w = 0; w < 32; ++w) { const long long t = wsum[w]; wsum[w] = a; a += t; }
        B.tstart[B.K] = a;
        B.counters[2] += 1;
        if ((B.counters[2] & 0x3fffffffu) == 0) B.counters[2] += 1;
    }
    __syncthreads();
    long long run = wsum[wid] + incl - loc;
    for (int q = 0; q < per; ++q) {
        const int k = threadIdx.x * per + q;
        if (k >= B.K) break;
        B.tstart[k] = run;
        long long lo, hi;
        pass_range(B, pass, k, lo, hi);
        const long long nt = (hi - lo + tile - 1) / tile;
        for (long long t = 0; t < nt; ++t) B.tile_inst[run + t] = (uint32_t)k;
        run += nt;
    }
}

// Rate of row j at energy v2 (FP32 table), for the per-step rate estimator (collrate).
__device__ __forceinline__ float rate_row32(const TableView& t, float v2, int j) {
    const float u = fmaf(v2, t.ke32, -t.e0n32);
    int k = (int)u;
    float w;
    if (!(u >= 0.0f && k <= t.neps - 2)) { k = u >= 0.0f ? t.neps - 2 : 0; w = u >= 0.0f ? 0.0f : 1.0f; }
    else w = (float)(k + 1) - u;
    const float a = __ldg(t.rate32 + (size_t)k * t.nrp + 1 + j), b = __ldg(t.rate32 + (size_t)(k + 1) * t.nrp + 1 + j);
    return fmaf(w, a - b, b);
}

template <int BLOCK>
struct BShared {
    RowsSmem<float> rows;
    double red[BLOCK / 32][kBM];
    uint32_t wtot[BLOCK / 32];
    Inst I;
    TableView tab;
    long long tile, first, ntl, n_entry;
    uint32_t count, excl, next;
    int k, ok, last;
    // the CTA's previous tile, whose secondaries wait in ranked buffer pend_par for their
    // place after the instance (pend < 0: none); par is the current tile's buffer
    long long pend, pend_first, pend_n_entry, pend_base, pend_cap;
    uint32_t pend_c;
    int pend_k, pend_last, pend_par, par;
};

// Per-CTA slice of the step's staging memory: the staging buffer of stage() (cap entries,
// unordered), then two ranked buffers (cap entries each: a tile's secondaries at their
// serial rank within the tile).
__host__ __device__ inline size_t bstage_bytes(uint32_t cap) { return ((size_t)cap * (8 * sizeof(float) + 9) + 255) & ~(size_t)255; }
__host__ __device__ inline size_t brank_bytes(uint32_t cap) { return ((size_t)cap * (8 * sizeof(float) + 1) + 255) & ~(size_t)255; }

struct RankBuf {
    float* f[8];
    uint8_t* act;
    __device__ __forceinline__ void init(const BatchDev& B, int par) {
        char* b = B.stage + (unsigned long long)blockIdx.x * B.stage_stride + bstage_bytes(B.stage_cap) +
                  (size_t)par * brank_bytes(B.stage_cap);
#pragma unroll
        for (int q = 0; q < 8; ++q) f[q] = reinterpret_cast<float*>(b + (size_t)q * B.stage_cap * sizeof(float));
        act = reinterpret_cast<uint8_t*>(b + (size_t)8 * B.stage_cap * sizeof(float));
    }
};

// Append the CTA's pending tile: wait (bounded) for the prefix of the instance's tiles
// before it -- they published their counts when their particles were done, and have had a
// whole tile of this CTA's time since -- and copy its ranked buffer to its place.
template <int BLOCK>
__device__ __forceinline__ void bappend_pending(const BatchDev& B, BShared<BLOCK>& sh, uint32_t epoch) {
    // every thread reads the pending tile before any goes on: with no pending tile the
    // caller's thread 0 next makes this tile the pending one, and a thread that read
    // sh.pend after that write would enter the append alone, out of step with the barriers
    const bool none = sh.pend < 0;
    __syncthreads();
    if (none) return;
    if (threadIdx.x < 32) {   // warp 0 looks back
        bool ok = true;
        uint32_t excl = 0;
        if (sh.pend != sh.pend_first)
            excl = tile_lookback_wait_warp(B.tstatus, (uint32_t)sh.pend_first, (uint32_t)sh.pend, epoch, sh.pend_c,
                                           B.status, &ok);
        if (threadIdx.x == 0) {
            sh.excl = excl;
            sh.ok = ok;
        }
    }
    if (threadIdx.x == 0) {
        const uint32_t excl = sh.excl;
        if (sh.pend_last) {
            long long nn = sh.pend_n_entry + (long long)excl + sh.pend_c;
            if (nn > sh.pend_cap) { nn = sh.pend_cap; atomicOr(B.status, ST_CAPACITY); }
            B.n1buf[sh.pend_k] = nn;
        }
    }
    __syncthreads();
    if (sh.ok) {
        RankBuf rb;
        rb.init(B, sh.pend_par);
        const long long d0 = sh.pend_n_entry + (long long)sh.excl;
        for (uint32_t r = threadIdx.x; r < sh.pend_c; r += BLOCK) {
            const long long dl = d0 + r;
            if (dl >= sh.pend_cap) { atomicOr(B.status, ST_CAPACITY); continue; }
            const long long d = sh.pend_base + dl;
#pragma unroll
            for (int q = 0; q < 8; ++q) B.f[q][d] = rb.f[q][r];
            B.act[d] = rb.act[r];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) sh.pend = -1;
    __syncthreads();
}

// ---------------------------------------------------------------------------------------
// Batched advance! (FP32, uniform field per instance, closed-form push between real
// collisions): the body of k_step_abs<float,...,CLOSED> with instance indirection.
// ---------------------------------------------------------------------------------------
template <int BLOCK, int PPT, int MINB, int REFILL>
__global__ void __launch_bounds__(BLOCK, MINB) k_bstep(BatchDev B) {
    constexpr int TILE = BLOCK * PPT;
    __shared__ BShared<BLOCK> sh;
    __shared__ uint32_t cnt[TILE];
    const long long T = B.tstart[B.K];
    const uint32_t epoch = B.counters[2];
    Stage<float> sg;
    {
        StepCtl C0{};
        C0.stage = B.stage;
        C0.stage_stride = B.stage_stride;
        C0.stage_cap = B.stage_cap;
        sg.init(C0);
    }
    StepCtl C{};
    C.flags = B.flags;
    C.status = B.status;
    C.tag = TAG_ADVANCE;
    if (threadIdx.x == 0) {
        sh.pend = -1;
        sh.par = 0;
    }
    for (;;) {
        if (threadIdx.x == 0) {
            const long long g = atomicAdd(&B.counters[0], 1u);
            sh.tile = g;
            sh.count = 0;
            sh.next = 0;
            if (g < T) {
                const int k = (int)B.tile_inst[g];
                sh.k = k;
                sh.I = B.inst[k];
                sh.tab = B.tabs[sh.I.table];
                sh.first = B.tstart[k];
                sh.ntl = B.tstart[k + 1] - B.tstart[k];
                sh.n_entry = B.n0buf[k];
            }
        }
        __syncthreads();
        const long long g = sh.tile;
        if (g >= T) break;
        load_rows(sh.rows, sh.tab);
        __syncthreads();
        const int k = sh.k;
        const Inst& I = sh.I;
        const long long lt = g - sh.first;
        const long long n_entry = sh.n_entry;
        const uint32_t stepk = B.step[k];
        const float ax = I.ax, ay = I.ay, az = I.az;
        const TableView& tab = sh.tab;
        C.seed = I.seed;
        C.step = stepk;

        // Particle queue: each lane runs one sub-step per pass and takes the tile's next
        // particle when its own is done; finished lanes write back and refill together once
        // a quarter of the warp is idle, so the warp stays converged on the sub-step body.
        const long long rest = n_entry - lt * TILE;
        const uint32_t tile_n = rest < TILE ? (uint32_t)rest : (uint32_t)TILE;
        const long long tbase = I.base + lt * TILE;
        bool have = false, drained = false, pending = false;
        uint32_t local = 0;
        long long i = 0;
        Event rng;
        float x = 0.f, y = 0.f, z = 0.f, vx = 0.f, vy = 0.f, vz = 0.f, w = 0.f, tau = 0.f;
        double s = 0.0, trem = 0.0;
        uint8_t act = 1;
        uint32_t ev = 0;
        for (;;) {
            const unsigned idle = __ballot_sync(0xffffffffu, !have);
            if (idle != 0xffffffffu && __popc(idle) < REFILL) goto substep;
            if (!have && pending) {
                B.f[0][i] = x; B.f[1][i] = y; B.f[2][i] = z;
                B.f[3][i] = vx; B.f[4][i] = vy; B.f[5][i] = vz;
                B.f[7][i] = (float)s;
                if (!act) B.act[i] = 0;
                cnt[local] = ev;
                pending = false;
            }
            while (!have && !drained) {
                const uint32_t q = atomicAdd(&sh.next, 1u);
                if (q >= (uint32_t)TILE) { drained = true; break; }
                if (q >= tile_n || !B.act[tbase + q]) { cnt[q] = 0; continue; }
                local = q;
                i = tbase + q;
                rng.init(I.seed, (uint32_t)(lt * TILE + q), stepk, TAG_ADVANCE);
                x = B.f[0][i]; y = B.f[1][i]; z = B.f[2][i];
                vx = B.f[3][i]; vy = B.f[4][i]; vz = B.f[5][i];
                w = B.f[6][i];
                s = (double)B.f[7][i];
                act = 1;
                ev = 0;
                tau = 0.f;
                trem = B.dt;
                if (!(trem > 0)) { cnt[q] = 0; continue; }   // dt == 0: state unchanged
                // the first sub-step's decision; an electron with no collision in the step
                // flies to its end and is written back here
                if (trem > s * tab.inv_maxrate) {
                    have = true;
                } else {
                    const double t = trem;
                    s -= t * tab.maxrate;
                    tau += (float)t;
                    trem -= t;
                    const float h2 = 0.5f * tau * tau;
                    B.f[0][i] = fmaf(ax, h2, fmaf(vx, tau, x));
                    B.f[1][i] = fmaf(ay, h2, fmaf(vy, tau, y));
                    B.f[2][i] = fmaf(az, h2, fmaf(vz, tau, z));
                    B.f[3][i] = fmaf(ax, tau, vx); B.f[4][i] = fmaf(ay, tau, vy); B.f[5][i] = fmaf(az, tau, vz);
                    B.f[7][i] = (float)s;
                    cnt[q] = 0;
                }
            }
            if (!__any_sync(0xffffffffu, have)) break;
        substep:
            if (!have) continue;
            {
                // one collision sub-step of advance! with the closed-form push of a uniform
                // field (have: the next collision falls inside the step), then the next
                // sub-step's decision; the free flight to the step's end finishes here, so an
                // electron takes one loop pass per collision.  The FP64 time arithmetic is
                // that of the sub-step sequence of advance!, operation for operation.
                const double t = s * tab.inv_maxrate;
                tau += (float)t;
                {
                    float cvx = fmaf(ax, tau, vx), cvy = fmaf(ay, tau, vy), cvz = fmaf(az, tau, vz);
                    Sec<float> sec;
                    const int out = collide_once<float>(sh.rows, tab, C, rng, cvx, cvy, cvz, sec);
                    if (out == OUT_PHOTO) atomicOr(C.status, ST_UNSUPPORTED);
                    if (out != OUT_NONE) {
                        const float h2 = 0.5f * tau * tau;
                        x = fmaf(ax, h2, fmaf(vx, tau, x));
                        y = fmaf(ay, h2, fmaf(vy, tau, y));
                        z = fmaf(az, h2, fmaf(vz, tau, z));
                        tau = 0.0f;
                        vx = cvx; vy = cvy; vz = cvz;
                    }
                    if (out == OUT_NEW) {
                        const float vals[8] = {x, y, z, sec.vx, sec.vy, sec.vz, w, sec.s};
                        stage(sg, &sh.count, local, ev++, vals, 0u, act, B.status);
                    } else if (out == OUT_REMOVE) {
                        act = 0;
                    }
                    s = (double)M<float>::nlog(uni32(rng.b.y));
                }
                trem -= t;   // > 0: the collision was strictly inside the step
                if (!(trem > s * tab.inv_maxrate)) {
                    const double tf = trem;
                    s -= tf * tab.maxrate;
                    tau += (float)tf;
                    trem -= tf;
                    const float h2 = 0.5f * tau * tau;
                    x = fmaf(ax, h2, fmaf(vx, tau, x));
                    y = fmaf(ay, h2, fmaf(vy, tau, y));
                    z = fmaf(az, h2, fmaf(vz, tau, z));
                    vx = fmaf(ax, tau, vx); vy = fmaf(ay, tau, vy); vz = fmaf(az, tau, vz);
                    have = false;
                    pending = true;
                }
            }
        }
        __syncthreads();

        // ---- this tile's secondaries: serial ranks within the tile, the tile's count
        // published at once (no wait), and the secondaries in the tile's ranked buffer ----
        uint32_t c = sh.count;
        if (c > sg.cap) c = sg.cap;
        {
            constexpr int PER = TILE / BLOCK;
            const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
            uint32_t v[PER];
            uint32_t sum = 0;
#pragma unroll
            for (int q = 0; q < PER; ++q) { v[q] = cnt[threadIdx.x * PER + q]; sum += v[q]; }
            uint32_t incl = sum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t yv = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += yv;
            }
            if (lane == 31) sh.wtot[wid] = incl;
            __syncthreads();
            if (threadIdx.x == 0) {
                uint32_t acc = 0;
                for (int q = 0; q < BLOCK / 32; ++q) { const uint32_t tq = sh.wtot[q]; sh.wtot[q] = acc; acc += tq; }
                // the instance's first tile knows its prefix (0): inclusive; the others their
                // aggregate, which the tiles after them sum in their look-back
                st_release_u64(&B.tstatus[g], tile_word(epoch, g == sh.first ? 2 : 1, c));
            }
            __syncthreads();
            uint32_t run = sh.wtot[wid] + incl - sum;
#pragma unroll
            for (int q = 0; q < PER; ++q) { cnt[threadIdx.x * PER + q] = run; run += v[q]; }
            __syncthreads();
        }
        RankBuf rb;
        rb.init(B, sh.par);
        for (uint32_t e = threadIdx.x; e < c; e += BLOCK) {
            const uint32_t key = sg.key[e];
            const uint32_t r = cnt[key >> 16] + (key & 0xffffu);
            if (r >= c) continue;   // only when staging overflowed (ST_OVERFLOW raised)
#pragma unroll
            for (int q = 0; q < 8; ++q) rb.f[q][r] = sg.f[q][e];
            rb.act[r] = sg.act[e];
        }

        // ---- tile moments (post-step actives incl. secondaries) ----
        {
            double m[kBM];
#pragma unroll
            for (int q = 0; q < kBM; ++q) m[q] = 0.0;
            auto add = [&](double x, double y, double z, float fvx, float fvy, float fvz, double w) {
                mom_add(m, x, y, z, (double)fvx, (double)fvy, (double)fvz, w);
                if (I.sel_row >= 0) {
                    const double r = rate_row32(tab, fmaf(fvx, fvx, fmaf(fvy, fvy, fvz * fvz)), I.sel_row);
                    m[kStepMoments] = __dadd_rn(m[kStepMoments], r);
                    m[kStepMoments + 1] = __fma_rn(r, r, m[kStepMoments + 1]);
                }
            };
            for (int jj = 0; jj < PPT; ++jj) {
                const long long il = lt * TILE + jj * BLOCK + threadIdx.x;
                const long long i = I.base + il;
                if (il < n_entry && B.act[i])
                    add(B.f[0][i], B.f[1][i], B.f[2][i], B.f[3][i], B.f[4][i], B.f[5][i], B.f[6][i]);
            }
            // secondaries in their serial order, from the ranked buffer
            __syncthreads();
            for (uint32_t r = threadIdx.x; r < c; r += BLOCK)
                if (rb.act[r]) add(rb.f[0][r], rb.f[1][r], rb.f[2][r], rb.f[3][r], rb.f[4][r], rb.f[5][r], rb.f[6][r]);
            const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
            for (int q = 0; q < kBM; ++q) {
                const double vq = warp_sum(m[q]);
                if (lane == 0) sh.red[wid][q] = vq;
            }
            __syncthreads();
            if (threadIdx.x < kBM) {
                double a = 0.0;
                for (int w2 = 0; w2 < BLOCK / 32; ++w2) a += sh.red[w2][threadIdx.x];
                B.tpart[g * kBM + threadIdx.x] = a;
            }
            __syncthreads();
        }
        // ---- the CTA that completes an instance's last tile reduces its moments ----
        if (threadIdx.x == 0) {
            __threadfence();
            const uint32_t d = atomicAdd(&B.done[k], 1u);
            sh.last = (d == (uint32_t)(sh.ntl - 1));
        }
        __syncthreads();
        if (sh.last) {
            // Same order as the single-population epilogue: Kahan over strided tiles per
            // thread, then the fixed warp/block reduction.
            __threadfence();
            const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
            double m[kBM];
#pragma unroll
            for (int q = 0; q < kBM; ++q) {
                double a = 0.0, comp = 0.0;
                for (long long t2 = threadIdx.x; t2 < sh.ntl; t2 += BLOCK) {
                    const double yv = B.tpart[(sh.first + t2) * kBM + q] - comp;
                    const double s2 = a + yv;
                    comp = (s2 - a) - yv;
                    a = s2;
                }
                m[q] = a;
            }
#pragma unroll
            for (int q = 0; q < kBM; ++q) {
                const double vq = warp_sum(m[q]);
                if (lane == 0) sh.red[wid][q] = vq;
            }
            __syncthreads();
            if (threadIdx.x < kBM) {
                double a = 0.0;
                for (int w2 = 0; w2 < BLOCK / 32; ++w2) a += sh.red[w2][threadIdx.x];
                B.curm[(long long)k * kBM + threadIdx.x] = a;
                B.log[((long long)k * kBatchLog + (B.logpos[k] % kBatchLog)) * kBM + threadIdx.x] = a;
            }
        }
        __syncthreads();
        // ---- the CTA's previous tile goes to its place; this one becomes pending ----
        bappend_pending<BLOCK>(B, sh, epoch);
        if (threadIdx.x == 0) {
            sh.pend = g;
            sh.pend_first = sh.first;
            sh.pend_n_entry = n_entry;
            sh.pend_base = I.base;
            sh.pend_cap = I.cap;
            sh.pend_c = c;
            sh.pend_k = k;
            sh.pend_last = lt == sh.ntl - 1;
            sh.pend_par = sh.par;
            sh.par ^= 1;
        }
        __syncthreads();
    }
    bappend_pending<BLOCK>(B, sh, epoch);
    // re-arm the ticket for the next pass
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t d = atomicAdd(&B.counters[1], 1u);
        if (d == gridDim.x - 1) {
            B.counters[0] = 0;
            B.counters[1] = 0;
        }
    }
}

// Instances with no particle (no tiles) still publish empty moments.
__global__ void k_bempty_moments(BatchDev B) {
    const long long T = B.tstart[B.K];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < B.K; k += gridDim.x * blockDim.x) {
        const long long nt = (k + 1 < B.K ? B.tstart[k + 1] : T) - B.tstart[k];
        if (nt == 0 && B.inst[k].live)
            for (int q = 0; q < kBM; ++q) {
                B.curm[(long long)k * kBM + q] = 0.0;
                B.log[((long long)k * kBatchLog + (B.logpos[k] % kBatchLog)) * kBM + q] = 0.0;
            }
    }
}


__device__ __forceinline__ void bcopy_slot(const BatchDev& B, long long dst, long long src) {
#pragma unroll
    for (int q = 0; q < 8; ++q) B.f[q][dst] = B.f[q][src];
    B.act[dst] = B.act[src];
}

// Tile header shared by the resample / repack passes: the next ticket and its instance.
struct RShared {
    long long g, first, ntl, base, lo, n, cap, A;
    unsigned long long seed;
    double pdrop, lam;
    uint32_t step1, excl;
    int k, mode, ok;
    uint32_t wtot[kRBlock / 32];
    uint32_t wtot2[kRBlock / 32];
};

__device__ __forceinline__ bool rtile_next(const BatchDev& B, RShared& sh, int pass) {
    if (threadIdx.x == 0) {
        const long long g = atomicAdd(&B.counters[0], 1u);
        sh.g = g;
        if (g < B.tstart[B.K]) {
            const int k = (int)B.tile_inst[g];
            const Inst I = B.inst[k];
            sh.k = k;
            sh.first = B.tstart[k];
            sh.ntl = B.tstart[k + 1] - sh.first;
            sh.base = I.base;
            sh.cap = I.cap;
            sh.lo = B.rlo[k];
            sh.seed = I.seed;
            if (pass == PASS_RESAMPLE) {
                sh.n = B.n1buf[k];
                sh.mode = B.mode[k];
                const double ncur = B.curm[(long long)k * kBM + SM_COUNT];
                sh.pdrop = (ncur - (double)I.n0) / ncur;
                sh.lam = ((double)I.n0 - ncur) / ncur;
                sh.step1 = B.step[k] + 1u;
            } else {
                sh.n = B.n0buf[k];
                sh.A = B.actives[k];
            }
        }
    }
    __syncthreads();
    return sh.g < B.tstart[B.K];
}

// Block-wide exclusive scan (slot order = thread order, kRItems consecutive slots per
// thread) of per-thread totals; returns this thread's offset, block total in *total.
__device__ __forceinline__ uint32_t rblock_scan(RShared& sh, uint32_t v, uint32_t* total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();   // the previous scan's readers are done with sh.wtot
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) sh.wtot[wid] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t a = 0;
        for (int q = 0; q < kRBlock / 32; ++q) { const uint32_t t = sh.wtot[q]; sh.wtot2[q] = a; a += t; }
        sh.wtot[0] = a;
    }
    __syncthreads();
    *total = sh.wtot[0];
    return sh.wtot2[wid] + incl - v;
}

__device__ __forceinline__ void rpass_done(const BatchDev& B) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t d = atomicAdd(&B.counters[1], 1u);
        if (d == gridDim.x - 1) { B.counters[0] = 0; B.counters[1] = 0; }
    }
}

// Active flags of this thread's kRItems slots starting at region-local l0 (slots at or
// beyond `lim` read as inactive).  Regions start on 16-slot boundaries and l0 is a multiple
// of 16, so one 16-byte load covers them.
__device__ __forceinline__ void load_flags(const BatchDev& B, long long base, long long l0, long long lim,
                                           uint8_t (&a)[kRItems]) {
    if (l0 >= lim) {
#pragma unroll
        for (int q = 0; q < kRItems; ++q) a[q] = 0;
        return;
    }
    const uint4 v = *reinterpret_cast<const uint4*>(B.act + base + l0);
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int q = 0; q < kRItems; ++q) a[q] = (l0 + q < lim) ? (uint8_t)((w[q >> 2] >> (8 * (q & 3))) & 0xffu) : 0;
}

// ---------------------------------------------------------------------------------------
// Swarm.resample!(popl, n0, tol) (Swarm/src/Swarm.jl:193-223) of every instance in one
// pass: roulette (drop mode) or Poisson clone counts (clone mode) from the stream
// {slot, step, k/4, TAG_SWARM_RESAMPLE}, the clones appended after the instance's particles
// in slot order (tile scan + look-back bounded to the instance's tiles), and the actives
// after resampling counted into B.actives (the A of repack!).
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kRBlock) k_bresample(BatchDev B) {
    __shared__ RShared sh;
    const uint32_t epoch = B.counters[2];
    for (;;) {
        if (!rtile_next(B, sh, PASS_RESAMPLE)) break;
        const long long lt = sh.g - sh.first;
        const long long l0 = lt * kRTile + (long long)threadIdx.x * kRItems;
        const long long n = sh.n, base = sh.base;
        uint8_t a[kRItems];
        load_flags(B, base, l0, n, a);
        uint32_t cnum[kRItems];
        uint32_t alive = 0, csum = 0;
#pragma unroll 1
        for (int q = 0; q < kRItems; ++q) {
            cnum[q] = 0;
            if (!a[q]) continue;
            if (sh.mode == MODE_DROP) {
                Rng r;
                r.init(sh.seed, (uint32_t)(l0 + q), sh.step1, TAG_SWARM_RESAMPLE);
                if (r.u64() < sh.pdrop) { B.act[base + l0 + q] = 0; continue; }
            } else if (sh.mode == MODE_CLONE) {
                Rng r;
                r.init(sh.seed, (uint32_t)(l0 + q), sh.step1, TAG_SWARM_RESAMPLE);
                cnum[q] = (uint32_t)poisson_draw(r, sh.lam);
                csum += cnum[q];
            }
            ++alive;
        }
        // survivors of the roulette; the clones actually written are added by the
        // instance's last tile below (clones are active)
        uint32_t tot_alive;
        rblock_scan(sh, alive, &tot_alive);
        if (threadIdx.x == 0 && tot_alive) atomicAdd(reinterpret_cast<unsigned long long*>(&B.actives[sh.k]),
                                                     (unsigned long long)tot_alive);
        if (sh.mode == MODE_CLONE) {
            uint32_t ctile;
            const uint32_t off = rblock_scan(sh, csum, &ctile);
            if (threadIdx.x < 32) {   // warp 0 looks back
                bool ok;
                const uint32_t ex =
                    tile_lookback_from_warp(B.tstatus, (uint32_t)sh.first, (uint32_t)sh.g, epoch, ctile, B.status, &ok);
                if (threadIdx.x == 0) {
                    sh.excl = ex;
                    sh.ok = ok;
                    if (lt == sh.ntl - 1) {
                        long long m = n + (long long)ex + ctile;
                        if (m > sh.cap) { m = sh.cap; atomicOr(B.status, ST_CAPACITY); }
                        B.tot[sh.k] = m - n;
                        B.n0buf[sh.k] = m;
                        if (m > n) atomicAdd(reinterpret_cast<unsigned long long*>(&B.actives[sh.k]),
                                             (unsigned long long)(m - n));
                    }
                }
            }
            __syncthreads();
            if (sh.ok) {
                long long d = n + (long long)sh.excl + off;
                for (int q = 0; q < kRItems; ++q)
                    for (uint32_t j = 0; j < cnum[q]; ++j, ++d) {
                        if (d >= sh.cap) { atomicOr(B.status, ST_CAPACITY); break; }
                        bcopy_slot(B, base + d, base + l0 + q);
                    }
            }
        }
        __syncthreads();
    }
    rpass_done(B);
}

// ---------------------------------------------------------------------------------------
// repack! (JuMC/src/population.jl:191-215) of every instance with holes: the k-th inactive
// slot below A (ascending) receives the k-th active slot at or above A counted from the end
// -- the pairing of the reference's two-pointer loop.  Pass 1 lists the holes in order.
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kRBlock) k_brepack_holes(BatchDev B) {
    __shared__ RShared sh;
    const uint32_t epoch = B.counters[2];
    for (;;) {
        if (!rtile_next(B, sh, PASS_HOLES)) break;
        const long long lt = sh.g - sh.first;
        const long long l0 = lt * kRTile + (long long)threadIdx.x * kRItems;
        const long long A = sh.A;
        uint8_t a[kRItems];
        load_flags(B, sh.base, l0, A, a);
        uint32_t h = 0;
#pragma unroll
        for (int q = 0; q < kRItems; ++q) h += (l0 + q < A && !a[q]) ? 1u : 0u;
        uint32_t htile;
        const uint32_t off = rblock_scan(sh, h, &htile);
        if (threadIdx.x < 32) {   // warp 0 looks back
            bool ok;
            const uint32_t ex =
                tile_lookback_from_warp(B.tstatus, (uint32_t)sh.first, (uint32_t)sh.g, epoch, htile, B.status, &ok);
            if (threadIdx.x == 0) {
                sh.excl = ex;
                sh.ok = ok;
            }
        }
        __syncthreads();
        if (sh.ok && h) {
            uint32_t r = sh.excl + off;
            for (int q = 0; q < kRItems; ++q)
                if (l0 + q < A && !a[q]) B.holes[sh.base + r++] = (uint32_t)(l0 + q);
        }
        __syncthreads();
    }
    rpass_done(B);
}

// Pass 2: the actives in [A, n), walked from the end (tile lt covers the lt-th block of
// kRTile slots counted back from n), so the look-back prefix is the count of actives after
// the tile and each active's rank from the end is its hole index.
__global__ void __launch_bounds__(kRBlock) k_brepack_move(BatchDev B) {
    __shared__ RShared sh;
    const uint32_t epoch = B.counters[2];
    for (;;) {
        if (!rtile_next(B, sh, PASS_MOVE)) break;
        const long long lt = sh.g - sh.first;
        const long long A = sh.A, n = sh.n;
        // this tile: slots [hi - kRTile, hi) with hi = n - lt*kRTile, clipped at A; thread t
        // takes the t-th group of kRItems counted back from hi
        const long long hi = n - lt * kRTile;
        const long long top = hi - (long long)threadIdx.x * kRItems;     // exclusive
        uint32_t m = 0;
        bool act[kRItems];
#pragma unroll
        for (int q = 0; q < kRItems; ++q) {
            const long long i = top - 1 - q;
            act[q] = i >= A && B.act[sh.base + i];
            m += act[q] ? 1u : 0u;
        }
        uint32_t mtile;
        const uint32_t off = rblock_scan(sh, m, &mtile);
        if (threadIdx.x < 32) {   // warp 0 looks back
            bool ok;
            const uint32_t ex =
                tile_lookback_from_warp(B.tstatus, (uint32_t)sh.first, (uint32_t)sh.g, epoch, mtile, B.status, &ok);
            if (threadIdx.x == 0) {
                sh.excl = ex;
                sh.ok = ok;
            }
        }
        __syncthreads();
        if (sh.ok && m) {
            uint32_t r = sh.excl + off;   // actives after this thread's group
            for (int q = 0; q < kRItems; ++q)
                if (act[q]) {
                    const long long i = top - 1 - q;
                    bcopy_slot(B, sh.base + (long long)B.holes[sh.base + r], sh.base + i);
                    ++r;
                }
        }
        __syncthreads();
    }
    rpass_done(B);
}

__global__ void k_bfinish(BatchDev B) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < B.K; k += gridDim.x * blockDim.x) {
        if (!B.inst[k].live) continue;
        // A = actives after repack!; never more than the slots in use (a capacity error has
        // been raised if the counts disagree)
        B.n0buf[k] = min(B.actives[k], B.n0buf[k]);
        B.step[k] += 1;
        B.logpos[k] += 1;
    }
}

// Join without host data: the instance's descriptor and counters, and its electrons drawn
// on the device (maxwellian_draw with the instance seed and instance-local slot).
__global__ void k_binit(BatchDev B, int k, Inst I, long long n, double sigma) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        B.inst[k] = I;
        B.n0buf[k] = n;
        B.n1buf[k] = n;
        B.step[k] = 0;
        B.logpos[k] = 0;
    }
    for (long long il = blockIdx.x * (long long)blockDim.x + threadIdx.x; il < n; il += (long long)gridDim.x * blockDim.x) {
        double vx, vy, vz, s;
        maxwellian_draw(I.seed, (uint32_t)il, sigma, vx, vy, vz, s);
        const long long i = I.base + il;
        B.f[0][i] = 0.f; B.f[1][i] = 0.f; B.f[2][i] = 0.f;
        B.f[3][i] = (float)vx; B.f[4][i] = (float)vy; B.f[5][i] = (float)vz;
        B.f[6][i] = 1.f;
        B.f[7][i] = (float)s;
        B.act[i] = 1;
    }
}

__global__ void k_bset_live(Inst* inst, int k, int live) { inst[k].live = live; }
__global__ void k_bset_table(TableView* tabs, int idx, TableView v) { tabs[idx] = v; }

}  // namespace mcs

// ---------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------
using namespace mcs;

struct BatchVariant {
    int block, ppt;
    const void* fn;
    int minb = 0;   // resident CTAs per SM the register budget is set for (0: compiler's choice)
    int refill = 8; // idle lanes of a warp before the particle queue refills
};

struct mcs_batch {
    mcs_ctx* ctx = nullptr;
    int K = 0;
    long long total_cap = 0;
    long long next_base = 0;
    std::vector<Inst> hinst;
    std::vector<const mcs_table*> gases;
    BatchDev d{};
    TableView* d_tabs = nullptr;
    long long max_tiles = 0;
    int variant = -1;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int grid[32] = {};              // persistent grid per variant (resident CTAs x SMs)
    int rgrid[3] = {};              // persistent grids of the resample / holes / move passes
    unsigned long long stage_stride[32] = {};   // per-variant secondary staging slice per CTA
    uint32_t stage_cap[32] = {};
    // double-buffered pinned copies of the per-step rings (mcs_batch_logs_enqueue / wait)
    double* hring[2] = {nullptr, nullptr};
    uint32_t* hpos[2] = {nullptr, nullptr};
    uint32_t* hstatus[2] = {nullptr, nullptr};
    cudaEvent_t lev[2] = {nullptr, nullptr};
    std::vector<void*> allocs;
};

namespace {

template <int BLOCK, int PPT, int MINB = 0, int REFILL = 8>
const void* bstep_fn() { return reinterpret_cast<const void*>(k_bstep<BLOCK, PPT, MINB, REFILL>); }

// The autotuner's space: threads per block x particles per thread, plus shapes that trade
// registers for resident CTAs (MINB) and longer tiles (16 particles per thread).
const BatchVariant kVariants[] = {
    {128, 1, bstep_fn<128, 1>()}, {128, 2, bstep_fn<128, 2>()}, {128, 4, bstep_fn<128, 4>()}, {128, 8, bstep_fn<128, 8>()},
    {256, 1, bstep_fn<256, 1>()}, {256, 2, bstep_fn<256, 2>()}, {256, 4, bstep_fn<256, 4>()}, {256, 8, bstep_fn<256, 8>()},
    {512, 1, bstep_fn<512, 1>()}, {512, 2, bstep_fn<512, 2>()}, {512, 4, bstep_fn<512, 4>()}, {512, 8, bstep_fn<512, 8>()},
    {128, 16, bstep_fn<128, 16>()}, {256, 16, bstep_fn<256, 16>()},
    {256, 8, bstep_fn<256, 8, 4>(), 4}, {256, 16, bstep_fn<256, 16, 4>(), 4},
    {128, 8, bstep_fn<128, 8, 8>(), 8}, {512, 8, bstep_fn<512, 8, 2>(), 2},
    // the particle queue's refill threshold (idle lanes of 32 before finished lanes write
    // back and refill together) on the 256 x 16, 4 CTAs/SM shape
    {256, 16, bstep_fn<256, 16, 4, 4>(), 4, 4}, {256, 16, bstep_fn<256, 16, 4, 12>(), 4, 12},
    {256, 16, bstep_fn<256, 16, 4, 16>(), 4, 16}, {256, 16, bstep_fn<256, 16, 4, 2>(), 4, 2},
};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);
static_assert(kNumVariants == MCS_BATCH_VARIANTS, "variant table and header disagree");
constexpr int kDefaultVariant = 15;  // 256 x 16 at 4 CTAs per SM (the autotuner's usual choice)

template <typename P>
int balloc(mcs_batch* b, P** p, size_t n) {
    void* q = nullptr;
    if (cudaMalloc(&q, (n ? n : 1) * sizeof(P)) != cudaSuccess) return set_err(b->ctx, MCS_ERR_NOMEM, "batch allocation");
    cudaMemset(q, 0, (n ? n : 1) * sizeof(P));
    b->allocs.push_back(q);
    *p = static_cast<P*>(q);
    return MCS_OK;
}

void drop_graph(mcs_batch* b) {
    if (b->exec || b->graph) cudaStreamSynchronize(b->ctx->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

int launch_variant(mcs_batch* b, int v, cudaStream_t s) {
    const BatchVariant& var = kVariants[v];
    BatchDev dv = b->d;
    dv.stage_stride = b->stage_stride[v];
    dv.stage_cap = b->stage_cap[v];
    void* args[] = {&dv};
    const cudaError_t e = cudaLaunchKernel(var.fn, dim3(b->grid[v]), dim3(var.block), args, 0, s);
    return e == cudaSuccess ? MCS_OK : set_err(b->ctx, MCS_ERR_CUDA, cudaGetErrorString(e));
}

// One batched step: plan + advance! + Swarm.resample! + repack!, all on stream s.
// One batched step on stream s: plan + advance! (k0/k1, optional, bracket the persistent
// step kernel), Swarm.resample!, repack! (holes, then moves), counters.
int enqueue_step(mcs_batch* b, int v, cudaStream_t s, cudaEvent_t k0 = nullptr, cudaEvent_t k1 = nullptr) {
    const int tile_step = kVariants[v].block * kVariants[v].ppt;
    const int kb = (b->K + 255) / 256;
    k_bplan<<<1, 1024, 0, s>>>(b->d, PASS_STEP, tile_step);
    if (k0) cudaEventRecord(k0, s);
    if (int st = launch_variant(b, v, s)) return st;
    if (k1) cudaEventRecord(k1, s);
    k_bempty_moments<<<kb, 256, 0, s>>>(b->d);
    k_bplan<<<1, 1024, 0, s>>>(b->d, PASS_RESAMPLE, kRTile);
    k_bresample<<<b->rgrid[0], kRBlock, 0, s>>>(b->d);
    k_bplan<<<1, 1024, 0, s>>>(b->d, PASS_HOLES, kRTile);
    k_brepack_holes<<<b->rgrid[1], kRBlock, 0, s>>>(b->d);
    k_bplan<<<1, 1024, 0, s>>>(b->d, PASS_MOVE, kRTile);
    k_brepack_move<<<b->rgrid[2], kRBlock, 0, s>>>(b->d);
    k_bfinish<<<kb, 256, 0, s>>>(b->d);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? MCS_OK : set_err(b->ctx, MCS_ERR_CUDA, cudaGetErrorString(e));
}

int upload_inst(mcs_batch* b, int k) {
    const cudaError_t e = cudaMemcpyAsync(b->d.inst + k, &b->hinst[k], sizeof(Inst), cudaMemcpyHostToDevice, b->ctx->stream);
    if (e != cudaSuccess) return set_err(b->ctx, MCS_ERR_CUDA, cudaGetErrorString(e));
    return cudaStreamSynchronize(b->ctx->stream) == cudaSuccess ? MCS_OK : MCS_ERR_CUDA;
}

int sync_status_b(mcs_batch* b) { return sync_status(b->ctx); }

}  // namespace

extern "C" {

MCS_API int mcs_batch_create(mcs_ctx* c, int max_instances, int64_t total_capacity, mcs_batch** out) {
    if (!c || !out || max_instances < 1 || max_instances > 8192 || total_capacity < 1 ||
        total_capacity > 0x7fffffffLL)
        return MCS_ERR_ARG;
    *out = nullptr;
    if (cudaSetDevice(c->device) != cudaSuccess) return MCS_ERR_CUDA;
    mcs_batch* b = new mcs_batch();
    b->ctx = c;
    b->K = max_instances;
    // room for every region's rounding to kSlotAlign slots
    b->total_cap = (total_capacity + kSlotAlign - 1) / kSlotAlign * kSlotAlign + (long long)kSlotAlign * max_instances;
    b->hinst.assign(max_instances, Inst{});
    b->max_tiles = b->total_cap / 128 + max_instances + 1;
    BatchDev& d = b->d;
    int st = MCS_OK;
    for (int q = 0; q < 8 && !st; ++q) st = balloc(b, &d.f[q], (size_t)b->total_cap);
    if (!st) st = balloc(b, &d.act, (size_t)b->total_cap);
    if (!st) st = balloc(b, &d.inst, (size_t)max_instances);
    if (!st) st = balloc(b, &d.n0buf, (size_t)max_instances);
    if (!st) st = balloc(b, &d.n1buf, (size_t)max_instances);
    if (!st) st = balloc(b, &d.step, (size_t)max_instances);
    if (!st) st = balloc(b, &d.tstart, (size_t)max_instances + 1);
    if (!st) st = balloc(b, &d.done, (size_t)max_instances);
    if (!st) st = balloc(b, &d.tpart, (size_t)b->max_tiles * kBM);
    if (!st) st = balloc(b, &d.curm, (size_t)max_instances * kBM);
    if (!st) st = balloc(b, &d.log, (size_t)max_instances * kBatchLog * kBM);
    if (!st) st = balloc(b, &d.logpos, (size_t)max_instances);
    if (!st) st = balloc(b, &d.tstatus, (size_t)b->max_tiles);
    if (!st) st = balloc(b, &d.counters, 8);
    if (!st) st = balloc(b, &d.holes, (size_t)b->total_cap);
    if (!st) st = balloc(b, &d.tile_inst, (size_t)b->max_tiles);
    if (!st) st = balloc(b, &d.rlo, (size_t)max_instances);
    if (!st) st = balloc(b, &d.tot, (size_t)max_instances);
    if (!st) st = balloc(b, &d.actives, (size_t)max_instances);
    if (!st) st = balloc(b, &d.mode, (size_t)max_instances);
    if (!st) st = balloc(b, &b->d_tabs, kMaxGases);
    // secondary staging: per variant a slice of 4 x TILE + 2048 entries per resident CTA
    size_t stage_bytes = 0;
    for (int v = 0; v < kNumVariants && !st; ++v) {
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kVariants[v].fn, kVariants[v].block, 0);
        b->grid[v] = std::max(occ, 1) * c->num_sms;
        const uint32_t cap = 4 * kVariants[v].block * kVariants[v].ppt + 2048;
        const size_t stride = bstage_bytes(cap) + 2 * brank_bytes(cap);
        b->stage_stride[v] = stride;
        b->stage_cap[v] = cap;
        stage_bytes = std::max(stage_bytes, stride * (size_t)b->grid[v]);
    }
    const void* rk[3] = {reinterpret_cast<const void*>(k_bresample), reinterpret_cast<const void*>(k_brepack_holes),
                         reinterpret_cast<const void*>(k_brepack_move)};
    for (int q = 0; q < 3; ++q) {
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, rk[q], kRBlock, 0);
        b->rgrid[q] = std::max(occ, 1) * c->num_sms;
    }
    char* stage = nullptr;
    if (!st) st = balloc(b, &stage, stage_bytes);
    if (st) { mcs_batch_destroy(b); return st; }
    d.stage = stage;
    d.stage_stride = b->stage_stride[kDefaultVariant];
    d.stage_cap = b->stage_cap[kDefaultVariant];
    d.status = c->d_status;
    d.tabs = b->d_tabs;
    d.K = max_instances;
    b->variant = kDefaultVariant;
    if (cudaDeviceSynchronize() != cudaSuccess) { mcs_batch_destroy(b); return MCS_ERR_CUDA; }
    *out = b;
    return MCS_OK;
}

MCS_API int mcs_batch_destroy(mcs_batch* b) {
    if (!b) return MCS_OK;
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    drop_graph(b);
    for (void* p : b->allocs) cudaFree(p);
    for (int q = 0; q < 2; ++q) {
        if (b->hring[q]) cudaFreeHost(b->hring[q]);
        if (b->hpos[q]) cudaFreeHost(b->hpos[q]);
        if (b->hstatus[q]) cudaFreeHost(b->hstatus[q]);
        if (b->lev[q]) cudaEventDestroy(b->lev[q]);
    }
    delete b;
    return MCS_OK;
}

}  // extern "C"

namespace {

// Host bookkeeping of a join: a free instance slot, a first-fit region of `capacity` slots
// and the gas table's index (registered on the device, stream-ordered, when new).
int place_instance(mcs_batch* b, const mcs_table* t, double ex, double ey, double ez, uint64_t seed, int64_t n0,
                   double tol, int64_t capacity, int* k_out, Inst* inst_out) {
    mcs_ctx* c = b->ctx;
    int k = -1;
    for (int q = 0; q < b->K; ++q)
        if (!b->hinst[q].live) { k = q; break; }
    if (k < 0) return set_err(c, MCS_ERR_CAPACITY, "no free instance slot");
    // region: first fit over the free space between live regions (ordered by base)
    std::vector<std::pair<long long, long long>> used;
    for (int q = 0; q < b->K; ++q)
        if (b->hinst[q].live) used.push_back({b->hinst[q].base, b->hinst[q].cap});
    std::sort(used.begin(), used.end());
    // regions are kSlotAlign-aligned and a multiple of it long (16-byte loads of the flags)
    const long long region = (capacity + kSlotAlign - 1) / kSlotAlign * kSlotAlign;
    long long base = 0;
    bool found = false;
    for (auto& u : used) {
        if (u.first - base >= region) { found = true; break; }
        base = u.first + (u.second + kSlotAlign - 1) / kSlotAlign * kSlotAlign;
    }
    if (!found && b->total_cap - base < region) return set_err(c, MCS_ERR_NOMEM, "no room for the instance");
    int gas = -1;
    for (size_t q = 0; q < b->gases.size(); ++q)
        if (b->gases[q] == t) gas = (int)q;
    if (gas < 0) {
        if ((int)b->gases.size() >= kMaxGases) return set_err(c, MCS_ERR_ARG, "too many distinct tables");
        gas = (int)b->gases.size();
        b->gases.push_back(t);
        k_bset_table<<<1, 1, 0, c->stream>>>(b->d_tabs, gas, t->v);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return set_err(c, MCS_ERR_CUDA, cudaGetErrorString(e));
    }
    Inst I{};
    I.base = base;
    I.cap = capacity;
    I.seed = seed;
    const double qm = (-kElementaryCharge) / kElectronMass;
    I.ax = (float)(qm * ex); I.ay = (float)(qm * ey); I.az = (float)(qm * ez);
    I.table = gas;
    I.live = 1;
    I.sel_row = -1;
    for (int j = 0; j < t->v.nrows; ++j)
        if (t->v.kind[j] == MCS_IONIZATION || t->v.kind[j] == MCS_IONIZATION_UNIFORM) { I.sel_row = j; break; }
    I.n0 = n0;
    I.tol = tol;
    *k_out = k;
    *inst_out = I;
    return MCS_OK;
}

}  // namespace

extern "C" {

MCS_API int mcs_batch_add(mcs_batch* b, const mcs_table* t, double ex, double ey, double ez, uint64_t seed,
                          int64_t n0, double tol, int64_t capacity, const double* x, const double* v,
                          const double* w, const double* s, const uint8_t* active, int64_t n, int* slot) {
    if (!b || !t || !slot || capacity < 1 || n < 0 || n > capacity) return MCS_ERR_ARG;
    if (t && t->photo_rows) return MCS_ERR_UNSUPPORTED;   // photo-emission needs mcs_advance_mixed
    if (n > 0 && (!x || !v || !w || !s || !active)) return MCS_ERR_ARG;
    mcs_ctx* c = b->ctx;
    if (cudaSetDevice(c->device) != cudaSuccess) return MCS_ERR_CUDA;
    if (int st = sync_status(c)) return st;  // host arrays are copied between steps
    int k = -1;
    Inst I{};
    if (int st = place_instance(b, t, ex, ey, ez, seed, n0, tol, capacity, &k, &I)) return st;
    const long long base = I.base;
    // particles: host -> device staging (doubles) -> FP32 SoA region
    if (n > 0) {
        std::vector<float> tmp((size_t)n);
        for (int q = 0; q < 8; ++q) {
            for (int64_t i = 0; i < n; ++i) {
                double val;
                if (q < 3) val = x[3 * i + q];
                else if (q < 6) val = v[3 * i + (q - 3)];
                else if (q == 6) val = w[i];
                else val = s[i];
                tmp[i] = (float)val;
            }
            if (cudaMemcpyAsync(b->d.f[q] + base, tmp.data(), (size_t)n * sizeof(float), cudaMemcpyHostToDevice,
                                c->stream) != cudaSuccess ||
                cudaStreamSynchronize(c->stream) != cudaSuccess)
                return set_err(c, MCS_ERR_CUDA, "instance upload");
        }
        std::vector<uint8_t> a((size_t)n);
        for (int64_t i = 0; i < n; ++i) a[i] = active[i] ? 1 : 0;
        if (cudaMemcpyAsync(b->d.act + base, a.data(), (size_t)n, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
            return set_err(c, MCS_ERR_CUDA, "instance upload");
    }
    const long long nn = n;
    const uint32_t zero = 0;
    cudaMemcpyAsync(b->d.n0buf + k, &nn, sizeof(nn), cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(b->d.n1buf + k, &nn, sizeof(nn), cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(b->d.step + k, &zero, sizeof(zero), cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(b->d.logpos + k, &zero, sizeof(zero), cudaMemcpyHostToDevice, c->stream);
    b->hinst[k] = I;
    if (int st = upload_inst(b, k)) return st;
    *slot = k;
    return MCS_OK;
}

// Join with electrons drawn on the device: n electrons at the origin, weight 1, isotropic
// Maxwellian velocities of mean energy mean_energy_ev.  Stream-ordered, no host wait.
MCS_API int mcs_batch_add_maxwellian(mcs_batch* b, const mcs_table* t, double ex, double ey, double ez,
                                     uint64_t seed, int64_t n0, double tol, int64_t capacity, int64_t n,
                                     double mean_energy_ev, int* slot) {
    if (!b || !t || !slot || capacity < 1 || n < 0 || n > capacity || !(mean_energy_ev >= 0)) return MCS_ERR_ARG;
    if (t && t->photo_rows) return MCS_ERR_UNSUPPORTED;   // photo-emission needs mcs_advance_mixed
    mcs_ctx* c = b->ctx;
    if (cudaSetDevice(c->device) != cudaSuccess) return MCS_ERR_CUDA;
    int k = -1;
    Inst I{};
    if (int st = place_instance(b, t, ex, ey, ez, seed, n0, tol, capacity, &k, &I)) return st;
    const int gr = (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, (long long)c->num_sms * 8));
    k_binit<<<gr, 256, 0, c->stream>>>(b->d, k, I, (long long)n, maxwellian_sigma(mean_energy_ev));
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_err(c, MCS_ERR_CUDA, cudaGetErrorString(e));
    b->hinst[k] = I;
    *slot = k;
    return MCS_OK;
}

// Leave: stream-ordered, so steps already enqueued still advance the instance.
MCS_API int mcs_batch_remove(mcs_batch* b, int slot) {
    if (!b || slot < 0 || slot >= b->K || !b->hinst[slot].live) return MCS_ERR_ARG;
    if (cudaSetDevice(b->ctx->device) != cudaSuccess) return MCS_ERR_CUDA;
    b->hinst[slot].live = 0;
    k_bset_live<<<1, 1, 0, b->ctx->stream>>>(b->d.inst, slot, 0);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? MCS_OK : set_err(b->ctx, MCS_ERR_CUDA, cudaGetErrorString(e));
}

// Enqueue copies of every slot's ring, logged-step counts and the status word into pinned
// host buffer `buf` (0 or 1), then clear the device status; returns without waiting.
MCS_API int mcs_batch_logs_enqueue(mcs_batch* b, int buf) {
    if (!b || buf < 0 || buf > 1) return MCS_ERR_ARG;
    mcs_ctx* c = b->ctx;
    if (cudaSetDevice(c->device) != cudaSuccess) return MCS_ERR_CUDA;
    const size_t ring_bytes = sizeof(double) * kBM * kBatchLog * b->K;
    if (!b->hring[buf]) {
        if (cudaHostAlloc(&b->hring[buf], ring_bytes, cudaHostAllocDefault) != cudaSuccess ||
            cudaHostAlloc(&b->hpos[buf], sizeof(uint32_t) * b->K, cudaHostAllocDefault) != cudaSuccess ||
            cudaHostAlloc(&b->hstatus[buf], sizeof(uint32_t), cudaHostAllocDefault) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->lev[buf], cudaEventDisableTiming) != cudaSuccess)
            return set_err(c, MCS_ERR_NOMEM, "pinned log buffers");
    }
    cudaError_t e = cudaMemcpyAsync(b->hring[buf], b->d.log, ring_bytes, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->hpos[buf], b->d.logpos, sizeof(uint32_t) * b->K, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->hstatus[buf], c->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_status, 0, sizeof(uint32_t), c->stream);
    if (e == cudaSuccess) e = cudaEventRecord(b->lev[buf], c->stream);
    return e == cudaSuccess ? MCS_OK : set_err(c, MCS_ERR_CUDA, cudaGetErrorString(e));
}

// Wait for buffer `buf`'s copies; *ring / *logpos point into the pinned buffer (valid until
// the next enqueue into it).  A device status raised before the copy is returned here.
MCS_API int mcs_batch_logs_wait(mcs_batch* b, int buf, const double** ring, const uint32_t** logpos) {
    if (!b || buf < 0 || buf > 1 || !b->lev[buf] || !ring || !logpos) return MCS_ERR_ARG;
    mcs_ctx* c = b->ctx;
    if (cudaEventSynchronize(b->lev[buf]) != cudaSuccess) return set_err(c, MCS_ERR_CUDA, "log copy");
    *ring = b->hring[buf];
    *logpos = b->hpos[buf];
    const uint32_t st = *b->hstatus[buf];
    if (st) {
        const int code = map_status(st);
        if (code) return set_err(c, code, status_text(code));
    }
    return MCS_OK;
}

MCS_API int mcs_batch_step(mcs_batch* b, double dt, int nsteps, int use_graph) {
    if (!b || nsteps < 0 || !(dt >= 0)) return MCS_ERR_ARG;
    mcs_ctx* c = b->ctx;
    if (cudaSetDevice(c->device) != cudaSuccess) return MCS_ERR_CUDA;
    if (b->d.dt != dt || b->d.flags != c->flags) { b->d.dt = dt; b->d.flags = c->flags; drop_graph(b); }
    if (!use_graph) {
        for (int i = 0; i < nsteps; ++i)
            if (int st = enqueue_step(b, b->variant, c->stream)) return st;
        return MCS_OK;
    }
    if (!b->exec) {
        cudaStream_t cs;
        if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return MCS_ERR_CUDA;
        cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        const int st = enqueue_step(b, b->variant, cs);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(cs, &g);
        cudaStreamDestroy(cs);
        if (st || e != cudaSuccess) { if (g) cudaGraphDestroy(g); return st ? st : set_err(c, MCS_ERR_CUDA, cudaGetErrorString(e)); }
        if (cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess) { cudaGraphDestroy(g); return set_err(c, MCS_ERR_CUDA, "graph instantiate"); }
        b->graph = g;
    }
    for (int i = 0; i < nsteps; ++i) {
        const cudaError_t e = cudaGraphLaunch(b->exec, c->stream);
        if (e != cudaSuccess) return set_err(c, MCS_ERR_CUDA, cudaGetErrorString(e));
    }
    return MCS_OK;
}

MCS_API int mcs_batch_sync(mcs_batch* b) {
    if (!b) return MCS_ERR_ARG;
    return sync_status_b(b);
}

// Per-instance counters: n particles, steps done (host arrays of max_instances).
MCS_API int mcs_batch_state(mcs_batch* b, int64_t* n, uint32_t* steps) {
    if (!b) return MCS_ERR_ARG;
    const int st = sync_status_b(b);
    if (n) cudaMemcpy(n, b->d.n0buf, sizeof(long long) * b->K, cudaMemcpyDeviceToHost);
    if (steps) cudaMemcpy(steps, b->d.step, sizeof(uint32_t) * b->K, cudaMemcpyDeviceToHost);
    return st;
}

// The last `count` per-step moments of an instance (oldest first), MCS_BATCH_MOMENTS each.
MCS_API int mcs_batch_read_log(mcs_batch* b, int slot, double* out, int count) {
    if (!b || !out || slot < 0 || slot >= b->K || count < 0 || count > kBatchLog) return MCS_ERR_ARG;
    const int st = sync_status_b(b);
    uint32_t pos = 0;
    cudaMemcpy(&pos, b->d.logpos + slot, sizeof(pos), cudaMemcpyDeviceToHost);
    std::vector<double> ring((size_t)kBatchLog * kBM);
    cudaMemcpy(ring.data(), b->d.log + (size_t)slot * kBatchLog * kBM, ring.size() * sizeof(double), cudaMemcpyDeviceToHost);
    for (int i = 0; i < count; ++i) {
        const long long step = (long long)pos - count + i;
        if (step < 0) { std::memset(out + (size_t)i * kBM, 0, kBM * sizeof(double)); continue; }
        std::memcpy(out + (size_t)i * kBM, ring.data() + (size_t)(step % kBatchLog) * kBM, kBM * sizeof(double));
    }
    return st;
}

// The sums of every instance's last step (max_instances x MCS_BATCH_MOMENTS) in one copy.
MCS_API int mcs_batch_read_current(mcs_batch* b, double* out) {
    if (!b || !out) return MCS_ERR_ARG;
    mcs_ctx* c = b->ctx;
    const cudaError_t e = cudaMemcpyAsync(out, b->d.curm, sizeof(double) * kBM * b->K, cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) return set_err(c, MCS_ERR_CUDA, cudaGetErrorString(e));
    return sync_status_b(b);
}

// The whole per-step ring of every slot ([max_instances][MCS_BATCH_LOG][MCS_BATCH_MOMENTS])
// and each slot's count of logged steps, in two copies.
MCS_API int mcs_batch_read_logs(mcs_batch* b, double* ring, uint32_t* logpos) {
    if (!b || !ring || !logpos) return MCS_ERR_ARG;
    mcs_ctx* c = b->ctx;
    cudaError_t e = cudaMemcpyAsync(ring, b->d.log, sizeof(double) * kBM * kBatchLog * b->K, cudaMemcpyDeviceToHost,
                                    c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(logpos, b->d.logpos, sizeof(uint32_t) * b->K, cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) return set_err(c, MCS_ERR_CUDA, cudaGetErrorString(e));
    return sync_status_b(b);
}

// Copy one instance's particles to the host (Julia layout).
MCS_API int mcs_batch_download(mcs_batch* b, int slot, double* x, double* v, double* w, double* s, uint8_t* active,
                               int64_t cap, int64_t* n_out) {
    if (!b || slot < 0 || slot >= b->K || !n_out) return MCS_ERR_ARG;
    const int st = sync_status_b(b);
    long long n = 0;
    cudaMemcpy(&n, b->d.n0buf + slot, sizeof(n), cudaMemcpyDeviceToHost);
    *n_out = n;
    if (n > cap) return MCS_ERR_ARG;
    const long long base = b->hinst[slot].base;
    std::vector<float> tmp((size_t)n);
    for (int q = 0; q < 8; ++q) {
        cudaMemcpy(tmp.data(), b->d.f[q] + base, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
        for (long long i = 0; i < n; ++i) {
            if (q < 3) x[3 * i + q] = tmp[i];
            else if (q < 6) v[3 * i + (q - 3)] = tmp[i];
            else if (q == 6) w[i] = tmp[i];
            else s[i] = tmp[i];
        }
    }
    cudaMemcpy(active, b->d.act + base, (size_t)n, cudaMemcpyDeviceToHost);
    return st;
}

// Time every (block, particles-per-thread) variant of the batched step on the current
// state (restored after each trial) and keep the fastest.  Returns the chosen index.
MCS_API int mcs_batch_autotune(mcs_batch* b, double dt, int trial_steps, int* chosen, float* times_ms) {
    if (!b || trial_steps < 1) return MCS_ERR_ARG;
    mcs_ctx* c = b->ctx;
    if (cudaSetDevice(c->device) != cudaSuccess) return MCS_ERR_CUDA;
    b->d.dt = dt;
    b->d.flags = c->flags;
    drop_graph(b);
    // snapshot of the mutable state
    const size_t cap = (size_t)b->total_cap;
    std::vector<void*> snap;
    auto save = [&](const void* src, size_t bytes) {
        void* p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) return false;
        cudaMemcpyAsync(p, src, bytes, cudaMemcpyDeviceToDevice, c->stream);
        snap.push_back(p);
        return true;
    };
    const void* srcs[] = {b->d.f[0], b->d.f[1], b->d.f[2], b->d.f[3], b->d.f[4], b->d.f[5], b->d.f[6], b->d.f[7],
                          b->d.act, b->d.n0buf, b->d.step, b->d.logpos};
    const size_t sizes[] = {cap * 4, cap * 4, cap * 4, cap * 4, cap * 4, cap * 4, cap * 4, cap * 4, cap,
                            sizeof(long long) * b->K, sizeof(uint32_t) * b->K, sizeof(uint32_t) * b->K};
    for (int q = 0; q < 12; ++q)
        if (!save(srcs[q], sizes[q])) {
            for (void* p : snap) cudaFree(p);
            return set_err(c, MCS_ERR_NOMEM, "autotune snapshot");
        }
    auto restore = [&]() {
        for (int q = 0; q < 12; ++q)
            cudaMemcpyAsync(const_cast<void*>(srcs[q]), snap[q], sizes[q], cudaMemcpyDeviceToDevice, c->stream);
    };
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    int bestv = kDefaultVariant;
    int st = MCS_OK;
    for (int v = 0; v < kNumVariants && !st; ++v) {
        restore();
        st = enqueue_step(b, v, c->stream);  // warm-up
        if (st) break;
        cudaEventRecord(e0, c->stream);
        for (int i = 0; i < trial_steps && !st; ++i) st = enqueue_step(b, v, c->stream);
        cudaEventRecord(e1, c->stream);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (times_ms) times_ms[v] = ms / trial_steps;
        if (ms < best) { best = ms; bestv = v; }
    }
    restore();
    cudaStreamSynchronize(c->stream);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (void* p : snap) cudaFree(p);
    if (st) return st;
    b->variant = bestv;
    if (chosen) *chosen = bestv;
    return sync_status_b(b);
}

// nsteps batched steps without the graph, timing the persistent step kernel and the whole
// step with CUDA events on the context's stream; averages per step in milliseconds.
MCS_API int mcs_batch_profile(mcs_batch* b, double dt, int nsteps, float* kernel_ms, float* step_ms) {
    if (!b || nsteps < 1 || !(dt >= 0)) return MCS_ERR_ARG;
    mcs_ctx* c = b->ctx;
    if (cudaSetDevice(c->device) != cudaSuccess) return MCS_ERR_CUDA;
    if (b->d.dt != dt || b->d.flags != c->flags) { b->d.dt = dt; b->d.flags = c->flags; drop_graph(b); }
    std::vector<cudaEvent_t> ev((size_t)nsteps * 4);
    for (auto& e : ev) cudaEventCreate(&e);
    int st = MCS_OK;
    for (int i = 0; i < nsteps && !st; ++i) {
        cudaEventRecord(ev[4 * i], c->stream);
        st = enqueue_step(b, b->variant, c->stream, ev[4 * i + 1], ev[4 * i + 2]);
        cudaEventRecord(ev[4 * i + 3], c->stream);
    }
    cudaStreamSynchronize(c->stream);
    float tk = 0.0f, ts = 0.0f;
    for (int i = 0; i < nsteps && !st; ++i) {
        float a = 0.0f, t = 0.0f;
        cudaEventElapsedTime(&a, ev[4 * i + 1], ev[4 * i + 2]);
        cudaEventElapsedTime(&t, ev[4 * i], ev[4 * i + 3]);
        tk += a;
        ts += t;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (st) return st;
    if (kernel_ms) *kernel_ms = tk / nsteps;
    if (step_ms) *step_ms = ts / nsteps;
    return sync_status_b(b);
}

MCS_API int mcs_batch_set_variant(mcs_batch* b, int variant) {
    if (!b || variant < 0 || variant >= kNumVariants) return MCS_ERR_ARG;
    b->variant = variant;
    drop_graph(b);
    return MCS_OK;
}

MCS_API int mcs_batch_variant_shape(int variant, int* block, int* ppt) {
    if (variant < 0 || variant >= kNumVariants || !block || !ppt) return MCS_ERR_ARG;
    *block = kVariants[variant].block;
    *ppt = kVariants[variant].ppt;
    return MCS_OK;
}

MCS_API int mcs_batch_variant_min_blocks(int variant, int* min_blocks) {
    if (variant < 0 || variant >= kNumVariants || !min_blocks) return MCS_ERR_ARG;
    *min_blocks = kVariants[variant].minb;
    return MCS_OK;
}

MCS_API int mcs_batch_variant_refill(int variant, int* idle_lanes) {
    if (variant < 0 || variant >= kNumVariants || !idle_lanes) return MCS_ERR_ARG;
    *idle_lanes = kVariants[variant].refill;
    return MCS_OK;
}

}  // extern "C"
