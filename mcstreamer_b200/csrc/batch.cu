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
constexpr int kBTile = 2048;        // tile of the scan / resample / repack passes

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
    uint32_t* u32a;
    uint32_t* u32b;
    long long* tot;
    int K;
    uint32_t flags;
    char* stage;
    unsigned long long stage_stride;
    uint32_t stage_cap;
    double dt;
};

// ---------------------------------------------------------------------------------------
// Plan: tile prefix over instances for a pass reading counts `nin` with tile size `tile`;
// defaults the pass's output counts to its input counts and advances the epoch.
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_bplan(BatchDev B, int in_is_n1, int tile) {
    __shared__ long long wsum[32];
    const long long* nin = in_is_n1 ? B.n1buf : B.n0buf;
    long long* nout = in_is_n1 ? B.n0buf : B.n1buf;
    const int per = (B.K + 1023) / 1024;
    long long loc = 0;
    for (int q = 0; q < per; ++q) {
        const int k = threadIdx.x * per + q;
        if (k < B.K) {
            const long long n = B.inst[k].live ? nin[k] : 0;
            loc += (n + tile - 1) / tile;
            nout[k] = nin[k];
            B.done[k] = 0;
        }
    }
    // block exclusive scan of loc
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
        if (k < B.K) {
            B.tstart[k] = run;
            const long long n = B.inst[k].live ? nin[k] : 0;
            run += (n + tile - 1) / tile;
        }
    }
}

__device__ __forceinline__ int find_inst(const long long* tstart, int K, long long g) {
    int lo = 0, hi = K;  // largest k with tstart[k] <= g, among k < K
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (tstart[mid] <= g) lo = mid; else hi = mid;
    }
    return lo;
}

// Rate of row j at energy v2 (FP32 table), for the per-step rate estimator (collrate).
__device__ __forceinline__ float rate_row32(const TableView& t, float v2, int j) {
    const float u = fmaf(v2, t.ke32, -t.e0n32);
    int k = (int)u;
    float w;
    if (!(u >= 0.0f && k <= t.neps - 2)) { k = u >= 0.0f ? t.neps - 2 : 0; w = u >= 0.0f ? 0.0f : 1.0f; }
    else w = (float)(k + 1) - u;
    const float a = __ldg(t.rate32 + (size_t)k * t.nrp + j), b = __ldg(t.rate32 + (size_t)(k + 1) * t.nrp + j);
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
};

// ---------------------------------------------------------------------------------------
// Batched advance! (FP32, uniform field per instance, closed-form push between real
// collisions): the body of k_step_abs<float,...,CLOSED> with instance indirection.
// ---------------------------------------------------------------------------------------
template <int BLOCK, int PPT>
__global__ void __launch_bounds__(BLOCK) k_bstep(BatchDev B) {
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
    for (;;) {
        if (threadIdx.x == 0) {
            const long long g = atomicAdd(&B.counters[0], 1u);
            sh.tile = g;
            sh.count = 0;
            sh.next = 0;
            if (g < T) {
                const int k = find_inst(B.tstart, B.K, g);
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
            if (idle != 0xffffffffu && __popc(idle) < 8) goto substep;
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
                have = trem > 0;
                if (!have) cnt[q] = 0;   // dt == 0: state unchanged
            }
            if (!__any_sync(0xffffffffu, have)) break;
        substep:
            if (!have) continue;
            {
                // one sub-step of advance! with the closed-form push of a uniform field
                const double tn = s * tab.inv_maxrate;
                double t;
                bool collides;
                if (trem > tn) { t = tn; collides = true; }
                else { t = trem; collides = false; s -= t * tab.maxrate; }
                tau += (float)t;
                if (collides) {
                    float cvx = fmaf(ax, tau, vx), cvy = fmaf(ay, tau, vy), cvz = fmaf(az, tau, vz);
                    Sec<float> sec;
                    const int out = collide_once<float>(sh.rows, tab, C, rng, cvx, cvy, cvz, sec);
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
                trem -= t;
                if (!(trem > 0)) {
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

        // ---- ordered append of this tile's secondaries within the instance ----
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
                bool ok;
                sh.excl = tile_lookback_from(B.tstatus, (uint32_t)sh.first, (uint32_t)g, epoch, c, B.status, &ok);
                sh.ok = ok;
                if (lt == sh.ntl - 1) {
                    long long nn = n_entry + (long long)sh.excl + c;
                    if (nn > I.cap) { nn = I.cap; atomicOr(B.status, ST_CAPACITY); }
                    B.n1buf[k] = nn;
                }
            }
            __syncthreads();
            uint32_t run = sh.wtot[wid] + incl - sum;
#pragma unroll
            for (int q = 0; q < PER; ++q) { cnt[threadIdx.x * PER + q] = run; run += v[q]; }
            __syncthreads();
        }
        if (sh.ok) {
            for (uint32_t e = threadIdx.x; e < c; e += BLOCK) {
                const uint32_t key = sg.key[e];
                const long long dl = n_entry + (long long)sh.excl + cnt[key >> 16] + (key & 0xffffu);
                if (dl >= I.cap) { atomicOr(B.status, ST_CAPACITY); continue; }
                const long long d = I.base + dl;
#pragma unroll
                for (int q = 0; q < 8; ++q) B.f[q][d] = sg.f[q][e];
                B.act[d] = sg.act[e];
            }
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
            // secondaries in their appended (serial) order
            __syncthreads();
            const long long d0 = n_entry + (long long)sh.excl;
            for (uint32_t r = threadIdx.x; r < c; r += BLOCK) {
                const long long dl = d0 + r;
                const long long d = I.base + dl;
                if (sh.ok && dl < I.cap && B.act[d])
                    add(B.f[0][d], B.f[1][d], B.f[2][d], B.f[3][d], B.f[4][d], B.f[5][d], B.f[6][d]);
            }
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
    }
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

// ---------------------------------------------------------------------------------------
// Segmented (per-instance) exclusive scan of u32 counts (in == nullptr: active flags) over
// the pass's tiles; totals per instance into B.tot.
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_bscan(BatchDev B, int in_is_n1, const uint32_t* __restrict__ in,
                                               uint32_t* __restrict__ out) {
    constexpr int ITEMS = kBTile / 256;
    __shared__ uint32_t s_warp[8];
    __shared__ long long s_g, s_first, s_ntl, s_base, s_n;
    __shared__ int s_k;
    __shared__ uint32_t s_excl;
    const long long T = B.tstart[B.K];
    const uint32_t epoch = B.counters[2];
    const long long* nin = in_is_n1 ? B.n1buf : B.n0buf;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (;;) {
        if (threadIdx.x == 0) {
            const long long g = atomicAdd(&B.counters[0], 1u);
            s_g = g;
            if (g < T) {
                const int k = find_inst(B.tstart, B.K, g);
                s_k = k;
                s_first = B.tstart[k];
                s_ntl = (k + 1 < B.K ? B.tstart[k + 1] : T) - s_first;
                s_base = B.inst[k].base;
                s_n = nin[k];
            }
        }
        __syncthreads();
        const long long g = s_g;
        if (g >= T) break;
        const long long lt = g - s_first;
        const long long l0 = lt * kBTile + (long long)threadIdx.x * ITEMS;
        uint32_t v[ITEMS];
        uint32_t tsum = 0;
#pragma unroll
        for (int q = 0; q < ITEMS; ++q) {
            const long long il = l0 + q;
            uint32_t cv = 0;
            if (il < s_n) cv = in ? in[s_base + il] : (uint32_t)(B.act[s_base + il] != 0);
            v[q] = tsum;
            tsum += cv;
        }
        uint32_t incl = tsum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t yv = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += yv;
        }
        if (lane == 31) s_warp[wid] = incl;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t acc = 0;
            for (int q = 0; q < 8; ++q) { const uint32_t t2 = s_warp[q]; s_warp[q] = acc; acc += t2; }
            bool ok;
            s_excl = tile_lookback_from(B.tstatus, (uint32_t)s_first, (uint32_t)g, epoch, acc, B.status, &ok);
            if (lt == s_ntl - 1) B.tot[s_k] = (long long)s_excl + acc;
        }
        __syncthreads();
        const uint32_t off = s_excl + s_warp[wid] + incl - tsum;
#pragma unroll
        for (int q = 0; q < ITEMS; ++q) {
            const long long il = l0 + q;
            if (il < s_n) out[s_base + il] = off + v[q];
        }
        __syncthreads();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t d = atomicAdd(&B.counters[1], 1u);
        if (d == gridDim.x - 1) { B.counters[0] = 0; B.counters[1] = 0; }
    }
}

// Zero totals of instances without tiles (their scans never run).
__global__ void k_bzero_tot(BatchDev B) {
    const long long T = B.tstart[B.K];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < B.K; k += gridDim.x * blockDim.x) {
        const long long nt = (k + 1 < B.K ? B.tstart[k + 1] : T) - B.tstart[k];
        if (nt == 0) B.tot[k] = 0;
    }
}

__device__ long long poisson_sample_b(Rng& r, double lam) {
    if (lam <= 0) return 0;
    if (lam < 10.0) {
        const double u = r.u64();
        double pr = exp(-lam), F = pr;
        long long kk = 0;
        while (u > F && kk < 1000) { ++kk; pr *= lam / (double)kk; F += pr; }
        return kk;
    }
    const double slam = sqrt(lam), loglam = log(lam);
    const double b = 0.931 + 2.53 * slam;
    const double a = -0.059 + 0.02483 * b;
    const double invalpha = 1.1239 + 1.1328 / (b - 3.4);
    const double vr = 0.9277 - 3.6224 / (b - 2.0);
    for (int it = 0; it < 1000; ++it) {
        const double U = r.u64() - 0.5;
        const double V = r.u64();
        const double us = 0.5 - fabs(U);
        const double kf = floor((2.0 * a / us + b) * U + lam + 0.43);
        if (us >= 0.07 && V <= vr) return (long long)kf;
        if (kf < 0 || (us < 0.013 && V > us)) continue;
        if (log(V) + log(invalpha) - log(a / (us * us) + b) <= -lam + kf * loglam - lgamma(kf + 1.0))
            return (long long)kf;
    }
    return (long long)floor(lam);
}

// Grid-stride over all live slots of all instances (pass reading n1).
template <typename F>
__device__ __forceinline__ void for_each_slot(const BatchDev& B, const long long* nin, F&& fn) {
    for (int k = blockIdx.y; k < B.K; k += gridDim.y) {
        const Inst I = B.inst[k];
        if (!I.live) continue;
        const long long n = nin[k];
        for (long long il = blockIdx.x * (long long)blockDim.x + threadIdx.x; il < n; il += (long long)gridDim.x * blockDim.x)
            fn(k, I, il);
    }
}

// Swarm.resample! decisions (Swarm.jl:193-223) for every instance: drop, or Poisson clone counts.
__global__ void k_bsres_count(BatchDev B) {
    for_each_slot(B, B.n1buf, [&](int k, const Inst& I, long long il) {
        const long long i = I.base + il;
        uint32_t cnum = 0;
        const long long ncur = (long long)B.curm[(long long)k * kBM + SM_COUNT];
        const bool skip = I.n0 <= 0 || ncur == 0 || fabs((double)(ncur - I.n0) / (double)I.n0) < I.tol;
        if (!skip && B.act[i]) {
            Rng r;
            r.init(I.seed, (uint32_t)il, B.step[k] + 1u, TAG_SWARM_RESAMPLE);
            if (ncur > I.n0) {
                if (r.u64() < (double)(ncur - I.n0) / (double)ncur) B.act[i] = 0;
            } else {
                cnum = (uint32_t)poisson_sample_b(r, (double)(I.n0 - ncur) / (double)ncur);
            }
        }
        B.u32a[i] = cnum;
    });
}

__device__ __forceinline__ void bcopy_slot(const BatchDev& B, long long dst, long long src) {
#pragma unroll
    for (int q = 0; q < 8; ++q) B.f[q][dst] = B.f[q][src];
    B.act[dst] = B.act[src];
}

__global__ void k_bsres_write(BatchDev B) {
    for_each_slot(B, B.n1buf, [&](int k, const Inst& I, long long il) {
        const long long i = I.base + il;
        const uint32_t cnum = B.u32a[i];
        const long long n = B.n1buf[k];
        for (uint32_t j = 0; j < cnum; ++j) {
            const long long dl = n + (long long)B.u32b[i] + j;
            if (dl >= I.cap) { atomicOr(B.status, ST_CAPACITY); break; }
            bcopy_slot(B, I.base + dl, i);
        }
    });
    if (blockIdx.x == 0)
        for (int k = blockIdx.y * blockDim.x + threadIdx.x; k < B.K; k += gridDim.y * blockDim.x) {
            if (!B.inst[k].live) continue;
            long long m = B.n1buf[k] + B.tot[k];
            if (m > B.inst[k].cap) { m = B.inst[k].cap; atomicOr(B.status, ST_CAPACITY); }
            B.n0buf[k] = m;
        }
}

// repack! (population.jl:191-215) per instance: holes below A get the actives at or
// above A, taken from the end.
__global__ void k_brepack_holes(BatchDev B) {
    for_each_slot(B, B.n0buf, [&](int k, const Inst& I, long long il) {
        const long long A = B.tot[k];
        const long long i = I.base + il;
        if (il < A && !B.act[i]) B.u32a[I.base + (il - (long long)B.u32b[i])] = (uint32_t)il;
    });
}

__global__ void k_brepack_move(BatchDev B) {
    for_each_slot(B, B.n0buf, [&](int k, const Inst& I, long long il) {
        const long long A = B.tot[k];
        const long long i = I.base + il;
        if (il >= A && B.act[i]) {
            const long long q = A - 1 - (long long)B.u32b[i];
            bcopy_slot(B, I.base + (long long)B.u32a[I.base + q], i);
        }
    });
}

__global__ void k_bfinish(BatchDev B) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < B.K; k += gridDim.x * blockDim.x) {
        if (!B.inst[k].live) continue;
        B.n0buf[k] = B.tot[k];      // A = actives after repack
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
    int grid[16] = {};              // persistent grid per variant (resident CTAs x SMs)
    // double-buffered pinned copies of the per-step rings (mcs_batch_logs_enqueue / wait)
    double* hring[2] = {nullptr, nullptr};
    uint32_t* hpos[2] = {nullptr, nullptr};
    uint32_t* hstatus[2] = {nullptr, nullptr};
    cudaEvent_t lev[2] = {nullptr, nullptr};
    std::vector<void*> allocs;
};

namespace {

template <int BLOCK, int PPT>
const void* bstep_fn() { return reinterpret_cast<const void*>(k_bstep<BLOCK, PPT>); }

const BatchVariant kVariants[] = {
    {128, 1, bstep_fn<128, 1>()}, {128, 2, bstep_fn<128, 2>()}, {128, 4, bstep_fn<128, 4>()}, {128, 8, bstep_fn<128, 8>()},
    {256, 1, bstep_fn<256, 1>()}, {256, 2, bstep_fn<256, 2>()}, {256, 4, bstep_fn<256, 4>()}, {256, 8, bstep_fn<256, 8>()},
    {512, 1, bstep_fn<512, 1>()}, {512, 2, bstep_fn<512, 2>()}, {512, 4, bstep_fn<512, 4>()}, {512, 8, bstep_fn<512, 8>()},
};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);
constexpr int kDefaultVariant = 5;  // 256 x 2

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
    void* args[] = {&b->d};
    const cudaError_t e = cudaLaunchKernel(var.fn, dim3(b->grid[v]), dim3(var.block), args, 0, s);
    return e == cudaSuccess ? MCS_OK : set_err(b->ctx, MCS_ERR_CUDA, cudaGetErrorString(e));
}

// One batched step: plan + advance! + Swarm.resample! + repack!, all on stream s.
// k0/k1 (optional) bracket the persistent step kernel.
int enqueue_step(mcs_batch* b, int v, cudaStream_t s, cudaEvent_t k0 = nullptr, cudaEvent_t k1 = nullptr) {
    const int tile_step = kVariants[v].block * kVariants[v].ppt;
    const dim3 g2((unsigned)std::max(1, b->ctx->num_sms * 2), (unsigned)std::min(b->K, 64));
    k_bplan<<<1, 1024, 0, s>>>(b->d, 0, tile_step);
    if (k0) cudaEventRecord(k0, s);
    if (int st = launch_variant(b, v, s)) return st;
    if (k1) cudaEventRecord(k1, s);
    k_bempty_moments<<<(b->K + 255) / 256, 256, 0, s>>>(b->d);
    // Swarm.resample!
    k_bplan<<<1, 1024, 0, s>>>(b->d, 1, kBTile);
    k_bsres_count<<<g2, 256, 0, s>>>(b->d);
    k_bzero_tot<<<(b->K + 255) / 256, 256, 0, s>>>(b->d);
    k_bscan<<<b->ctx->num_sms * 4, 256, 0, s>>>(b->d, 1, b->d.u32a, b->d.u32b);
    k_bsres_write<<<g2, 256, 0, s>>>(b->d);
    // repack!
    k_bplan<<<1, 1024, 0, s>>>(b->d, 0, kBTile);
    k_bzero_tot<<<(b->K + 255) / 256, 256, 0, s>>>(b->d);
    k_bscan<<<b->ctx->num_sms * 4, 256, 0, s>>>(b->d, 0, nullptr, b->d.u32b);
    k_brepack_holes<<<g2, 256, 0, s>>>(b->d);
    k_brepack_move<<<g2, 256, 0, s>>>(b->d);
    k_bfinish<<<(b->K + 255) / 256, 256, 0, s>>>(b->d);
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
    b->total_cap = total_capacity;
    b->hinst.assign(max_instances, Inst{});
    b->max_tiles = total_capacity / 128 + max_instances + 1;
    BatchDev& d = b->d;
    int st = MCS_OK;
    for (int q = 0; q < 8 && !st; ++q) st = balloc(b, &d.f[q], (size_t)total_capacity);
    if (!st) st = balloc(b, &d.act, (size_t)total_capacity);
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
    if (!st) st = balloc(b, &d.u32a, (size_t)total_capacity);
    if (!st) st = balloc(b, &d.u32b, (size_t)total_capacity);
    if (!st) st = balloc(b, &d.tot, (size_t)max_instances);
    if (!st) st = balloc(b, &b->d_tabs, kMaxGases);
    // staging for the largest variant grid
    int maxgrid = 0;
    size_t stride = 0;
    for (int v = 0; v < kNumVariants && !st; ++v) {
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kVariants[v].fn, kVariants[v].block, 0);
        b->grid[v] = std::max(occ, 1) * c->num_sms;
        maxgrid = std::max(maxgrid, b->grid[v]);
        const uint32_t cap = 4 * kVariants[v].block * kVariants[v].ppt + 2048;
        stride = std::max(stride, (((size_t)cap * (8 * sizeof(float) + 9)) + 255) & ~(size_t)255);
    }
    char* stage = nullptr;
    if (!st) st = balloc(b, &stage, stride * (size_t)maxgrid);
    if (st) { mcs_batch_destroy(b); return st; }
    d.stage = stage;
    d.stage_stride = stride;
    d.stage_cap = (uint32_t)((stride - 255) / (8 * sizeof(float) + 9));
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
    long long base = 0;
    bool found = false;
    for (auto& u : used) {
        if (u.first - base >= capacity) { found = true; break; }
        base = u.first + u.second;
    }
    if (!found && b->total_cap - base < capacity) return set_err(c, MCS_ERR_NOMEM, "no room for the instance");
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

}  // extern "C"
