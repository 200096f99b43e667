// step_kernel.cuh -- persistent tile skeleton and the step kernels:
//   k_step_abs   absolute positions (swarms, cylindrical parity mode, 3-D field)
//   k_collisions collisions! (fixed-step collision sampling, no push)
//   k_step_mesh  3-D mesh, (cell, in-cell offset) layout, fused tracker + deposit
#pragma once
#include <type_traits>

#include "step.cuh"

namespace mcs {

struct YoshidaC {
    double c1, c2, c3, c4, d1, d2, d3, qm;  // electron.jl:38-46; qm = charge/mass
};

constexpr uint32_t kOutsideCell = 0xffffffffu;

template <typename T, int BLOCK, int TILE>
struct TileShared {
    RowsSmem<T> rows;
    uint32_t cnt[TILE];              // secondaries per tile-local parent, then exclusive prefix
    uint32_t wtot[BLOCK / 32];
    double red[BLOCK / 32][kStepMoments];
    uint32_t count;                  // staged entries of the current tile
    uint32_t next;                   // next unclaimed tile slot (particle queue)
    uint32_t tile;
    uint32_t excl;
    int ok;
    int last;
    unsigned long long pool_off;     // mesh step: the tile's first pool entry
};

// Add one particle to the step sums m[0..kStepMoments).  Every product and sum is rounded
// explicitly, so the bits do not depend on where the compiler contracts into FMAs and all
// kernels that form these sums (single population, batched instances) agree exactly.
template <int N>
__device__ __forceinline__ void mom_add(double (&m)[N], double x, double y, double z, double vx, double vy, double vz,
                                        double w) {
    m[SM_COUNT] = __dadd_rn(m[SM_COUNT], 1.0);
    m[SM_W] = __dadd_rn(m[SM_W], w);
    m[SM_X] = __dadd_rn(m[SM_X], x);
    m[SM_Y] = __dadd_rn(m[SM_Y], y);
    m[SM_Z] = __dadd_rn(m[SM_Z], z);
    m[SM_XX] = __dadd_rn(m[SM_XX], __dmul_rn(x, x));
    m[SM_YY] = __dadd_rn(m[SM_YY], __dmul_rn(y, y));
    m[SM_ZZ] = __dadd_rn(m[SM_ZZ], __dmul_rn(z, z));
    m[SM_VX] = __dadd_rn(m[SM_VX], vx);
    m[SM_VY] = __dadd_rn(m[SM_VY], vy);
    m[SM_VZ] = __dadd_rn(m[SM_VZ], vz);
    const double v2 = __dadd_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)), __dmul_rn(vz, vz));
    m[SM_E] = __dadd_rn(m[SM_E], __dmul_rn(0.5 * kElectronMass, v2));
}

template <typename T>
struct MomAcc {
    double m[kStepMoments];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int q = 0; q < kStepMoments; ++q) m[q] = 0.0;
    }
    __device__ __forceinline__ void add(double x, double y, double z, double vx, double vy, double vz, double w) {
        mom_add(m, x, y, z, vx, vy, vz, w);
    }
};

// Block-reduce one accumulator per thread into out[kStepMoments] (fixed order).
template <int BLOCK, typename SH>
__device__ __forceinline__ void block_reduce_moments(SH& sh, const double (&m)[kStepMoments], double* out) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kStepMoments; ++q) {
        const double v = warp_sum(m[q]);
        if (lane == 0) sh.red[wid][q] = v;
    }
    __syncthreads();
    if (threadIdx.x < kStepMoments) {
        double a = 0.0;
        for (int wv = 0; wv < BLOCK / 32; ++wv) a += sh.red[wv][threadIdx.x];
        out[threadIdx.x] = a;
    }
    __syncthreads();
}

// In-place exclusive scan of sh.cnt[0..TILE) by the whole block.
template <int BLOCK, int TILE, typename SH>
__device__ __forceinline__ void block_scan_counts(SH& sh) {
    constexpr int PER = TILE / BLOCK;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t v[PER];
    uint32_t sum = 0;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        v[q] = sh.cnt[threadIdx.x * PER + q];
        sum += v[q];
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) sh.wtot[wid] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (int q = 0; q < BLOCK / 32; ++q) { const uint32_t t = sh.wtot[q]; sh.wtot[q] = acc; acc += t; }
    }
    __syncthreads();
    uint32_t run = sh.wtot[wid] + incl - sum;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        sh.cnt[threadIdx.x * PER + q] = run;
        run += v[q];
    }
    __syncthreads();
}

// Append the tile's staged secondaries after all earlier tiles' secondaries (called by all
// threads after the particle loop and a __syncthreads).  `writer(e, dst)` stores staged
// entry e into population slot dst.  Returns the number of staged entries.
template <typename T, int BLOCK, int TILE, typename SH, typename Writer>
__device__ __forceinline__ uint32_t tile_append(SH& sh, const Stage<T>& sg, const StepCtl& C, long long tile,
                                                long long ntiles, long long n_entry, long long cap, long long* n_out,
                                                const Writer& writer) {
    uint32_t cnt = sh.count;
    if (cnt > sg.cap) cnt = sg.cap;
    block_scan_counts<BLOCK, TILE>(sh);
    if (threadIdx.x < 32) {   // warp 0 looks back
        bool ok;
        const uint32_t ex = tile_lookback_from_warp(C.tile_status, 0u, (uint32_t)tile, C.epoch, cnt, C.status, &ok);
        if (threadIdx.x == 0) {
            sh.excl = ex;
            sh.ok = ok;
            if (tile == ntiles - 1) {
                long long n = n_entry + (long long)ex + cnt;
                if (n > cap) { n = cap; atomicOr(C.status, ST_CAPACITY); }
                *n_out = n;
            }
        }
    }
    __syncthreads();
    if (sh.ok) {
        for (uint32_t e = threadIdx.x; e < cnt; e += BLOCK) {
            const uint32_t key = sg.key[e];
            const long long dst = n_entry + (long long)sh.excl + sh.cnt[key >> 16] + (key & 0xffffu);
            if (dst >= cap) { atomicOr(C.status, ST_CAPACITY); continue; }
            writer(e, dst);
        }
    }
    return cnt;
}

// Last-CTA epilogue: reduce tile partials in tile order into moments_out, publish the count
// when there were no tiles, and re-arm the tile ticket / done counters for the next launch.
template <int BLOCK, typename SH>
__device__ __forceinline__ void grid_epilogue(SH& sh, const StepCtl& C, long long ntiles, long long n_entry,
                                              long long* n_out) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t d = atomicAdd(&C.counters[1], 1u);
        sh.last = (d == gridDim.x - 1);
    }
    __syncthreads();
    if (!sh.last) return;
    __threadfence();
    if (C.moments_out) {
        double m[kStepMoments];
#pragma unroll
        for (int q = 0; q < kStepMoments; ++q) {
            double a = 0.0, comp = 0.0;  // Kahan over this thread's strided tiles
            for (long long t = threadIdx.x; t < ntiles; t += BLOCK) {
                const double y = C.tile_partials[t * kStepMoments + q] - comp;
                const double s = a + y;
                comp = (s - a) - y;
                a = s;
            }
            m[q] = a;
        }
        block_reduce_moments<BLOCK>(sh, m, C.moments_out);
    }
    if (threadIdx.x == 0) {
        if (ntiles == 0) *n_out = n_entry;
        C.counters[0] = 0;
        C.counters[1] = 0;
    }
}

// Fetch the next tile (or -1 when done); resets the per-tile staging count.
template <typename SH>
__device__ __forceinline__ long long next_tile(SH& sh, const StepCtl& C, long long ntiles) {
    if (threadIdx.x == 0) {
        sh.tile = atomicAdd(&C.counters[0], 1u);
        sh.count = 0;
        sh.next = 0;
    }
    __syncthreads();
    const long long tile = sh.tile;
    return tile < ntiles ? tile : -1;
}

// Process selection of one collision event (do_one_collision!, collisions.jl:159-192): draws
// the event's block and returns the selected row, or -1 for a null collision.
template <typename T, class Ev>
__device__ __forceinline__ int select_event(const TableView& tab, const StepCtl& C, Ev& rng, T vx, T vy, T vz) {
    if constexpr (sizeof(T) == 8) {
        rng.begin();
        const double eng = 0.5 * kElectronMass * ((double)vx * vx + (double)vy * vy + (double)vz * vz);
        const double xi = rng.template xi<double>() * tab.maxrate;
        return select_row64(tab, eng, xi, C.flags, C.status);
    } else {
        // the first rows' loads go out before the event's block is drawn
        const float v2 = fmaf(vx, vx, fmaf(vy, vy, vz * vz));
        Sel32 sel;
        select32_begin(tab, v2, sel);
        rng.begin();
        const float xi = rng.template xi<float>() * tab.maxrate32;
        return select32_finish(tab, sel, xi, C.flags, C.status);
    }
}

// The collision of a selected row `j` of kind `kind` (not K_NULL), applied to the velocity
// in place.  Returns OUT_CHANGE, OUT_NEW (sec filled), OUT_REMOVE or OUT_PHOTO.  The energy
// is recomputed from the velocity by the selection's expression.
template <typename T, typename RowsT, class Ev>
__device__ __forceinline__ int collide_row(const RowsT& rows, int j, int kind, Ev& rng, T& vx, T& vy, T& vz,
                                           Sec<T>& sec) {
    int out;
    if constexpr (sizeof(T) == 8) {
        const double eng = 0.5 * kElectronMass * ((double)vx * vx + (double)vy * vy + (double)vz * vz);
        Sec<double> s64;
        double a = vx, b = vy, c = vz;
        out = collide64(kind, (double)rows.par[j], eng, rng, a, b, c, s64);
        vx = a; vy = b; vz = c;
        sec.vx = s64.vx; sec.vy = s64.vy; sec.vz = s64.vz; sec.s = s64.s;
    } else {
        const float v2 = fmaf(vx, vx, fmaf(vy, vy, vz * vz));
        Sec<float> s32;
        float a = vx, b = vy, c = vz;
        out = collide32(kind, (float)rows.par[j], v2, rng, a, b, c, s32);
        vx = a; vy = b; vz = c;
        sec.vx = s32.vx; sec.vy = s32.vy; sec.vz = s32.vz; sec.s = s32.s;
    }
    return out == OUT_NONE ? OUT_CHANGE : out;
}

// Shared collision body: select a process for velocity (vx, vy, vz) and apply it in place.
// Returns OUT_NONE (null collision), OUT_CHANGE, OUT_NEW (sec filled) or OUT_REMOVE.
template <typename T, typename RowsT, class Ev>
__device__ __forceinline__ int collide_once(const RowsT& rows, const TableView& tab, const StepCtl& C, Ev& rng,
                                            T& vx, T& vy, T& vz, Sec<T>& sec, int* row_out = nullptr) {
    const int j = select_event<T>(tab, C, rng, vx, vy, vz);
    const int kind = j >= 0 ? rows.kind[j] : K_NULL;
    if (row_out) *row_out = j;
    if (kind == K_NULL) return OUT_NONE;
    return collide_row<T>(rows, j, kind, rng, vx, vy, vz, sec);
}

// apply!(::MultiplePhotonOutcome) of an electron's photo-emission (electron.jl:141-144,
// collisions.jl:125-141): rand(Poisson(w / photon_multiplier / photon_weight)) photons of
// collision event `jev` at (x, y, z).  The photons themselves are made after the step, in
// serial parent order, from the recorded event (photons.cu); `pcnt` counts the parent's
// photons of the step so far.
__device__ __forceinline__ void photo_event(const StepCtl& C, const TableView& tab, int row, uint32_t slot_local,
                                            uint32_t jev, double x, double y, double z, double w, uint8_t act,
                                            uint32_t& pcnt) {
    if (!C.photo.events) {
        atomicOr(C.status, ST_UNSUPPORTED);
        return;
    }
    Rng r;
    r.init(C.seed, slot_local + C.slot_base, C.step, TAG_PHOTON_COUNT | jev);
    const long long n = poisson_draw(r, w / tab.pe_mult / tab.pe_pw);
    if (n <= 0) return;
    const uint32_t e = atomicAdd(C.photo.count, 1u);
    if (e < C.photo.cap) {
        PhotoEvent ev;
        ev.x = x; ev.y = y; ev.z = z;
        ev.slot = slot_local; ev.jev = jev; ev.poff = pcnt; ev.nphot = (uint32_t)n;
        ev.row = row; ev.act = act;
        C.photo.events[e] = ev;
    } else {
        atomicOr(C.status, ST_OVERFLOW);
    }
    pcnt += (uint32_t)n;
}

// ---------------------------------------------------------------------------------------
// Absolute-position step (swarms, cylindrical parity mode, 3-D field on absolute positions).
// CLOSED: uniform-field FP32 fast path.  The Yoshida composition is exact for a constant
// force (its drift coefficients sum to 1 and its drift-kick weight is 1/2), so the trajectory
// between real collisions is x0 + v0*tau + a*tau^2/2 and null sub-steps cost no push; the
// sub-step sequence, draws and decisions are those of advance!.
// ---------------------------------------------------------------------------------------
template <typename T, int BLOCK, int PPT, class Field, bool CLOSED, class Ev = Event>
__global__ void __launch_bounds__(BLOCK) k_step_abs(PopView<T> P, TableView tab, GridView fgrid, GridView tgrid,
                                                    StepCtl C, Field field, YoshidaC Y, double ax, double ay,
                                                    double az) {
    constexpr int TILE = BLOCK * PPT;
    __shared__ TileShared<T, BLOCK, TILE> sh;
    load_rows(sh.rows, tab);
    Stage<T> sg;
    sg.init(C);
    const long long n_entry = *P.n_in;
    const long long ntiles = (n_entry + TILE - 1) / TILE;
    const bool tracking = tgrid.type != 0 && tgrid.qfixed != nullptr;

    for (;;) {
        const long long tile = next_tile(sh, C, ntiles);
        if (tile < 0) break;
        const long long base = tile * TILE;

#pragma unroll 1
        for (int jj = 0; jj < PPT; ++jj) {
            const uint32_t local = jj * BLOCK + threadIdx.x;
            const long long i = base + local;
            uint32_t ev = 0;
            uint32_t pcnt = 0;   // photons emitted by this particle in this step
            if (i < n_entry && P.act[i]) {
                Ev rng;
                rng.init(C.seed, (uint32_t)i + C.slot_base, C.step, C.tag);
                if constexpr (!std::is_same<Ev, Event>::value)
                    rng.bind(C.inj_u, C.inj_pos, C.inj_end, C.inj_n, C.status);
                T x = P.f[0][i], y = P.f[1][i], z = P.f[2][i];
                T vx = P.f[3][i], vy = P.f[4][i], vz = P.f[5][i];
                const T w = P.f[6][i];
                double s = (double)P.f[7][i];
                uint8_t act = 1;
                double trem = C.dt;
                float tau = 0.0f;  // CLOSED: time since the last real collision
                while (trem > 0) {
                    double tn, t;
                    if constexpr (sizeof(T) == 8) tn = s / tab.maxrate;
                    else tn = s * tab.inv_maxrate;
                    bool collides;
                    if (trem > tn) { t = tn; collides = true; }
                    else { t = trem; collides = false; s -= t * tab.maxrate; }
                    if constexpr (CLOSED) {
                        tau += (float)t;
                    } else {
                        // advance_free_yoshida, JuMC/src/electron.jl:51-62
                        T ex, ey, ez;
                        T x1 = x + (T)(Y.c1 * t) * vx, y1 = y + (T)(Y.c1 * t) * vy, z1 = z + (T)(Y.c1 * t) * vz;
                        field(fgrid, x1, y1, z1, ex, ey, ez, C.status);
                        const T k1 = (T)((Y.d1 * t) * Y.qm);
                        T vx1 = vx + k1 * ex, vy1 = vy + k1 * ey, vz1 = vz + k1 * ez;
                        T x2 = x1 + (T)(Y.c2 * t) * vx1, y2 = y1 + (T)(Y.c2 * t) * vy1, z2 = z1 + (T)(Y.c2 * t) * vz1;
                        field(fgrid, x2, y2, z2, ex, ey, ez, C.status);
                        const T k2 = (T)((Y.d2 * t) * Y.qm);
                        T vx2 = vx1 + k2 * ex, vy2 = vy1 + k2 * ey, vz2 = vz1 + k2 * ez;
                        T x3 = x2 + (T)(Y.c3 * t) * vx2, y3 = y2 + (T)(Y.c3 * t) * vy2, z3 = z2 + (T)(Y.c3 * t) * vz2;
                        field(fgrid, x3, y3, z3, ex, ey, ez, C.status);
                        const T k3 = (T)((Y.d3 * t) * Y.qm);
                        vx = vx2 + k3 * ex; vy = vy2 + k3 * ey; vz = vz2 + k3 * ez;
                        x = x3 + (T)(Y.c4 * t) * vx; y = y3 + (T)(Y.c4 * t) * vy; z = z3 + (T)(Y.c4 * t) * vz;
                    }
                    if (collides) {
                        // do_one_collision!, collisions.jl:159-192
                        T cvx = vx, cvy = vy, cvz = vz;
                        if constexpr (CLOSED) {
                            cvx = fmaf((float)ax, tau, (float)vx);
                            cvy = fmaf((float)ay, tau, (float)vy);
                            cvz = fmaf((float)az, tau, (float)vz);
                        }
                        Sec<T> sec;
                        int row = -1;
                        const int out = collide_once<T>(sh.rows, tab, C, rng, cvx, cvy, cvz, sec, &row);
                        if (out == OUT_PHOTO) {
                            double px = (double)x, py = (double)y, pz = (double)z;
                            if constexpr (CLOSED) {   // the position at the collision time
                                const float h2 = 0.5f * tau * tau;
                                px = fmaf((float)ax, h2, fmaf((float)vx, tau, (float)x));
                                py = fmaf((float)ay, h2, fmaf((float)vy, tau, (float)y));
                                pz = fmaf((float)az, h2, fmaf((float)vz, tau, (float)z));
                            }
                            photo_event(C, tab, row, local + (uint32_t)base, rng.jev(), px, py, pz, (double)w, act,
                                        pcnt);
                        } else if (out != OUT_NONE) {
                            if constexpr (CLOSED) {  // settle the segment at the collision time
                                const float h2 = 0.5f * tau * tau;
                                x = fmaf((float)ax, h2, fmaf((float)vx, tau, (float)x));
                                y = fmaf((float)ay, h2, fmaf((float)vy, tau, (float)y));
                                z = fmaf((float)az, h2, fmaf((float)vz, tau, (float)z));
                                tau = 0.0f;
                            }
                            vx = cvx; vy = cvy; vz = cvz;
                        }
                        if (out == OUT_NEW) {
                            if (tracking) track_abs(tgrid, (double)x, (double)y, (double)z, (double)w, C.status);
                            const T vals[8] = {x, y, z, sec.vx, sec.vy, sec.vz, w, sec.s};
                            stage(sg, &sh.count, local, ev++, vals, 0u, act, C.status);
                        } else if (out == OUT_REMOVE) {
                            if (tracking) track_abs(tgrid, (double)x, (double)y, (double)z, -(double)w, C.status);
                            act = 0;  // the particle keeps sub-stepping (mixed_population.jl:32)
                        }
                        if constexpr (sizeof(T) == 8) s = -log(rng.template snew<double>());
                        else s = (double)M<float>::nlog(rng.template snew<float>());
                    }
                    trem -= t;
                }
                rng.finish();
                if constexpr (CLOSED) {
                    const float h2 = 0.5f * tau * tau;
                    x = fmaf((float)ax, h2, fmaf((float)vx, tau, (float)x));
                    y = fmaf((float)ay, h2, fmaf((float)vy, tau, (float)y));
                    z = fmaf((float)az, h2, fmaf((float)vz, tau, (float)z));
                    vx = fmaf((float)ax, tau, (float)vx);
                    vy = fmaf((float)ay, tau, (float)vy);
                    vz = fmaf((float)az, tau, (float)vz);
                }
                P.f[0][i] = x; P.f[1][i] = y; P.f[2][i] = z;
                P.f[3][i] = vx; P.f[4][i] = vy; P.f[5][i] = vz;
                P.f[7][i] = (T)s;
                if (!act) P.act[i] = 0;
            }
            if (C.photo.per_slot && i < n_entry) C.photo.per_slot[i] = pcnt;
            sh.cnt[local] = ev;
        }
        __syncthreads();

        const uint32_t cnt = tile_append<T, BLOCK, TILE>(
            sh, sg, C, tile, ntiles, n_entry, P.cap, P.n_out, [&](uint32_t e, long long dst) {
#pragma unroll
                for (int q = 0; q < 8; ++q) P.f[q][dst] = sg.f[q][e];
                P.act[dst] = sg.act[e];
            });

        if (C.moments_out) {
            MomAcc<T> acc;
            acc.zero();
            for (int jj = 0; jj < PPT; ++jj) {
                const long long i = base + jj * BLOCK + threadIdx.x;
                if (i < n_entry && P.act[i])
                    acc.add(P.f[0][i], P.f[1][i], P.f[2][i], P.f[3][i], P.f[4][i], P.f[5][i], P.f[6][i]);
            }
            // secondaries in their appended (serial) order, so the sums do not depend on the
            // order in which lanes staged them
            __syncthreads();
            const long long d0 = n_entry + (long long)sh.excl;
            for (uint32_t r = threadIdx.x; r < cnt; r += BLOCK) {
                const long long d = d0 + r;
                if (sh.ok && d < P.cap && P.act[d])
                    acc.add(P.f[0][d], P.f[1][d], P.f[2][d], P.f[3][d], P.f[4][d], P.f[5][d], P.f[6][d]);
            }
            block_reduce_moments<BLOCK>(sh, acc.m, C.tile_partials + tile * kStepMoments);
        }
        __syncthreads();
    }
    grid_epilogue<BLOCK>(sh, C, ntiles, n_entry, P.n_out);
}

// ---------------------------------------------------------------------------------------
// collisions!(mpopl, dt, tracker): JuMC/src/mixed_population.jl:61-77 (no push).
// ---------------------------------------------------------------------------------------
template <typename T, int BLOCK, int PPT, class Ev = Event>
__global__ void __launch_bounds__(BLOCK) k_collisions(PopView<T> P, TableView tab, GridView tgrid, StepCtl C) {
    constexpr int TILE = BLOCK * PPT;
    __shared__ TileShared<T, BLOCK, TILE> sh;
    load_rows(sh.rows, tab);
    Stage<T> sg;
    sg.init(C);
    const long long n_entry = *P.n_in;
    const long long ntiles = (n_entry + TILE - 1) / TILE;
    const bool tracking = tgrid.type != 0 && tgrid.qfixed != nullptr;
    for (;;) {
        const long long tile = next_tile(sh, C, ntiles);
        if (tile < 0) break;
        const long long base = tile * TILE;
        for (int jj = 0; jj < PPT; ++jj) {
            const uint32_t local = jj * BLOCK + threadIdx.x;
            const long long i = base + local;
            uint32_t ev = 0;
            if (i < n_entry && P.act[i]) {
                double s = (double)P.f[7][i] - C.dt * tab.maxrate;
                if (s <= 0) {
                    Ev rng;
                    rng.init(C.seed, (uint32_t)i + C.slot_base, C.step, C.tag);
                    if constexpr (!std::is_same<Ev, Event>::value)
                        rng.bind(C.inj_u, C.inj_pos, C.inj_end, C.inj_n, C.status);
                    const T x = P.f[0][i], y = P.f[1][i], z = P.f[2][i];
                    T vx = P.f[3][i], vy = P.f[4][i], vz = P.f[5][i];
                    const T w = P.f[6][i];
                    Sec<T> sec;
                    const int out = collide_once<T>(sh.rows, tab, C, rng, vx, vy, vz, sec);
                    if (out == OUT_PHOTO) atomicOr(C.status, ST_UNSUPPORTED);
                    if (out == OUT_NEW) {
                        if (tracking) track_abs(tgrid, (double)x, (double)y, (double)z, (double)w, C.status);
                        const T vals[8] = {x, y, z, sec.vx, sec.vy, sec.vz, w, sec.s};
                        stage(sg, &sh.count, local, ev++, vals, 0u, (uint8_t)1, C.status);
                    } else if (out == OUT_REMOVE) {
                        if (tracking) track_abs(tgrid, (double)x, (double)y, (double)z, -(double)w, C.status);
                        P.act[i] = 0;
                    }
                    if constexpr (sizeof(T) == 8) s = -log(rng.template snew<double>());
                    else s = (double)M<float>::nlog(rng.template snew<float>());
                    rng.finish();
                    P.f[3][i] = vx; P.f[4][i] = vy; P.f[5][i] = vz;
                }
                P.f[7][i] = (T)s;
            }
            sh.cnt[local] = ev;
        }
        __syncthreads();
        tile_append<T, BLOCK, TILE>(sh, sg, C, tile, ntiles, n_entry, P.cap, P.n_out, [&](uint32_t e, long long dst) {
#pragma unroll
            for (int q = 0; q < 8; ++q) P.f[q][dst] = sg.f[q][e];
            P.act[dst] = sg.act[e];
        });
        __syncthreads();
    }
    grid_epilogue<BLOCK>(sh, C, ntiles, n_entry, P.n_out);
}

// ---------------------------------------------------------------------------------------
// 3-D mesh layout.  The trilinear field of one cell as a polynomial in the in-cell offset
// f in [0,1)^3:  E(f) = a + fx*(bx + fy*(bxy + fz*bxyz) + fz*bxz) + fy*(by + fz*byz) + fz*bz,
// 24 coefficients held in registers while the particle stays in the cell.
// ---------------------------------------------------------------------------------------
template <typename T>
struct CellField {
    T a[3], bx[3], by[3], bz[3], bxy[3], bxz[3], byz[3], bxyz[3];

    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int c = 0; c < 3; ++c) a[c] = bx[c] = by[c] = bz[c] = bxy[c] = bxz[c] = byz[c] = bxyz[c] = (T)0;
    }
    __device__ __forceinline__ void set(const T (&e)[8][3]) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const T e000 = e[0][c], e100 = e[1][c], e010 = e[2][c], e110 = e[3][c];
            const T e001 = e[4][c], e101 = e[5][c], e011 = e[6][c], e111 = e[7][c];
            a[c] = e000;
            bx[c] = e100 - e000;
            by[c] = e010 - e000;
            bz[c] = e001 - e000;
            bxy[c] = (e110 - e010) - (e100 - e000);
            bxz[c] = (e101 - e001) - (e100 - e000);
            byz[c] = (e011 - e001) - (e010 - e000);
            bxyz[c] = ((e111 - e011) - (e101 - e001)) - ((e110 - e010) - (e100 - e000));
        }
    }
    __device__ __forceinline__ void eval(T fx, T fy, T fz, T& ex, T& ey, T& ez) const {
        T r[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const T tx = bx[c] + fy * (bxy[c] + fz * bxyz[c]) + fz * bxz[c];
            const T ty = by[c] + fz * byz[c];
            r[c] = a[c] + fx * tx + fy * ty + fz * bz[c];
        }
        ex = r[0]; ey = r[1]; ez = r[2];
    }
};

// Node field of cell (ix,iy,iz): corners 000,100,010,110,001,101,011,111 (x fastest).
template <typename T>
__device__ __forceinline__ void load_cell_field(const GridView& g, int ix, int iy, int iz, CellField<T>& cf) {
    const long long sy = g.nx + 1, sz = (long long)(g.nx + 1) * (g.ny + 1);
    const long long b = ix + iy * sy + iz * sz;
    T e[8][3];
    if constexpr (sizeof(T) == 4) {
        const float4* n4 = reinterpret_cast<const float4*>(g.e32);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const float4 v = __ldg(n4 + b + (q & 1) + ((q >> 1) & 1) * sy + (q >> 2) * sz);
            e[q][0] = v.x; e[q][1] = v.y; e[q][2] = v.z;
        }
    } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const double* p = g.e64 + 3 * (b + (q & 1) + ((q >> 1) & 1) * sy + (q >> 2) * sz);
            e[q][0] = __ldg(p); e[q][1] = __ldg(p + 1); e[q][2] = __ldg(p + 2);
        }
    }
    cf.set(e);
}

// Renormalise (cell, offset) after a drift; returns true when the field must be reloaded.
// Inside the mesh the offset is in [0,1) of cell (ix,iy,iz); outside (in == false) the
// offset holds the absolute position in cell units and the field is zero.
template <typename T>
__device__ __forceinline__ bool relocate(const GridView& g, int& ix, int& iy, int& iz, bool& in, T& ox, T& oy, T& oz) {
    if (in && ox >= (T)0 && ox < (T)1 && oy >= (T)0 && oy < (T)1 && oz >= (T)0 && oz < (T)1) return false;
    T o[3] = {ox, oy, oz};
    int ic[3] = {ix, iy, iz};
    if (!in) { ic[0] = ic[1] = ic[2] = 0; }
    bool inside = true;
    const int nc[3] = {g.nx, g.ny, g.nz};
    double cd[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        T fl = floor(o[d]);
        T r = o[d] - fl;
        if (r >= (T)1) { r -= (T)1; fl += (T)1; }
        cd[d] = (double)ic[d] + (double)fl;
        inside = inside && cd[d] >= 0.0 && cd[d] < (double)nc[d];
        o[d] = r;
    }
    if (inside) {
        ix = (int)cd[0]; iy = (int)cd[1]; iz = (int)cd[2];
        ox = o[0]; oy = o[1]; oz = o[2];
    } else {
        ox = (T)(cd[0] + (double)o[0]);
        oy = (T)(cd[1] + (double)o[1]);
        oz = (T)(cd[2] + (double)o[2]);
    }
    const bool reload = inside || in;
    in = inside;
    return reload;
}

__device__ __forceinline__ uint32_t cell_index(const GridView& g, bool in, int ix, int iy, int iz) {
    return in ? (uint32_t)ix + (uint32_t)g.nx * ((uint32_t)iy + (uint32_t)g.ny * (uint32_t)iz) : kOutsideCell;
}

// Absolute position of a (cell, offset) pair.
__device__ __forceinline__ void mesh_abs(const GridView& g, uint32_t cell, double ox, double oy, double oz, double& x,
                                         double& y, double& z) {
    double cx = 0.0, cy = 0.0, cz = 0.0;
    if (cell != kOutsideCell) {
        uint32_t ux, uy, uz;
        cell_split(g, cell, ux, uy, uz);
        cx = (double)ux;
        cy = (double)uy;
        cz = (double)uz;
    }
    x = g.x0 + g.h * (cx + ox);
    y = g.y0 + g.h * (cy + oy);
    z = g.z0 + g.h * (cz + oz);
}

// ---------------------------------------------------------------------------------------
// Mesh-layout step: advance! with the trilinear node-field gather of a 3-D mesh, the
// collision tracker (+w ionization / -w attachment into qfixed, CIC int64) and, when
// dep_val != 0, the particle deposit density!(qpart, dep_val) of the post-step state.
//
// Work distribution: a particle needs a variable number of sub-steps (one per real or null
// collision), so a fixed particle-per-lane mapping leaves most lanes of a warp idle while
// the slowest particle finishes.  Here every lane executes one sub-step per loop pass and,
// when its particle is done, takes the tile's next particle from a shared-memory counter;
// the warp stays converged on the sub-step body and the idle tail is about one particle.
// ---------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ bool in_unit_cube(T ox, T oy, T oz) {
    if constexpr (sizeof(T) == 4) {
        // offsets in [0,1) <=> bit patterns below 1.0f (negative values have the sign bit)
        const uint32_t m = max(__float_as_uint(ox), max(__float_as_uint(oy), __float_as_uint(oz)));
        return m < 0x3f800000u;
    } else {
        return ox >= 0.0 && ox < 1.0 && oy >= 0.0 && oy < 1.0 && oz >= 0.0 && oz < 1.0;
    }
}

template <typename T, int BLOCK, int PPT, int MINB = 1, int REFILL = 8>
__global__ void __launch_bounds__(BLOCK, MINB) k_step_mesh(PopView<T> P, TableView tab, GridView g, int tracking, StepCtl C,
                                                     YoshidaC Y, double dep_val) {
    constexpr int TILE = BLOCK * PPT;
    __shared__ TileShared<T, BLOCK, TILE> sh;
    load_rows(sh.rows, tab);
    Stage<T> sg;
    sg.init(C);
    const long long n_entry = *P.n_in;
    const long long ntiles = (n_entry + TILE - 1) / TILE;
    // drift / kick factors per unit time: offsets in cell units, velocities in m/s
    const T cd1 = (T)(Y.c1 * g.inv_h), cd2 = (T)(Y.c2 * g.inv_h), cd3 = (T)(Y.c3 * g.inv_h), cd4 = (T)(Y.c4 * g.inv_h);
    const T kd1 = (T)(Y.d1 * Y.qm), kd2 = (T)(Y.d2 * Y.qm), kd3 = (T)(Y.d3 * Y.qm);

    for (;;) {
        const long long tile = next_tile(sh, C, ntiles);
        if (tile < 0) break;
        const long long base = tile * TILE;
        const long long rest = n_entry - base;
        const uint32_t tile_n = rest < TILE ? (uint32_t)rest : (uint32_t)TILE;

        // per-lane particle state
        bool have = false, drained = false;
        uint32_t local = 0;
        long long i = 0;
        Event rng;
        T ox = 0, oy = 0, oz = 0, vx = 0, vy = 0, vz = 0, w = 0;
        double s = 0.0, trem = 0.0;
        bool in = false;
        int ix = 0, iy = 0, iz = 0;
        CellField<T> cf;
        uint8_t act = 1;
        uint32_t ev = 0;

        auto drift = [&](T c) {
            ox += c * vx; oy += c * vy; oz += c * vz;
            if (in && in_unit_cube(ox, oy, oz)) return;
            if (relocate(g, ix, iy, iz, in, ox, oy, oz)) {
                if (in) load_cell_field(g, ix, iy, iz, cf);
                else cf.zero();
            }
        };
        auto kick = [&](T k) {
            T ex, ey, ez;
            cf.eval(ox, oy, oz, ex, ey, ez);
            vx += k * ex; vy += k * ey; vz += k * ez;
        };

        // the collision of a selected row (not a null one) of the lane's particle
        auto real_collision = [&](int row) {
            Sec<T> sec;
            const int out = collide_row<T>(sh.rows, row, sh.rows.kind[row], rng, vx, vy, vz, sec);
            if (out == OUT_PHOTO) atomicOr(C.status, ST_UNSUPPORTED);
            if ((out == OUT_NEW || out == OUT_REMOVE) && tracking && in)
                cic_fixed(g.qfixed, g.nx, g.ny, ix, iy, iz, (double)ox, (double)oy, (double)oz,
                          out == OUT_NEW ? (double)w : -(double)w, C.status);
            if (out == OUT_NEW) {
                const T vals[8] = {ox, oy, oz, sec.vx, sec.vy, sec.vz, w, sec.s};
                stage(sg, &sh.count, local, ev++, vals, cell_index(g, in, ix, iy, iz), act, C.status);
            } else if (out == OUT_REMOVE) {
                act = 0;
            }
        };

        bool pending = false;   // finished particle not yet written back
        for (;;) {
            // Finished lanes wait until REFILL lanes of the warp are idle (or all of it),
            // then write back and refill together: the store/load path runs with many
            // lanes active instead of once per finishing lane.
            const unsigned idle = __ballot_sync(0xffffffffu, !have);
            if (idle != 0xffffffffu && __popc(idle) < REFILL) goto substep;
            if (!have && pending) {
                P.cell[i] = cell_index(g, in, ix, iy, iz);
                P.f[0][i] = ox; P.f[1][i] = oy; P.f[2][i] = oz;
                P.f[3][i] = vx; P.f[4][i] = vy; P.f[5][i] = vz;
                P.f[7][i] = (T)s;
                if (!act) P.act[i] = 0;
                sh.cnt[local] = ev;
                pending = false;
            }
            // refill: an idle lane takes the next particle of the tile
            while (!have && !drained) {
                const uint32_t q = atomicAdd(&sh.next, 1u);
                if (q >= (uint32_t)TILE) { drained = true; break; }
                if (q >= tile_n) { sh.cnt[q] = 0; continue; }
                // the slot's flag, cell and state in one round of loads, then the test
                const long long i2 = base + q;
                const uint8_t a = P.act[i2];
                const uint32_t cell0 = P.cell[i2];
                T f[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) f[k] = P.f[k][i2];
                if (!a) { sh.cnt[q] = 0; continue; }
                local = q;
                i = i2;
                rng.init(C.seed, (uint32_t)i + C.slot_base, C.step, C.tag);
                ox = f[0]; oy = f[1]; oz = f[2];
                vx = f[3]; vy = f[4]; vz = f[5];
                w = f[6];
                s = (double)f[7];
                in = cell0 != kOutsideCell;
                if (in) {
                    uint32_t ux, uy, uz;
                    cell_split(g, cell0, ux, uy, uz);
                    ix = (int)ux;
                    iy = (int)uy;
                    iz = (int)uz;
                    load_cell_field(g, ix, iy, iz, cf);
                } else {
                    cf.zero();
                }
                act = 1;
                ev = 0;
                trem = C.dt;
                have = trem > 0;
                if (!have) sh.cnt[q] = 0;   // dt == 0: nothing to do, state unchanged
            }
            if (!__any_sync(0xffffffffu, have)) break;
        substep:
            if (!have) continue;

            // one sub-step of advance! (mixed_population.jl:32-51)
            double tn, t;
            if constexpr (sizeof(T) == 8) tn = s / tab.maxrate;
            else tn = s * tab.inv_maxrate;
            bool collides;
            if (trem > tn) { t = tn; collides = true; }
            else { t = trem; collides = false; s -= t * tab.maxrate; }
            const T tt = (T)t;
            // advance_free_yoshida (electron.jl:51-62) in cell units
            drift(cd1 * tt);
            kick(kd1 * tt);
            drift(cd2 * tt);
            kick(kd2 * tt);
            drift(cd3 * tt);
            kick(kd3 * tt);
            drift(cd4 * tt);
            if (collides) {
                const int row = select_event<T>(tab, C, rng, vx, vy, vz);
                if (row >= 0 && sh.rows.kind[row] != K_NULL) real_collision(row);
                // the next free flight comes from the event's block, whatever the outcome
                if constexpr (sizeof(T) == 8) s = -log(rng.template snew<double>());
                else s = (double)M<float>::nlog(rng.template snew<float>());
            }
            trem -= t;
            if (!(trem > 0)) {
                have = false;
                pending = true;
            }
        }
        __syncthreads();

        // density!(qpart, dep_val) of the tile's post-step particles, in slot order so that
        // cell-sorted neighbours share their atomics (cic_fixed_warp); the data is L2-hot
        if (dep_val != 0.0) {
            for (uint32_t q0 = 0; q0 < tile_n; q0 += BLOCK) {
                const uint32_t q = q0 + threadIdx.x;
                const long long j = base + q;
                bool valid = false;
                uint32_t cl = kOutsideCell;
                int dx = 0, dy = 0, dz = 0;
                double fx = 0.0, fy = 0.0, fz = 0.0, ch = 0.0;
                if (q < tile_n) {
                    // all six loads at once (one L2 round trip), then the tests
                    const uint8_t a = P.act[j];
                    const uint32_t c0 = P.cell[j];
                    const T x0 = P.f[0][j], y0 = P.f[1][j], z0 = P.f[2][j], w0 = P.f[6][j];
                    if (a && c0 != kOutsideCell) {
                        valid = true;
                        cl = c0;
                        uint32_t ux, uy, uz;
                        cell_split(g, cl, ux, uy, uz);
                        dx = (int)ux;
                        dy = (int)uy;
                        dz = (int)uz;
                        fx = (double)x0; fy = (double)y0; fz = (double)z0;
                        ch = (double)w0 * dep_val;
                    }
                }
                cic_fixed_warp(g.qpart, g.nx, g.ny, valid, cl, dx, dy, dz, fx, fy, fz, ch, C.status);
            }
        }

        // The tile's secondaries go to the pool in their serial order (parent, event), at
        // entries reserved without waiting for the tiles before it; k_pool_copy appends
        // the tiles' runs after the population in tile order once every tile is done.
        const uint32_t cnt = sh.count < sg.cap ? sh.count : sg.cap;
        block_scan_counts<BLOCK, TILE>(sh);
        if (threadIdx.x == 0) {
            const unsigned long long off = cnt ? atomicAdd(C.pool_top, (unsigned long long)cnt) : 0ull;
            sh.pool_off = off;
            C.app_cnt[tile] = cnt;
            C.app_off[tile] = off;
        }
        __syncthreads();
        const unsigned long long poff = sh.pool_off;
        for (uint32_t e = threadIdx.x; e < cnt; e += BLOCK) {
            const uint32_t key = sg.key[e];
            const uint32_t rank = sh.cnt[key >> 16] + (key & 0xffffu);
            if (rank >= cnt) continue;   // only when staging overflowed (ST_OVERFLOW raised)
            const unsigned long long q = poff + rank;
            if (q >= (unsigned long long)P.cap) { atomicOr(C.status, ST_CAPACITY); continue; }
#pragma unroll
            for (int k = 0; k < 8; ++k) static_cast<T*>(C.pool_f[k])[q] = sg.f[k][e];
            C.pool_cell[q] = sg.cell[e];
            C.pool_act[q] = sg.act[e];
        }
        // secondaries are part of the post-step population: deposit them too
        if (dep_val != 0.0) {
            for (uint32_t e = threadIdx.x; e < cnt; e += BLOCK) {
                const uint32_t cl = sg.cell[e];
                if (!sg.act[e] || cl == kOutsideCell) continue;
                uint32_t ux, uy, uz;
                cell_split(g, cl, ux, uy, uz);
                cic_fixed(g.qpart, g.nx, g.ny, (int)ux, (int)uy, (int)uz, (double)sg.f[0][e], (double)sg.f[1][e],
                          (double)sg.f[2][e], (double)sg.f[6][e] * dep_val, C.status);
            }
        }
        if (C.moments_out) {
            MomAcc<T> acc;
            acc.zero();
            double x, y, z;
            for (uint32_t q = threadIdx.x; q < tile_n; q += BLOCK) {
                const long long j = base + q;
                if (P.act[j]) {
                    mesh_abs(g, P.cell[j], (double)P.f[0][j], (double)P.f[1][j], (double)P.f[2][j], x, y, z);
                    acc.add(x, y, z, P.f[3][j], P.f[4][j], P.f[5][j], P.f[6][j]);
                }
            }
            // secondaries in their serial order, from the pool (sums independent of staging order)
            __syncthreads();
            const T* const* pf = reinterpret_cast<T* const*>(C.pool_f);
            for (uint32_t r = threadIdx.x; r < cnt; r += BLOCK) {
                const unsigned long long d = poff + r;
                if (d < (unsigned long long)P.cap && C.pool_act[d]) {
                    mesh_abs(g, C.pool_cell[d], (double)pf[0][d], (double)pf[1][d], (double)pf[2][d], x, y, z);
                    acc.add(x, y, z, pf[3][d], pf[4][d], pf[5][d], pf[6][d]);
                }
            }
            block_reduce_moments<BLOCK>(sh, acc.m, C.tile_partials + tile * kStepMoments);
        }
        __syncthreads();
    }
    grid_epilogue<BLOCK>(sh, C, ntiles, n_entry, P.n_out);
}

// ---------------------------------------------------------------------------------------
// Append of the mesh step's secondaries.  k_step_mesh leaves each tile's secondaries as a run
// in the pool (app_off[t], app_cnt[t] entries, serial order within the tile); the runs go
// after the population in tile order, which is the serial reference order (ascending parent).
// ---------------------------------------------------------------------------------------
// One block: exclusive scan of the tiles' counts (each thread a contiguous range of tiles),
// the population count after the step, and the pool's reset for the next launch.
template <int NT>
__global__ void __launch_bounds__(NT) k_pool_scan(const long long* n_in, long long* n_out, long long cap, int tile_sz,
                                                  const uint32_t* cnt, unsigned long long* excl,
                                                  unsigned long long* pool_top, uint32_t* status) {
    __shared__ unsigned long long wsum[NT / 32];
    const long long n_entry = *n_in;
    const long long ntiles = (n_entry + tile_sz - 1) / tile_sz;
    const long long per = (ntiles + NT - 1) / NT;
    const long long t0 = (long long)threadIdx.x * per;
    const long long t1 = t0 + per < ntiles ? t0 + per : ntiles;
    unsigned long long sum = 0;
    for (long long t = t0; t < t1; ++t) sum += cnt[t];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned long long incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long a = 0;
        for (int w = 0; w < NT / 32; ++w) { const unsigned long long v = wsum[w]; wsum[w] = a; a += v; }
        long long n = n_entry + (long long)a;
        if (n > cap) { n = cap; atomicOr(status, ST_CAPACITY); }
        *n_out = n;
        *pool_top = 0;
    }
    __syncthreads();
    unsigned long long run = wsum[wid] + incl - sum;
    for (long long t = t0; t < t1; ++t) {
        excl[t] = run;
        run += cnt[t];
    }
}

// Copy each tile's run from the pool to its place after the population (a block per tile).
template <typename T>
__global__ void __launch_bounds__(128) k_pool_copy(PopView<T> P, StepCtl C, int tile_sz, const unsigned long long* excl) {
    const long long n_entry = *P.n_in;
    const long long ntiles = (n_entry + tile_sz - 1) / tile_sz;
    const T* const* pf = reinterpret_cast<T* const*>(C.pool_f);
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const uint32_t c = C.app_cnt[t];
        const unsigned long long src0 = C.app_off[t];
        const long long dst0 = n_entry + (long long)excl[t];
        for (uint32_t r = threadIdx.x; r < c; r += blockDim.x) {
            const unsigned long long src = src0 + r;
            const long long dst = dst0 + r;
            if (dst >= P.cap || src >= (unsigned long long)P.cap) continue;   // flagged by the step / scan
#pragma unroll
            for (int q = 0; q < 8; ++q) P.f[q][dst] = pf[q][src];
            P.cell[dst] = C.pool_cell[src];
            P.act[dst] = C.pool_act[src];
        }
    }
}

}  // namespace mcs
