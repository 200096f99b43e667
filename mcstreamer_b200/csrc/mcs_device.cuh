// mcs_device.cuh -- device-side building blocks shared by every kernel of the library:
// Philox4x32-10 streams, uniform conversion, status bits, the ordered-append tile
// protocol (decoupled look-back) and block reductions.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mcs {

constexpr double kElementaryCharge = 1.6021766208e-19;  // JuMC/src/constants.jl:50
constexpr double kElectronMass = 9.10938356e-31;        // JuMC/src/constants.jl:52

// Sticky device status bits (atomicOr into the context's status word).
enum : uint32_t {
    ST_CAPACITY = 1u,    // population capacity exceeded (population.jl:90 assert)
    ST_ENERGY = 2u,      // energy outside the collision table (util.jl:28 assert)
    ST_FIELD = 4u,       // |E| > 1e8 V/m (gridfields.jl:179-187)
    ST_NONFINITE = 8u,   // NaN/Inf in particle state
    ST_OVERFLOW = 16u,   // a tile produced more secondaries than its staging holds
    ST_TIMEOUT = 32u,    // a bounded wait gave up
    ST_UNSUPPORTED = 64u,  // a process this kernel does not apply (photo-emission without photons)
    ST_UNIFORMS = 128u,    // a particle ran past its injected uniforms
    ST_CHARGE = 256u,      // a charge beyond the int64 fixed-point range of the deposits
};

// Int64 fixed-point deposits count charge in units of 2^-32 e: one particle's charge must
// stay below 2^30 e (W < 2^62), and a node or cell sum at or above 2^62 units (2^30 e) is
// reported before it can reach 2^63.
constexpr double kMaxDepositCharge = 0x1p30;
constexpr long long kMaxNodeCharge = 1LL << 62;

// Philox stream tags (4th counter word); must match the oracle.
enum : uint32_t { TAG_ADVANCE = 0, TAG_SWARM_RESAMPLE = 1, TAG_CELL_RESAMPLE = 2, TAG_INIT = 3,
                  TAG_COLLISIONS = 4, TAG_PHOTON = 5, TAG_DENSITY = 6 };
// initfromfiles!: cell c's count draws from {c, 0, k/4, TAG_DENSITY}, its electron k from the four
// words of {c, k, 0, TAG_DENSITY | TAG_DENSITY_PARTICLE} (r, z, phi, s).
constexpr uint32_t TAG_DENSITY_PARTICLE = 0x40000000u;
// Photo-emission streams of collision event j of an electron: the photon count draws from
// {slot, step, k/4, TAG_PHOTON_COUNT | j}, photon p from {slot, step, p, TAG_PHOTON_DRAW | j}.
constexpr uint32_t TAG_PHOTON_COUNT = 0x20000000u;
constexpr uint32_t TAG_PHOTON_DRAW = 0x40000000u;

// Process kinds; must match include/mcs.h.
enum : int { K_NULL = 0, K_ELASTIC = 1, K_EXCITATION = 2, K_IONIZATION = 3, K_ATTACHMENT = 4,
             K_IONIZATION_UNIFORM = 5, K_PHOTOEMISSION = 6 };

// ---------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11).  Counter = {c0, c1, block, tag}, key = 64-bit seed.
// ---------------------------------------------------------------------------------------
struct U4 { uint32_t x, y, z, w; };

__device__ __forceinline__ U4 philox10(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        // one 32x32 -> 64-bit product per multiplier gives both halves
        const unsigned long long p0 = 0xD2511F53ull * c.x, p1 = 0xCD9E8D57ull * c.z;
        c = U4{(uint32_t)(p1 >> 32) ^ c.y ^ k0, (uint32_t)p1, (uint32_t)(p0 >> 32) ^ c.w ^ k1, (uint32_t)p0};
    }
    return c;
}

// One particle's (or cell's) uniform stream: word #k comes from block k/4, lane k%4.
struct Rng {
    uint32_t k0, k1, c0, c1, tag, k;
    U4 buf;
    __device__ __forceinline__ void init(uint64_t seed, uint32_t a, uint32_t b, uint32_t t) {
        k0 = (uint32_t)seed; k1 = (uint32_t)(seed >> 32); c0 = a; c1 = b; tag = t; k = 0;
    }
    __device__ __forceinline__ uint32_t word() {
        const uint32_t lane = k & 3u;
        if (lane == 0) buf = philox10(U4{c0, c1, k >> 2, tag}, k0, k1);
        ++k;
        uint32_t r = buf.x;
        r = lane == 1 ? buf.y : r;
        r = lane == 2 ? buf.z : r;
        r = lane == 3 ? buf.w : r;
        return r;
    }
    // (w + 0.5) * 2^-32, bit-identical to the oracle's uniform.
    __device__ __forceinline__ double u64() { return __fma_rn((double)word(), 0x1p-32, 0x1p-33); }
    // float in (0, 1]: the float nearest to the same uniform (within one ulp).
    __device__ __forceinline__ float u32() { return __uint2float_rn(word() | 1u) * 0x1p-32f; }
};

__device__ __forceinline__ double uni64(uint32_t w) { return __fma_rn((double)w, 0x1p-32, 0x1p-33); }
__device__ __forceinline__ float uni32(uint32_t w) { return __uint2float_rn(w | 1u) * 0x1p-32f; }

// The draws of one collision event (do_one_collision! plus the new free-flight time).
// Event j of particle `slot` during step `step` owns block b = Philox(seed; {slot, step, j,
// tag}) -- xi, new s, direction (phi, u) -- and, only for processes that need more,
// c = Philox(seed; {slot, step, j | 2^31, tag}) -- secondary direction, secondary s and the
// energy-sharing fraction.  Every colliding lane generates its block at the same point of
// the sub-step, so the generator runs converged across the warp.
//
// The collision code reads the draws through named accessors, called in the order the
// reference draws them (xi; the process's own draws; the new s), which is what lets the
// injected source below replay a serial stream.  T = double gives the FP64 uniform, float
// the FP32 one.
template <typename T> __device__ __forceinline__ T uni_t(uint32_t w);
template <> __device__ __forceinline__ double uni_t<double>(uint32_t w) { return uni64(w); }
template <> __device__ __forceinline__ float uni_t<float>(uint32_t w) { return uni32(w); }

struct Event {
    uint32_t k0, k1, slot, step, tag, j;
    U4 b, c;
    __device__ __forceinline__ void init(uint64_t seed, uint32_t slot_, uint32_t step_, uint32_t tag_) {
        k0 = (uint32_t)seed; k1 = (uint32_t)(seed >> 32); slot = slot_; step = step_; tag = tag_; j = 0;
    }
    __device__ __forceinline__ void begin() {
        b = philox10(U4{slot, step, j, tag}, k0, k1);
        ++j;
    }
    __device__ __forceinline__ void second() { c = philox10(U4{slot, step, (j - 1) | 0x80000000u, tag}, k0, k1); }
    __device__ __forceinline__ uint32_t jev() const { return j - 1; }   // index of the current event
    template <typename T> __device__ __forceinline__ T xi() { return uni_t<T>(b.x); }
    template <typename T> __device__ __forceinline__ T phi1() { return uni_t<T>(b.z); }
    template <typename T> __device__ __forceinline__ T cos1() { return uni_t<T>(b.w); }
    template <typename T> __device__ __forceinline__ T phi2() { return uni_t<T>(c.x); }
    template <typename T> __device__ __forceinline__ T cos2() { return uni_t<T>(c.y); }
    template <typename T> __device__ __forceinline__ T s2() { return uni_t<T>(c.z); }
    template <typename T> __device__ __forceinline__ T share() { return uni_t<T>(c.w); }
    template <typename T> __device__ __forceinline__ T snew() { return uni_t<T>(b.y); }
    __device__ __forceinline__ void finish() {}
};

// Injected uniforms (mcs_set_uniform_source): the particle of slot `slot` reads its own
// caller-given values one after the other, in whatever order the collision code asks for
// them -- the reference's serial order.  Running past the range raises ST_UNIFORMS and
// reads 0.5, so the step still ends; finish() stores the position for the next step.
struct EventInj {
    const double* u;
    long long* pos_out;
    long long pos, end;
    uint32_t* status;
    uint32_t j, slot;
    bool has;   // the slot has a range
    __device__ __forceinline__ void bind(const double* u_, long long* pos_, const long long* end_, long long n,
                                         uint32_t* status_) {
        u = u_; pos_out = pos_; status = status_;
        has = (long long)slot < n;
        if (has) { pos = pos_[slot]; end = end_[slot]; }
        else { pos = 0; end = 0; }
    }
    __device__ __forceinline__ void init(uint64_t, uint32_t slot_, uint32_t, uint32_t) { slot = slot_; j = 0; }
    __device__ __forceinline__ void begin() { ++j; }
    __device__ __forceinline__ void second() {}
    __device__ __forceinline__ uint32_t jev() const { return j - 1; }
    __device__ __forceinline__ double next() {
        if (pos < end) return __ldg(u + pos++);
        atomicOr(status, ST_UNIFORMS);
        return 0.5;
    }
    template <typename T> __device__ __forceinline__ T xi() { return (T)next(); }
    template <typename T> __device__ __forceinline__ T phi1() { return (T)next(); }
    template <typename T> __device__ __forceinline__ T cos1() { return (T)next(); }
    template <typename T> __device__ __forceinline__ T phi2() { return (T)next(); }
    template <typename T> __device__ __forceinline__ T cos2() { return (T)next(); }
    template <typename T> __device__ __forceinline__ T s2() { return (T)next(); }
    template <typename T> __device__ __forceinline__ T share() { return (T)next(); }
    template <typename T> __device__ __forceinline__ T snew() { return (T)next(); }
    __device__ __forceinline__ void finish() {
        if (has) pos_out[slot] = pos;
    }
};

// rand(Poisson(lam)) from a stream: inversion below 10, PTRS (Hoermann 1993) above; the
// oracle's algorithm (only the law of the reference's Distributions.Poisson is matched).
__device__ __forceinline__ long long poisson_draw(Rng& r, double lam) {
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

// Initial electron of slot `slot`: an isotropic Maxwellian velocity whose components have
// standard deviation `sigma` (m/s) and a free-flight s = -log(u).  Five uniforms of the
// stream {slot, 0, k/4, TAG_INIT}: Box-Muller on (u0, u1) gives vx, vy and on (u2, u3) vz;
// u4 gives s.
__device__ __forceinline__ void maxwellian_draw(uint64_t seed, uint32_t slot, double sigma, double& vx, double& vy,
                                                double& vz, double& s) {
    Rng r;
    r.init(seed, slot, 0u, TAG_INIT);
    const double u0 = r.u64(), u1 = r.u64(), u2 = r.u64(), u3 = r.u64(), u4 = r.u64();
    const double r0 = sqrt(-2.0 * log(u0)), r1 = sqrt(-2.0 * log(u2));
    double s0, c0, s1, c1;
    sincos(6.283185307179586 * u1, &s0, &c0);
    sincos(6.283185307179586 * u3, &s1, &c1);
    vx = sigma * (r0 * c0);
    vy = sigma * (r0 * s0);
    vz = sigma * (r1 * c1);
    s = -log(u4);
}

template <typename T> struct Uni;
template <> struct Uni<double> { __device__ static double get(Rng& r) { return r.u64(); } };
template <> struct Uni<float> { __device__ static float get(Rng& r) { return r.u32(); } };

// ---------------------------------------------------------------------------------------
// Precision-specific math.  FP64 follows the reference's operations; FP32 uses the SFU
// approximations where the Monte Carlo tolerates their error (documented per call).
// ---------------------------------------------------------------------------------------
template <typename T> struct M;
template <> struct M<double> {
    __device__ static double nlog(double u) { return -log(u); }
    // randsphere: JuMC/src/util.jl:4-12, from the uniforms (uphi, uu)
    __device__ static void dir(double uphi, double uu, double& dx, double& dy, double& dz) {
        const double phi = 6.283185307179586 * uphi;
        double s, c;
        sincos(phi, &s, &c);
        const double u = 2.0 * uu - 1.0;
        const double v = sqrt(1.0 - u * u);
        dx = v * c; dy = v * s; dz = u;
    }
    __device__ static double sq(double x) { return sqrt(x); }
};
template <> struct M<float> {
    __device__ static float nlog(float u) { return -__logf(u); }
    __device__ static void dir(float uphi, float uu, float& dx, float& dy, float& dz) {
        // phi = 2*pi*U evaluated as (2U-1)*pi + pi so the SFU sees |arg| <= pi.
        const float ph = fmaf(uphi, 6.28318530718f, -3.14159265359f);
        float s, c;
        __sincosf(ph, &s, &c);
        const float u = fmaf(2.0f, uu, -1.0f);
        const float v = sqrtf(fmaxf(0.0f, 1.0f - u * u));
        dx = -v * c; dy = -v * s; dz = u;
    }
    __device__ static float sq(float x) { return sqrtf(x); }
};

// ---------------------------------------------------------------------------------------
// Block-wide helpers
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Ordered-append tile status word: [epoch:30][flag:2][value:32].
// flag 1 = aggregate of this tile only, flag 2 = inclusive prefix through this tile.
__device__ __forceinline__ unsigned long long tile_word(uint32_t epoch, uint32_t flag, uint32_t v) {
    return ((unsigned long long)(epoch & 0x3fffffffu) << 34) | ((unsigned long long)flag << 32) | v;
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Exclusive prefix of `count` over tiles [0, tile) by decoupled look-back (Merrill &
// Garland 2016).  Tiles are handed out in increasing order by an atomic ticket, so every
// predecessor is owned by a running CTA and the wait ends; it is still bounded, and on
// timeout ST_TIMEOUT is raised and the returned prefix is flagged invalid (ok=false).
// Called by one thread.
// `first` is the first tile of the segment being scanned (0 for a whole population; the
// first tile of an instance in a batch, so instances are prefixed independently).
// The waiting half, for a tile (not the first) whose aggregate `count` is published already:
// sums the tiles before it back to one with an inclusive prefix, then publishes its own.
__device__ __forceinline__ uint32_t tile_lookback_wait(unsigned long long* status, uint32_t first, uint32_t tile,
                                                       uint32_t epoch, uint32_t count, uint32_t* st_word, bool* ok,
                                                       uint32_t max_spins = 1u << 24) {
    *ok = true;
    uint32_t excl = 0;
    int64_t p = (int64_t)tile - 1;
    uint32_t spins = 0;
    const uint32_t ep = epoch & 0x3fffffffu;
    while (p >= (int64_t)first) {
        const unsigned long long s = ld_acquire_u64(&status[p]);
        const uint32_t e = (uint32_t)(s >> 34);
        const uint32_t f = (uint32_t)(s >> 32) & 3u;
        if (e != ep || f == 0) {
            if (++spins > max_spins) {  // the default is about a second with the backoff below
                atomicOr(st_word, ST_TIMEOUT);
                *ok = false;
                break;
            }
            if (spins > 64) __nanosleep(64);
            continue;
        }
        excl += (uint32_t)s;
        if (f == 2) break;
        --p;
    }
    st_release_u64(&status[tile], tile_word(epoch, 2, excl + count));
    return excl;
}

// Publish the tile's count and return the sum of the counts of tiles first..tile-1.
__device__ __forceinline__ uint32_t tile_lookback_from(unsigned long long* status, uint32_t first, uint32_t tile,
                                                       uint32_t epoch, uint32_t count, uint32_t* st_word, bool* ok,
                                                       uint32_t max_spins = 1u << 24) {
    *ok = true;
    if (tile == first) {
        st_release_u64(&status[tile], tile_word(epoch, 2, count));
        return 0;
    }
    st_release_u64(&status[tile], tile_word(epoch, 1, count));
    return tile_lookback_wait(status, first, tile, epoch, count, st_word, ok, max_spins);
}

__device__ __forceinline__ uint32_t tile_lookback(unsigned long long* status, uint32_t tile, uint32_t epoch,
                                                  uint32_t count, uint32_t* st_word, bool* ok) {
    return tile_lookback_from(status, 0u, tile, epoch, count, st_word, ok);
}

// The waiting half by a whole warp (all 32 lanes call it; every lane gets the prefix): each
// round reads the status words of the 32 tiles before the window at once, and the window
// ends at the nearest one with an inclusive prefix once every tile up to it has published.
// Tiles before `first` count as an inclusive prefix of 0.  Bounded like the one-thread form.
__device__ __forceinline__ uint32_t tile_lookback_wait_warp(unsigned long long* status, uint32_t first, uint32_t tile,
                                                            uint32_t epoch, uint32_t count, uint32_t* st_word,
                                                            bool* ok, uint32_t max_spins = 1u << 24) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const uint32_t ep = epoch & 0x3fffffffu;
    uint32_t excl = 0, spins = 0;
    bool good = true;
    int64_t p = (int64_t)tile - 1;
    while (p >= (int64_t)first) {
        const int64_t q = p - lane;
        const bool in = q >= (int64_t)first;
        const unsigned long long s = in ? ld_acquire_u64(&status[q]) : 0ull;
        const uint32_t e = (uint32_t)(s >> 34), f = (uint32_t)(s >> 32) & 3u;
        const unsigned incm = __ballot_sync(FULL, !in || (e == ep && f == 2));
        const unsigned readym = __ballot_sync(FULL, !in || (e == ep && f != 0));
        const unsigned need = incm ? (FULL >> (31 - (__ffs(incm) - 1))) : FULL;   // lanes up to the inclusive one
        if ((readym & need) != need) {
            if (++spins > max_spins) {  // about a second with the backoff below
                if (lane == 0) atomicOr(st_word, ST_TIMEOUT);
                good = false;
                break;
            }
            if (spins > 64) __nanosleep(64);
            continue;
        }
        uint32_t v = (in && ((need >> lane) & 1u)) ? (uint32_t)s : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
        excl += v;
        if (incm) break;
        p -= 32;
    }
    *ok = good;
    if (lane == 0) st_release_u64(&status[tile], tile_word(epoch, 2, excl + count));
    return excl;
}

// Publish the tile's count and return the prefix of tiles first..tile-1, by a whole warp.
__device__ __forceinline__ uint32_t tile_lookback_from_warp(unsigned long long* status, uint32_t first, uint32_t tile,
                                                            uint32_t epoch, uint32_t count, uint32_t* st_word,
                                                            bool* ok) {
    const int lane = threadIdx.x & 31;
    if (tile == first) {
        if (lane == 0) st_release_u64(&status[tile], tile_word(epoch, 2, count));
        *ok = true;
        return 0;
    }
    if (lane == 0) st_release_u64(&status[tile], tile_word(epoch, 1, count));
    __syncwarp();
    return tile_lookback_wait_warp(status, first, tile, epoch, count, st_word, ok);
}

}  // namespace mcs
