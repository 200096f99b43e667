// step.cuh -- the electron step (advance!, JuMC/src/mixed_population.jl:24-54) as one
// persistent, tiled sm_100a kernel per field model:
//
//   * each CTA takes tiles of BLOCK*PPT consecutive slots from an atomic ticket;
//   * every active particle is pushed, collided and tracked with its state in registers;
//     each collision event draws from its own Philox block (seed; slot, step, event, tag);
//   * secondaries are staged in a per-CTA global buffer, ranked by (parent slot, event #)
//     with a block scan of per-parent counts, and appended after the tiles before them
//     (decoupled look-back on per-tile counts), so the population order equals the
//     serial reference order (ascending parent index);
//   * per-tile partial moments are reduced by the last CTA in tile order (deterministic).
//
// Included by step_f32.cu (FMA contraction on) and step_f64.cu (-fmad=false, so the FP64
// operation sequence matches the reference's unfused arithmetic).
#pragma once
#include "mcs_device.cuh"
#include "mcs_internal.h"

namespace mcs {

constexpr uint32_t FLAG_CLAMP = MCS_FLAG_CLAMP_ENERGY;

// ---------------------------------------------------------------------------------------
// Shared-memory copy of the per-row process description.
// ---------------------------------------------------------------------------------------
template <typename T>
struct RowsSmem {
    int kind[kMaxRows];
    T par[kMaxRows];   // FP64: threshold (J) or mass ratio.  FP32: 2*th/m (v^2 units) or m/(M+m)
};

template <typename T>
__device__ __forceinline__ void load_rows(RowsSmem<T>& r, const TableView& t) {
    for (int j = threadIdx.x; j < kMaxRows; j += blockDim.x) {
        const int kd = j < t.nrows ? t.kind[j] : K_NULL;
        r.kind[j] = kd;
        double p = j < t.nrows ? t.param[j] : 0.0;
        if (sizeof(T) == 4) {
            if (kd == K_ELASTIC) p = p / (1.0 + p);
            else p = 2.0 * p / kElectronMass;
        }
        r.par[j] = (T)p;
    }
}

// ---------------------------------------------------------------------------------------
// Table lookup + process selection: do_one_collision!, JuMC/src/collisions.jl:159-192
// (indweight util.jl:23-30, rate collisions.jl:35-39).  Returns the row or -1.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ int select_row64(const TableView& t, double eng, double xi, uint32_t flags,
                                            uint32_t* status) {
    const double x = eng - t.e0;
    double fk = floor(x / t.step);                 // Julia fld: exact floor of the quotient
    if (__fma_rn(fk, t.step, -x) > 0.0) fk -= 1.0;
    long long k;
    double w;
    if (!(fk >= 0.0 && fk <= (double)(t.neps - 2))) {
        const bool low = !(fk >= 0.0) && eng < t.e0;
        k = low ? 0 : t.neps - 2;
        w = low ? 1.0 : 0.0;
        if (!(flags & FLAG_CLAMP)) atomicOr(status, ST_ENERGY);
    } else {
        k = (long long)fk;
        const double tt = (double)(k + 1) / (double)(t.neps - 1);  // LinRange lerpi
        const double ek1 = (1.0 - tt) * t.e0 + tt * t.emax;
        w = (ek1 - eng) / t.step;
    }
    const double* c0 = t.rate64 + k * t.nrows;
    const double* c1 = c0 + t.nrows;
    for (int j = 0; j < t.nrows; ++j) {
        const double nu = w * __ldg(c0 + j) + (1.0 - w) * __ldg(c1 + j);
        if (nu > xi) return j;
        xi -= nu;
    }
    return -1;
}

// FP32 selection, u = v^2 * (m/2/step) - e0/step being the position on the energy grid, in
// two halves so that the first rows' loads are in flight while the caller draws xi:
// select32_begin places the energy on the grid and loads the first quad of both columns
// (the total real rate and rows 0-2); select32_finish tests xi against the interpolated
// total first -- most events are null collisions and end there -- and otherwise scans the
// rows against xi.  The FP32 mode is statistically, not bitwise, the reference's: the total
// test and the scan can disagree only within a rounding of the total.
struct Sel32 {
    int k;
    float w;
    bool bad;
    float4 a, b;
};

__device__ __forceinline__ void select32_begin(const TableView& t, float v2, Sel32& s) {
    const float u = fmaf(v2, t.ke32, -t.e0n32);
    const int k = (int)u;
    const bool low = !(u >= 0.0f);
    s.bad = low || k > t.neps - 2;
    s.k = s.bad ? (low ? 0 : t.neps - 2) : k;
    s.w = s.bad ? (low ? 1.0f : 0.0f) : (float)(k + 1) - u;
    s.a = __ldg(reinterpret_cast<const float4*>(t.rate32 + (size_t)s.k * t.nrp));
    s.b = __ldg(reinterpret_cast<const float4*>(t.rate32 + (size_t)(s.k + 1) * t.nrp));
}

__device__ __forceinline__ int select32_finish(const TableView& t, const Sel32& s, float xi, uint32_t flags,
                                               uint32_t* status) {
    if (s.bad && !(flags & FLAG_CLAMP)) atomicOr(status, ST_ENERGY);
    const float w = s.w;
    float4 a = s.a, b = s.b;
    if (!(xi < fmaf(w, a.x - b.x, b.x))) return -1;   // beyond the total real rate: null
    // row r sits at element r + 1 of the quads
    float nu = fmaf(w, a.y - b.y, b.y);
    if (nu > xi) return 0;
    xi -= nu;
    nu = fmaf(w, a.z - b.z, b.z);
    if (nu > xi) return 1 < t.nrows ? 1 : -1;
    xi -= nu;
    nu = fmaf(w, a.w - b.w, b.w);
    if (nu > xi) return 2 < t.nrows ? 2 : -1;
    xi -= nu;
    const int nq = t.nrp >> 2;
    for (int q = 1; q < nq; ++q) {
        a = __ldg(reinterpret_cast<const float4*>(t.rate32 + (size_t)s.k * t.nrp) + q);
        b = __ldg(reinterpret_cast<const float4*>(t.rate32 + (size_t)(s.k + 1) * t.nrp) + q);
        const int j = (q << 2) - 1;
        nu = fmaf(w, a.x - b.x, b.x);
        if (nu > xi) return j < t.nrows ? j : -1;
        xi -= nu;
        nu = fmaf(w, a.y - b.y, b.y);
        if (nu > xi) return j + 1 < t.nrows ? j + 1 : -1;
        xi -= nu;
        nu = fmaf(w, a.z - b.z, b.z);
        if (nu > xi) return j + 2 < t.nrows ? j + 2 : -1;
        xi -= nu;
        nu = fmaf(w, a.w - b.w, b.w);
        if (nu > xi) return j + 3 < t.nrows ? j + 3 : -1;
        xi -= nu;
    }
    return -1;
}

// Outcome of a collision: nothing (null), new particle, removal, velocity change.
// collide64/collide32 report OUT_NONE for the velocity-changing kinds; collide_once
// turns that into OUT_CHANGE.
enum { OUT_NONE = 0, OUT_NEW = 1, OUT_REMOVE = 2, OUT_CHANGE = 3, OUT_PHOTO = 4 };

template <typename T>
struct Sec { T vx, vy, vz, s; };

// collide: JuMC/src/electron.jl:108-139.  FP64 follows the reference's expressions.  The
// draws are read in the reference's order (the event's accessors, mcs_device.cuh): a
// direction is phi then u (randsphere, util.jl:4-12); ionization draws the primary's
// direction, the secondary's and then the secondary's free flight (electron.jl:121-125); the
// uniform-sharing ionization draws its sharing fraction first.
template <class Ev>
__device__ __forceinline__ int collide64(int kind, double par, double eng, Ev& e, double& vx, double& vy,
                                         double& vz, Sec<double>& sec) {
    const double m = kElectronMass;
    if (kind == K_ELASTIC) {
        const double f = par / (1.0 + par);
        const double cx = f * vx, cy = f * vy, cz = f * vz;
        const double dx = vx - cx, dy = vy - cy, dz = vz - cz;
        const double nrm = sqrt(dx * dx + dy * dy + dz * dz);
        double ux, uy, uz;
        const double a = e.template phi1<double>(), b = e.template cos1<double>();
        M<double>::dir(a, b, ux, uy, uz);
        vx = ux * nrm + cx; vy = uy * nrm + cy; vz = uz * nrm + cz;
        return OUT_NONE;
    }
    if (kind == K_EXCITATION) {
        const double E1 = fmax(0.0, eng - par);
        const double va = sqrt(2.0 * E1 / m);
        double ux, uy, uz;
        const double a = e.template phi1<double>(), b = e.template cos1<double>();
        M<double>::dir(a, b, ux, uy, uz);
        vx = ux * va; vy = uy * va; vz = uz * va;
        return OUT_NONE;
    }
    if (kind == K_IONIZATION || kind == K_IONIZATION_UNIFORM) {
        e.second();
        double va1, va2;
        if (kind == K_IONIZATION) {
            const double E1 = fmax(0.0, eng - par) / 2.0;
            va1 = va2 = sqrt(2.0 * E1 / m);
        } else {
            const double Ea = fmax(0.0, eng - par);
            const double E2 = e.template share<double>() * Ea;
            const double E1 = Ea - E2;
            va1 = sqrt(2.0 * E1 / m);
            va2 = sqrt(2.0 * E2 / m);
        }
        double ux, uy, uz, wx, wy, wz;
        const double a1 = e.template phi1<double>(), b1 = e.template cos1<double>();
        M<double>::dir(a1, b1, ux, uy, uz);
        const double a2 = e.template phi2<double>(), b2 = e.template cos2<double>();
        M<double>::dir(a2, b2, wx, wy, wz);
        sec.vx = wx * va2; sec.vy = wy * va2; sec.vz = wz * va2;
        sec.s = -log(e.template s2<double>());
        vx = ux * va1; vy = uy * va1; vz = uz * va1;
        return OUT_NEW;
    }
    if (kind == K_ATTACHMENT) return OUT_REMOVE;
    if (kind == K_PHOTOEMISSION) return OUT_PHOTO;   // the electron is unchanged
    return OUT_NONE;
}

// FP32: energies in v^2 units (par = 2*threshold/m), the same draws as collide64.
template <class Ev>
__device__ __forceinline__ int collide32(int kind, float par, float v2, Ev& e, float& vx, float& vy, float& vz,
                                         Sec<float>& sec) {
    if (kind == K_ELASTIC) {
        const float cx = par * vx, cy = par * vy, cz = par * vz;
        const float dx = vx - cx, dy = vy - cy, dz = vz - cz;
        const float nrm = sqrtf(fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
        float ux, uy, uz;
        const float a = e.template phi1<float>(), b = e.template cos1<float>();
        M<float>::dir(a, b, ux, uy, uz);
        vx = fmaf(ux, nrm, cx); vy = fmaf(uy, nrm, cy); vz = fmaf(uz, nrm, cz);
        return OUT_NONE;
    }
    if (kind == K_EXCITATION) {
        const float va = sqrtf(fmaxf(0.0f, v2 - par));
        float ux, uy, uz;
        const float a = e.template phi1<float>(), b = e.template cos1<float>();
        M<float>::dir(a, b, ux, uy, uz);
        vx = ux * va; vy = uy * va; vz = uz * va;
        return OUT_NONE;
    }
    if (kind == K_IONIZATION || kind == K_IONIZATION_UNIFORM) {
        e.second();
        float va1, va2;
        const float ea = fmaxf(0.0f, v2 - par);
        if (kind == K_IONIZATION) {
            va1 = va2 = sqrtf(0.5f * ea);
        } else {
            const float f2 = e.template share<float>();
            va1 = sqrtf(ea - f2 * ea);
            va2 = sqrtf(f2 * ea);
        }
        float ux, uy, uz, wx, wy, wz;
        const float a1 = e.template phi1<float>(), b1 = e.template cos1<float>();
        M<float>::dir(a1, b1, ux, uy, uz);
        const float a2 = e.template phi2<float>(), b2 = e.template cos2<float>();
        M<float>::dir(a2, b2, wx, wy, wz);
        sec.vx = wx * va2; sec.vy = wy * va2; sec.vz = wz * va2;
        sec.s = M<float>::nlog(e.template s2<float>());
        vx = ux * va1; vy = uy * va1; vz = uz * va1;
        return OUT_NEW;
    }
    if (kind == K_ATTACHMENT) return OUT_REMOVE;
    if (kind == K_PHOTOEMISSION) return OUT_PHOTO;
    return OUT_NONE;
}

// ---------------------------------------------------------------------------------------
// Deposits.  Int64 fixed point at 2^-32 elementary charges; the arithmetic is the oracle's
// (seven rounded corners, the eighth takes the remainder: node sum == llrint(q*2^32)).
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void cic_fixed(long long* q, int nx, int ny, int ix, int iy, int iz, double fx,
                                          double fy, double fz, double charge, uint32_t* status) {
    if (!(fabs(charge) < kMaxDepositCharge)) {   // also NaN
        atomicOr(status, ST_CHARGE);
        return;
    }
    const long long W = __double2ll_rn(charge * 0x1p32);
    const double Wd = (double)W;
    const double gx[2] = {1.0 - fx, fx}, gy[2] = {1.0 - fy, fy}, gz[2] = {1.0 - fz, fz};
    const long long sy = nx + 1, sz = (long long)(nx + 1) * (ny + 1);
    long long* b = q + ix + iy * sy + iz * sz;
    long long acc = 0;
#pragma unroll
    for (int c = 0; c < 7; ++c) {
        const int a0 = c & 1, a1 = (c >> 1) & 1, a2 = (c >> 2) & 1;
        const double wc = __dmul_rn(__dmul_rn(gx[a0], gy[a1]), gz[a2]);
        const long long qb = __double2ll_rn(__dmul_rn(Wd, wc));
        acc += qb;
        if (qb) atomicAdd(reinterpret_cast<unsigned long long*>(b + a0 + a1 * sy + a2 * sz),
                          (unsigned long long)qb);
    }
    const long long last = W - acc;
    if (last) atomicAdd(reinterpret_cast<unsigned long long*>(b + 1 + sy + sz), (unsigned long long)last);
}

// The same CIC deposit for one particle per lane (all 32 lanes call it; `valid` lanes
// deposit).  Lanes of a run of equal `cell` (adjacent in the warp, as cell-sorted particles
// are) add their eight corner values with a segmented shuffle sum and the first lane of the
// run issues the eight atomics, so a warp inside one cell makes 8 atomics instead of 256.
// Integer sums: the node totals are bit-identical to per-particle atomics.
__device__ __forceinline__ void cic_fixed_warp(long long* q, int nx, int ny, bool valid, uint32_t cell, int ix, int iy,
                                               int iz, double fx, double fy, double fz, double charge,
                                               uint32_t* status) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    if (valid && !(fabs(charge) < kMaxDepositCharge)) {
        atomicOr(status, ST_CHARGE);
        valid = false;
    }
    long long v[8];
    if (valid) {
        const long long W = __double2ll_rn(charge * 0x1p32);
        const double Wd = (double)W;
        const double gx[2] = {1.0 - fx, fx}, gy[2] = {1.0 - fy, fy}, gz[2] = {1.0 - fz, fz};
        long long acc = 0;
#pragma unroll
        for (int c = 0; c < 7; ++c) {
            const int a0 = c & 1, a1 = (c >> 1) & 1, a2 = (c >> 2) & 1;
            const double wc = __dmul_rn(__dmul_rn(gx[a0], gy[a1]), gz[a2]);
            v[c] = __double2ll_rn(__dmul_rn(Wd, wc));
            acc += v[c];
        }
        v[7] = W - acc;
    } else {
#pragma unroll
        for (int c = 0; c < 8; ++c) v[c] = 0;
    }
    const uint32_t key = valid ? cell : 0xffffffffu;
    const uint32_t nkey = __shfl_down_sync(FULL, key, 1);
    const unsigned same = __ballot_sync(FULL, valid && lane < 31 && nkey == key);
    const unsigned stops = ~same & (0xffffffffu << lane);      // lanes >= me that end a run
    const int end = __ffs(stops) - 1;
    const bool leader = valid && (lane == 0 || !((same >> (lane - 1)) & 1u));
    const long long sy = nx + 1, sz = (long long)(nx + 1) * (ny + 1);
    long long* b = q + ix + iy * sy + iz * sz;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        long long x = v[c];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long t = __shfl_down_sync(FULL, x, o);
            if (lane + o <= end) x += t;
        }
        if (leader && x) {
            const int a0 = c & 1, a1 = (c >> 1) & 1, a2 = (c >> 2) & 1;
            atomicAdd(reinterpret_cast<unsigned long long*>(b + a0 + a1 * sy + a2 * sz), (unsigned long long)x);
        }
    }
}

// Cell location on the 3-D mesh of an absolute position (checkbounds semantics: [0, n)).
__device__ __forceinline__ bool cart_locate(const GridView& g, double x, double y, double z, int& ix, int& iy,
                                            int& iz, double& fx, double& fy, double& fz) {
    const double ux = (x - g.x0) / g.h, uy = (y - g.y0) / g.h, uz = (z - g.z0) / g.h;
    const double flx = floor(ux), fly = floor(uy), flz = floor(uz);
    if (!(flx >= 0.0 && flx < (double)g.nx && fly >= 0.0 && fly < (double)g.ny && flz >= 0.0 &&
          flz < (double)g.nz))
        return false;
    ix = (int)flx; iy = (int)fly; iz = (int)flz;
    fx = ux - flx; fy = uy - fly; fz = uz - flz;
    return true;
}

// Cylindrical NGP cell (cellindex, MCStreamer/src/grid.jl:84-90); deposits only where
// density!/track1 do (1 <= i <= M, 0 <= j <= N+1).  Stored as int64 weight sums;
// density = q * 2^-32 / dV(i) on read.
__device__ __forceinline__ void cyl_track(const GridView& g, long long* q, double x, double y, double z,
                                          double charge, uint32_t* status) {
    if (!(fabs(charge) < kMaxDepositCharge)) {
        atomicOr(status, ST_CHARGE);
        return;
    }
    const double rho = sqrt(x * x + y * y);
    double fi = floor(rho / g.dr);
    if (__fma_rn(fi, g.dr, -rho) > 0.0) fi -= 1.0;
    double fj = floor(z / g.dz);
    if (__fma_rn(fj, g.dz, -z) > 0.0) fj -= 1.0;
    fi += 1.0; fj += 1.0;
    if (!(fi >= 1.0 && fi <= (double)g.M && fj >= 0.0 && fj <= (double)g.N + 1.0)) return;
    const long long idx = (long long)fi + (long long)fj * (g.M + 2);
    const long long W = __double2ll_rn(charge * 0x1p32);
    atomicAdd(reinterpret_cast<unsigned long long*>(q + idx), (unsigned long long)W);
}

// CollisionTracker at an absolute position (gridfields.jl:203-224).
__device__ __forceinline__ void track_abs(const GridView& g, double x, double y, double z, double charge,
                                          uint32_t* status) {
    if (g.type == GRID_CART3D) {
        int ix, iy, iz;
        double fx, fy, fz;
        if (cart_locate(g, x, y, z, ix, iy, iz, fx, fy, fz))
            cic_fixed(g.qfixed, g.nx, g.ny, ix, iy, iz, fx, fy, fz, charge, status);
    } else if (g.type == GRID_CYL) {
        cyl_track(g, g.qfixed, x, y, z, charge, status);
    }
}

// ---------------------------------------------------------------------------------------
// Secondary staging: each CTA owns a slice of a global buffer (L2-resident while the tile
// runs).  An entry carries its (tile-local parent index, event #) key; the final slot is
// n_entry + (secondaries of earlier tiles) + (secondaries of earlier parents in the tile)
// + event #, i.e. ascending parent slot then event order, the serial reference order.
// ---------------------------------------------------------------------------------------
template <typename T>
struct Stage {
    T* f[8];
    uint32_t* cell;
    uint32_t* key;   // (local << 16) | event
    uint8_t* act;
    uint32_t cap;
    __device__ __forceinline__ void init(const StepCtl& C) {
        char* b = C.stage + (unsigned long long)blockIdx.x * C.stage_stride;
        cap = C.stage_cap;
#pragma unroll
        for (int q = 0; q < 8; ++q) f[q] = reinterpret_cast<T*>(b + (size_t)q * cap * sizeof(T));
        cell = reinterpret_cast<uint32_t*>(b + (size_t)8 * cap * sizeof(T));
        key = cell + cap;
        act = reinterpret_cast<uint8_t*>(key + cap);
    }
};

template <typename T>
__device__ __forceinline__ void stage(const Stage<T>& sg, uint32_t* count, uint32_t local, uint32_t ev,
                                      const T (&v)[8], uint32_t cell, uint8_t act, uint32_t* status) {
    const uint32_t pos = atomicAdd(count, 1u);
    if (pos < sg.cap && ev < 65536u) {
#pragma unroll
        for (int q = 0; q < 8; ++q) sg.f[q][pos] = v[q];
        sg.cell[pos] = cell;
        sg.key[pos] = (local << 16) | ev;
        sg.act[pos] = act;
    } else {
        atomicOr(status, ST_OVERFLOW);
    }
}

// Field models for the literal Yoshida push on absolute positions.
struct FieldUniform {
    double ex, ey, ez;
    template <typename T>
    __device__ __forceinline__ void operator()(const GridView&, T, T, T, T& e0, T& e1, T& e2, uint32_t*) const {
        e0 = (T)ex; e1 = (T)ey; e2 = (T)ez;
    }
};

// Cylindrical FieldInterp, MCStreamer/src/gridfields.jl:115-190 (FP64 face fields).
struct FieldCyl {
    template <typename T>
    __device__ __forceinline__ void operator()(const GridView& g, T x0, T x1, T x2, T& e0, T& e1, T& e2,
                                               uint32_t* status) const {
        if constexpr (sizeof(T) == 4) {
            gather32(g, x0, x1, x2, e0, e1, e2, status);
            return;
        }
        const double x = x0, y = x1, z = x2;
        e0 = e1 = e2 = (T)0;
        const double r0 = sqrt(x * x + y * y);
        if (!((0.0 < r0 && r0 < g.R) && (0.0 < z && z < g.L))) return;
        double r = r0;
        if (r == 0.0) r = g.drc / 10.0;
        const double qr = r / g.drc;              // normdivrem(r - first(rf), dr(grid))
        long long i = (long long)trunc(qr);
        const double dr_ = qr - (double)i;
        const double qz = z / g.dzc;
        long long j = (long long)trunc(qz);
        const double dz_ = qz - (double)j;
        long long i1, j1;
        double dr1, dz1;
        if (dr_ < 0.5) { i1 = i; dr1 = dr_ + 0.5; } else { i1 = i + 1; dr1 = dr_ - 0.5; }
        if (dz_ < 0.5) { j1 = j; dz1 = dz_ + 0.5; } else { j1 = j + 1; dz1 = dz_ - 0.5; }
        i += 1; j += 1;
        const long long ld = g.M + 3;
        const double* er = g.er;
        const double* ez = g.ez;
        const double er1 = __ldg(er + i + j1 * ld) * (1 - dr_) * (1 - dz1) + __ldg(er + i + 1 + j1 * ld) * dr_ * (1 - dz1) +
                           __ldg(er + i + (j1 + 1) * ld) * (1 - dr_) * dz1 + __ldg(er + i + 1 + (j1 + 1) * ld) * dr_ * dz1;
        const double ez1 = __ldg(ez + i1 + j * ld) * (1 - dr1) * (1 - dz_) + __ldg(ez + i1 + 1 + j * ld) * dr1 * (1 - dz_) +
                           __ldg(ez + i1 + (j + 1) * ld) * (1 - dr1) * dz_ + __ldg(ez + i1 + 1 + (j + 1) * ld) * dr1 * dz_;
        const double a = er1 * x / r, b = er1 * y / r;
        if (sqrt(a * a + b * b + ez1 * ez1) > 1e8) atomicOr(status, ST_FIELD);
        e0 = (T)a; e1 = (T)b; e2 = (T)ez1;
    }

    // The FP32 push's gather: the same cells and weights in single precision from the FP32
    // face copies, reciprocal cell sizes (of step(grid.rc), step(grid.zc)), and
    // |E|^2 > 1e16 for the field check.  Indices stay inside the (M+3) x (N+3) faces: a
    // rounded-up r / dr or z / dz of M or N reads face M+2 or N+2 at most.
    __device__ __forceinline__ void gather32(const GridView& g, float x, float y, float z, float& e0, float& e1,
                                             float& e2, uint32_t* status) const {
        e0 = e1 = e2 = 0.0f;
        const float r = sqrtf(fmaf(x, x, y * y));
        if (!((0.0f < r && r < g.R32) && (0.0f < z && z < g.L32))) return;
        const float qr = r * g.inv_dr32, qz = z * g.inv_dz32;
        int i = min((int)qr, g.M), j = min((int)qz, g.N);
        const float dr_ = qr - (float)i, dz_ = qz - (float)j;
        int i1, j1;
        float dr1, dz1;
        if (dr_ < 0.5f) { i1 = i; dr1 = dr_ + 0.5f; } else { i1 = i + 1; dr1 = dr_ - 0.5f; }
        if (dz_ < 0.5f) { j1 = j; dz1 = dz_ + 0.5f; } else { j1 = j + 1; dz1 = dz_ - 0.5f; }
        i += 1; j += 1;
        const int ld = g.M + 3;
        const float* er = g.er32;
        const float* ez = g.ez32;
        const float a0 = __ldg(er + i + j1 * ld), a1 = __ldg(er + i + 1 + j1 * ld);
        const float a2 = __ldg(er + i + (j1 + 1) * ld), a3 = __ldg(er + i + 1 + (j1 + 1) * ld);
        const float b0 = __ldg(ez + i1 + j * ld), b1 = __ldg(ez + i1 + 1 + j * ld);
        const float b2 = __ldg(ez + i1 + (j + 1) * ld), b3 = __ldg(ez + i1 + 1 + (j + 1) * ld);
        const float er1 = fmaf(dz1, fmaf(dr_, a3 - a2, a2) - fmaf(dr_, a1 - a0, a0), fmaf(dr_, a1 - a0, a0));
        const float ez1 = fmaf(dz_, fmaf(dr1, b3 - b2, b2) - fmaf(dr1, b1 - b0, b0), fmaf(dr1, b1 - b0, b0));
        const float f = er1 / r;
        const float a = f * x, b = f * y;
        if (fmaf(a, a, fmaf(b, b, ez1 * ez1)) > 1e16f) atomicOr(status, ST_FIELD);
        e0 = a; e1 = b; e2 = ez1;
    }
};

// Trilinear node-field gather at an absolute position (3-D mesh, zero outside).
struct FieldCartAbs {
    template <typename T>
    __device__ __forceinline__ void operator()(const GridView& g, T x0, T x1, T x2, T& e0, T& e1, T& e2,
                                               uint32_t*) const {
        e0 = e1 = e2 = (T)0;
        const double u[3] = {((double)x0 - g.x0) / g.h, ((double)x1 - g.y0) / g.h, ((double)x2 - g.z0) / g.h};
        const int nc[3] = {g.nx, g.ny, g.nz};
        long long ic[3];
        double fr[3];
        for (int d = 0; d < 3; ++d) {
            if (!(u[d] > 0.0 && u[d] < (double)nc[d])) return;
            double fl = floor(u[d]);
            if (fl > nc[d] - 1) fl = nc[d] - 1;
            ic[d] = (long long)fl;
            fr[d] = u[d] - fl;
        }
        const long long sy = g.nx + 1, sz = (long long)(g.nx + 1) * (g.ny + 1);
        const long long base = ic[0] + ic[1] * sy + ic[2] * sz;
        double acc[3] = {0, 0, 0};
        for (int b = 0; b < 8; ++b) {
            const int a0 = b & 1, a1 = (b >> 1) & 1, a2 = (b >> 2) & 1;
            const double wgt = (a0 ? fr[0] : 1.0 - fr[0]) * (a1 ? fr[1] : 1.0 - fr[1]) * (a2 ? fr[2] : 1.0 - fr[2]);
            const long long nd = base + a0 + a1 * sy + a2 * sz;
            for (int c = 0; c < 3; ++c) {
                const double ev = g.e64 ? __ldg(g.e64 + 3 * nd + c) : (double)__ldg(g.e32 + 4 * nd + c);
                acc[c] += wgt * ev;
            }
        }
        e0 = (T)acc[0]; e1 = (T)acc[1]; e2 = (T)acc[2];
    }
};

}  // namespace mcs
