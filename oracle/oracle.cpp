/*
 * oracle.cpp -- CPU FP64 restatement of JuMC's electron step.  TEST INFRASTRUCTURE ONLY.
 *
 * Loaded (via ctypes) only by tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / --impl reference arm, and only as the checker or the CPU baseline.
 * Parity against the Julia reference is UNPINNED (no reference tests or fixtures
 * exist and Julia is not installed); see oracle.h for what is pinned.
 *
 * Every function cites the reference file:line it restates (paths inside the
 * aluque/mcstreamer project).  Random numbers come from a counter-based
 * Philox4x32-10 stream (Salmon, Moraes, Dror, Shaw, SC'11) instead of Julia's
 * task-local Xoshiro, so that the CUDA kernels can be fed identical uniforms.  A Philox
 * word w maps to the uniform (w + 0.5) * 2^-32.  Collision event j of particle `slot`
 * during step `step` draws from Philox(key=seed, ctr={slot, step, j, tag}) (xi, new s,
 * direction) and, when needed, ctr={slot, step, j | 2^31, tag} (secondary); other
 * per-particle or per-cell streams take word k from ctr={id, call, k/4, tag}.
 */
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <functional>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

/* internal status flags, mapped to the public codes by status_code() */
enum { F_CAP = 1, F_ENERGY = 2, F_FIELD = 4, F_UNSUPPORTED = 8, F_UNIFORMS = 16 };
inline int status_code(int f) {
    if (f & F_UNIFORMS) return 11;
    if (f & F_CAP) return 3;
    if (f & F_ENERGY) return 4;
    if (f & F_FIELD) return 5;
    if (f & F_UNSUPPORTED) return 7;
    return 0;
}

/* ---------------- constants: JuMC/src/constants.jl:50-54 ---------------- */
const double ELEMENTARY_CHARGE = 1.6021766208e-19;
const double ELECTRON_MASS = 9.10938356e-31;
const double SPEED_OF_LIGHT = 299792458.0;   /* co.c (Constants/src/Constants.jl:39) */

/* Yoshida-4 coefficients: JuMC/src/electron.jl:38-46 */
struct Yoshida {
    double w0, w1, c1, c2, c3, c4, d1, d2, d3;
    Yoshida() {
        const double cb = std::pow(2.0, 1.0 / 3.0);
        w0 = -cb / (2.0 - cb);
        w1 = 1.0 / (2.0 - cb);
        c1 = w1 / 2.0;
        c2 = (w0 + w1) / 2.0;
        c3 = c2;
        c4 = c1;
        d1 = w1;
        d2 = w0;
        d3 = d1;
    }
};
const Yoshida YO;

/* ---------------- Philox4x32-10 ---------------- */
inline void philox_round(uint32_t c[4], const uint32_t k[2]) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t n0 = hi1 ^ c[1] ^ k[0];
    const uint32_t n2 = hi0 ^ c[3] ^ k[1];
    c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
}

inline void philox10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    uint32_t k[2] = {key[0], key[1]};
    for (int r = 0; r < 10; ++r) {
        if (r > 0) { k[0] += 0x9E3779B9u; k[1] += 0xBB67AE85u; }
        philox_round(c, k);
    }
    out[0] = c[0]; out[1] = c[1]; out[2] = c[2]; out[3] = c[3];
}

inline double word_to_uniform(uint32_t w) { return ((double)w + 0.5) * 0x1p-32; }

/* One particle's (or cell's) uniform stream for one call. */
struct Stream {
    uint32_t key[2];
    uint32_t c0, c1, tag, k;
    uint32_t buf[4];
    Stream(uint64_t seed, uint32_t c0_, uint32_t c1_, uint32_t tag_)
        : c0(c0_), c1(c1_), tag(tag_), k(0) {
        key[0] = (uint32_t)seed; key[1] = (uint32_t)(seed >> 32);
    }
    double next() {  /* Julia rand(): util.jl:5,8,17; collisions.jl:166 */
        if ((k & 3u) == 0) {
            const uint32_t ctr[4] = {c0, c1, k >> 2, tag};
            philox10(ctr, key, buf);
        }
        return word_to_uniform(buf[(k++) & 3u]);
    }
};

/* The draws of one collision event (do_one_collision! + the new free-flight time).
 * Event j of particle `slot` during step `step` owns Philox block
 *   B = Philox(seed; {slot, step, j, tag})            -> xi, new s, direction (phi, u)
 * and, only when the process needs more draws,
 *   C = Philox(seed; {slot, step, j | 2^31, tag})      -> secondary direction, secondary s,
 *                                                         energy-sharing fraction
 * so every colliding particle generates exactly one block per event. */
/* Injected uniforms: slot i reads u[pos[i]] .. u[end[i] - 1] in the order its draws are made
 * (the reference's serial rand() order); see orc_advance_injected. */
struct Injected {
    const double* u;
    int64_t* pos;
    const int64_t* end;
    int64_t nslots;
};

struct Event {
    uint32_t key[2];
    uint32_t c0, c1, tag, j;
    uint32_t b[4], c[4];
    bool have_c;
    const Injected* inj = nullptr;   /* non-null: sequential injected values instead of Philox */
    int64_t pos = 0, end = 0;
    int* status = nullptr;
    Event(uint64_t seed, uint32_t slot, uint32_t step, uint32_t tag_) : c0(slot), c1(step), tag(tag_), j(0) {
        key[0] = (uint32_t)seed; key[1] = (uint32_t)(seed >> 32);
        have_c = false;
    }
    void inject(const Injected* in, int64_t slot, int* st) {
        inj = in;
        status = st;
        if (in && slot < in->nslots) { pos = in->pos[slot]; end = in->end[slot]; }
    }
    void finish(int64_t slot) {
        if (inj && slot < inj->nslots) inj->pos[slot] = pos;
    }
    void begin() {
        ++j;
        if (inj) return;
        const uint32_t ctr[4] = {c0, c1, j - 1, tag};
        philox10(ctr, key, b);
        have_c = false;
    }
    double u(int idx) {  /* Julia rand() draws of this event */
        if (inj) {
            if (pos < end) return inj->u[pos++];
            *status |= F_UNIFORMS;
            return 0.5;
        }
        if (idx < 4) return word_to_uniform(b[idx]);
        if (!have_c) {
            const uint32_t ctr[4] = {c0, c1, (j - 1) | 0x80000000u, tag};
            philox10(ctr, key, c);
            have_c = true;
        }
        return word_to_uniform(c[idx - 4]);
    }
};
enum { U_XI = 0, U_S = 1, U_PHI = 2, U_COS = 3, U_PHI2 = 4, U_COS2 = 5, U_S2 = 6, U_SHARE = 7 };

/* ---------------- util.jl ---------------- */
/* randsphere: JuMC/src/util.jl:4-12, from the uniforms (uphi, uu) */
inline void randsphere(double uphi, double uu, double out[3]) {
    const double phi = 6.283185307179586 * uphi;
    const double sphi = std::sin(phi), cphi = std::cos(phi);
    const double u = 2.0 * uu - 1.0;
    const double v = std::sqrt(1.0 - u * u);
    out[0] = v * cphi; out[1] = v * sphi; out[2] = u;
}

/* nextcoll: JuMC/src/util.jl:17 */
inline double nextcoll(double u) { return -std::log(u); }

/* Julia fld(x, y) for floats: round((x - mod(x, y)) / y), mod via exact fmod. */
inline double julia_fld(double x, double y) {
    double m = std::fmod(x, y);
    if (m != 0.0 && ((y < 0.0) != (m < 0.0))) m += y;
    return std::nearbyint((x - m) / y);
}

/* Base range.jl lerpi(j, d, a, b) = (1 - j/d) a + (j/d) b: LinRange getindex r[j+1]. */
inline double lerpi(int64_t j, int64_t d, double a, double b) {
    const double t = (double)j / (double)d;
    return (1.0 - t) * a + t * b;
}

/* Grid's cell-centre range of one axis (MCStreamer/src/grid.jl:33-41): faces
 * f = LinRange(0, len, m + 1), c = 0.5 * (f[2:end] + f[1:end-1]) = LinRange(0.5 (f[2] + f[1]),
 * 0.5 (f[m+1] + f[m]), m).  first/last point and step(c) = dr(grid) / dz(grid). */
struct CentreRange {
    double first, last, step;
    int64_t lendiv;
    CentreRange(double len, int m) {
        const double f1 = lerpi(0, m, 0.0, len), f2 = lerpi(1, m, 0.0, len);
        const double fm = lerpi(m - 1, m, 0.0, len), fm1 = lerpi(m, m, 0.0, len);
        first = 0.5 * (f2 + f1);
        last = 0.5 * (fm1 + fm);
        lendiv = m > 1 ? m - 1 : 1;
        step = (last - first) / (double)lendiv;
    }
    double at(int64_t i) const { return lerpi(i - 1, lendiv, first, last); }   /* c[i], 1-based */
};

/* LinRange getindex (0-based j): lerpi(j, lendiv, start, stop), Base range.jl */
inline double linrange_at(const orc_table* t, int64_t j) {
    const double lendiv = (double)(t->neps - 1);
    const double tt = (double)j / lendiv;
    return (1.0 - tt) * t->e0 + tt * t->emax;
}

/* energy: JuMC/src/electron.jl:27 */
inline double energy_of(const double v[3]) {
    return 0.5 * ELECTRON_MASS * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
}

/* rate: JuMC/src/collisions.jl:35-39 */
inline double rate_at(const orc_table* t, int j, int64_t k, double w) {
    return w * t->rate[k * t->nrows + j] + (1.0 - w) * t->rate[(k + 1) * t->nrows + j];
}

/* ---------------- fields ---------------- */
/* FieldInterp for the 3-D node mesh (the configs' trilinear gather; the cylindrical
 * analogue is MCStreamer/src/gridfields.jl:115-190).  Zero outside, like :116. */
void efield_cart3d(const orc_field* f, const double x[3], double e[3]) {
    e[0] = e[1] = e[2] = 0.0;
    const double u[3] = {(x[0] - f->x0) / f->h, (x[1] - f->y0) / f->h, (x[2] - f->z0) / f->h};
    const int nc[3] = {f->nx, f->ny, f->nz};
    int64_t ic[3];
    double fr[3];
    for (int d = 0; d < 3; ++d) {
        if (!(u[d] > 0.0 && u[d] < (double)nc[d])) return;  /* grid.jl:45-49 (strict) */
        double fl = std::floor(u[d]);
        if (fl > nc[d] - 1) fl = nc[d] - 1;
        ic[d] = (int64_t)fl;
        fr[d] = u[d] - fl;
    }
    const int64_t sx = 1, sy = f->nx + 1, sz = (int64_t)(f->nx + 1) * (f->ny + 1);
    const int64_t base = ic[0] * sx + ic[1] * sy + ic[2] * sz;
    for (int c = 0; c < 3; ++c) {
        double acc = 0.0;
        for (int b = 0; b < 8; ++b) {
            const int a0 = b & 1, a1 = (b >> 1) & 1, a2 = (b >> 2) & 1;
            const double wgt = (a0 ? fr[0] : 1.0 - fr[0]) * (a1 ? fr[1] : 1.0 - fr[1]) *
                               (a2 ? fr[2] : 1.0 - fr[2]);
            acc += wgt * f->enodes[3 * (base + a0 * sx + a1 * sy + a2 * sz) + c];
        }
        e[c] = acc;
    }
}

/* normdivrem / staggered: MCStreamer/src/gridfields.jl:94-109 */
inline void normdivrem(double x, double y, int64_t* m, double* rem) {
    const double r = x / y;
    const int64_t mi = (int64_t)std::trunc(r);
    *m = mi;
    *rem = r - (double)mi;
}
inline void staggered(int64_t i, double d, int64_t* i1, double* d1) {
    if (d < 0.5) { *i1 = i; *d1 = d + 0.5; }
    else { *i1 = i + 1; *d1 = d - 0.5; }
}

/* Cylindrical FieldInterp: MCStreamer/src/gridfields.jl:115-190.  Returns F_FIELD if |E|>1e8. */
int efield_cyl(const orc_field* f, const double x[3], double e[3]) {
    e[0] = e[1] = e[2] = 0.0;
    const double r0 = std::sqrt(x[0] * x[0] + x[1] * x[1]);
    /* inside: grid.jl:45-49 with rf = LinRange(0, R, M+1), zf = LinRange(0, L, N+1) */
    if (!((0.0 < r0 && r0 < f->R) && (0.0 < x[2] && x[2] < f->L))) return 0;
    const double drc = CentreRange(f->R, f->M).step, dzc = CentreRange(f->L, f->N).step;  /* dr(grid), dz(grid) */
    double r = r0;
    if (r == 0.0) r = drc / 10.0;
    int64_t i, j, i1, j1;
    double dr_, dz_, dr1, dz1;
    normdivrem(r - 0.0, drc, &i, &dr_);
    staggered(i, dr_, &i1, &dr1);
    normdivrem(x[2] - 0.0, dzc, &j, &dz_);
    staggered(j, dz_, &j1, &dz1);
    i += 1; j += 1;
    const int64_t ld = f->M + 3;
    auto ER = [&](int64_t a, int64_t b) { return f->er[a + b * ld]; };
    auto EZ = [&](int64_t a, int64_t b) { return f->ez[a + b * ld]; };
    const double er1 = ER(i, j1) * (1 - dr_) * (1 - dz1) + ER(i + 1, j1) * dr_ * (1 - dz1) +
                       ER(i, j1 + 1) * (1 - dr_) * dz1 + ER(i + 1, j1 + 1) * dr_ * dz1;
    const double ez1 = EZ(i1, j) * (1 - dr1) * (1 - dz_) + EZ(i1 + 1, j) * dr1 * (1 - dz_) +
                       EZ(i1, j + 1) * (1 - dr1) * dz_ + EZ(i1 + 1, j + 1) * dr1 * dz_;
    e[0] = er1 * x[0] / r;
    e[1] = er1 * x[1] / r;
    e[2] = ez1;
    const double nrm = std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
    return nrm > 1e8 ? F_FIELD : 0;
}

int efield_any(const orc_field* f, const double x[3], double e[3]) {
    switch (f->type) {
    case ORC_FIELD_UNIFORM:  /* Swarm/src/Swarm.jl:28-32 FixedField */
        e[0] = f->e[0]; e[1] = f->e[1]; e[2] = f->e[2];
        return 0;
    case ORC_FIELD_CART3D:
        efield_cart3d(f, x, e);
        return 0;
    default:
        return efield_cyl(f, x, e);
    }
}

/* advance_free_yoshida: JuMC/src/electron.jl:51-62 */
int yoshida(const orc_field* f, double x[3], double v[3], double dt) {
    const double qm = (-ELEMENTARY_CHARGE) / ELECTRON_MASS;  /* charge(p)/mass(p) */
    double E[3];
    int st = 0;
    double x1[3], v1[3], x2[3], v2[3], x3[3], v3[3];
    for (int d = 0; d < 3; ++d) x1[d] = x[d] + YO.c1 * dt * v[d];
    st |= efield_any(f, x1, E);
    for (int d = 0; d < 3; ++d) v1[d] = v[d] + YO.d1 * dt * qm * E[d];
    for (int d = 0; d < 3; ++d) x2[d] = x1[d] + YO.c2 * dt * v1[d];
    st |= efield_any(f, x2, E);
    for (int d = 0; d < 3; ++d) v2[d] = v1[d] + YO.d2 * dt * qm * E[d];
    for (int d = 0; d < 3; ++d) x3[d] = x2[d] + YO.c3 * dt * v2[d];
    st |= efield_any(f, x3, E);
    for (int d = 0; d < 3; ++d) v3[d] = v2[d] + YO.d3 * dt * qm * E[d];
    for (int d = 0; d < 3; ++d) { x[d] = x3[d] + YO.c4 * dt * v3[d]; v[d] = v3[d]; }
    return st;
}

/* ---------------- trackers (deposits) ---------------- */
inline void atomic_add_i64(int64_t* p, int64_t v) { __atomic_fetch_add(p, v, __ATOMIC_RELAXED); }

/* CIC with int64 fixed point at 2^-32 elementary charges.  Seven corners are rounded,
 * the eighth takes the remainder so the node sum equals llrint(q*2^32) exactly. */
void cic_fixed(int64_t* q, int nx, int ny, const int64_t ic[3], const double fr[3], double charge) {
    const int64_t W = std::llrint(charge * 0x1p32);
    const double Wd = (double)W;
    const double g[3][2] = {{1.0 - fr[0], fr[0]}, {1.0 - fr[1], fr[1]}, {1.0 - fr[2], fr[2]}};
    const int64_t sy = nx + 1, sz = (int64_t)(nx + 1) * (ny + 1);
    const int64_t base = ic[0] + ic[1] * sy + ic[2] * sz;
    int64_t acc = 0;
    for (int b = 0; b < 7; ++b) {
        const int a0 = b & 1, a1 = (b >> 1) & 1, a2 = (b >> 2) & 1;
        const double wc = (g[0][a0] * g[1][a1]) * g[2][a2];
        const int64_t qb = std::llrint(Wd * wc);
        acc += qb;
        atomic_add_i64(&q[base + a0 + a1 * sy + a2 * sz], qb);
    }
    atomic_add_i64(&q[base + 1 + sy + sz], W - acc);
}

/* Cell and in-cell fraction of an absolute position on the 3-D mesh; false if outside
 * [0, n) on any axis.  quantize rounds the fraction to float like the device layout. */
bool cart3d_locate(int nx, int ny, int nz, double h, double x0, double y0, double z0,
                   const double x[3], int64_t ic[3], double fr[3], bool quantize) {
    const double u[3] = {(x[0] - x0) / h, (x[1] - y0) / h, (x[2] - z0) / h};
    const int nc[3] = {nx, ny, nz};
    for (int d = 0; d < 3; ++d) {
        const double fl = std::floor(u[d]);
        if (!(fl >= 0.0 && fl < (double)nc[d])) return false;
        ic[d] = (int64_t)fl;
        double r = u[d] - fl;
        if (quantize) {
            float rf = (float)r;
            if (rf >= 1.0f) rf = 0x1.fffffep-1f;
            r = (double)rf;
        }
        fr[d] = r;
    }
    return true;
}

/* track1: MCStreamer/src/gridfields.jl:203-213 (cyl NGP) and the 3-D CIC analogue. */
void track_charge(orc_tracker* t, const double x[3], double val, std::vector<double>* cyl_local) {
    if (!t || t->type == ORC_TRACK_NONE) return;
    if (t->type == ORC_TRACK_CART3D) {
        int64_t ic[3]; double fr[3];
        if (!cart3d_locate(t->nx, t->ny, t->nz, t->h, t->x0, t->y0, t->z0, x, ic, fr, false)) return;
        cic_fixed(t->qnodes, t->nx, t->ny, ic, fr, val);
        return;
    }
    /* cellindex: MCStreamer/src/grid.jl:84-90; dV: grid.jl:76 */
    const double rho = std::sqrt(x[0] * x[0] + x[1] * x[1]);
    const double drf = t->R / t->M, dzf = t->L / t->N;
    const double fi = julia_fld(rho - 0.0, drf) + 1.0;
    const double fj = julia_fld(x[2] - 0.0, dzf) + 1.0;
    if (!(fi >= 1.0 && fi <= (double)t->M)) return;      /* checkbounds(grid.rc, i) */
    if (!(fj >= 0.0 && fj <= (double)t->N + 1.0)) return; /* checkbounds(qfixed, j) */
    const int64_t i = (int64_t)fi, j = (int64_t)fj;
    const CentreRange rcr(t->R, t->M);
    const double dV = 2.0 * M_PI * rcr.at(i) * rcr.step * CentreRange(t->L, t->N).step;   /* grid.jl:76 */
    (*cyl_local)[i + j * (t->M + 2)] += val / dV;
}

/* ---------------- tables ---------------- */
/* indweight: JuMC/src/util.jl:23-30.  Energies beyond the table raise a BoundsError /
 * @assert in the reference; here they use the edge column (flat extrapolation) and
 * return F_ENERGY unless `clamp` asks for silent clamping. */
int indweight(const orc_table* t, double eng, int64_t* k, double* w, int clamp) {
    const double step = (t->emax - t->e0) / (double)(t->neps - 1);
    double fk = julia_fld(eng - t->e0, step);
    if (!(fk >= 0.0 && fk <= (double)(t->neps - 2))) {
        const bool low = !(fk >= 0.0) && eng < t->e0;
        fk = low ? 0.0 : (double)(t->neps - 2);
        *k = (int64_t)fk;
        *w = low ? 1.0 : 0.0;
        return clamp ? 0 : F_ENERGY;
    }
    *k = (int64_t)fk;
    *w = (linrange_at(t, *k + 1) - eng) / step;
    return 0;
}

struct Secondary { double x[3], v[3], w, s; uint8_t active; };
struct PhotonOut { double x[3], v[3], nu, w, s; uint8_t active; };

struct StepCtx {
    const orc_table* tab;
    const orc_field* fld;
    orc_tracker* trk;
    std::vector<double>* cyl_local;
    std::vector<Secondary>* out;
    int clamp;
    int status;
    std::vector<PhotonOut>* photons;   /* photo-emission output (NULL: rows rejected) */
};

/* Poisson sampler: inversion for lambda < 10, PTRS (Hoermann 1993) otherwise.
 * The reference draws Distributions.Poisson (Swarm.jl:216); only the law is matched. */
int64_t poisson_sample(Stream& rng, double lam) {
    if (lam <= 0) return 0;
    if (lam < 10.0) {
        const double u = rng.next();
        double p = std::exp(-lam), F = p;
        int64_t k = 0;
        while (u > F && k < 1000) { ++k; p *= lam / (double)k; F += p; }
        return k;
    }
    const double slam = std::sqrt(lam), loglam = std::log(lam);
    const double b = 0.931 + 2.53 * slam;
    const double a = -0.059 + 0.02483 * b;
    const double invalpha = 1.1239 + 1.1328 / (b - 3.4);
    const double vr = 0.9277 - 3.6224 / (b - 2.0);
    for (int it = 0; it < 1000; ++it) {
        const double U = rng.next() - 0.5;
        const double V = rng.next();
        const double us = 0.5 - std::fabs(U);
        const double kf = std::floor((2.0 * a / us + b) * U + lam + 0.43);
        if (us >= 0.07 && V <= vr) return (int64_t)kf;
        if (kf < 0 || (us < 0.013 && V > us)) continue;
        if (std::log(V) + std::log(invalpha) - std::log(a / (us * us) + b) <=
            -lam + kf * loglam - std::lgamma(kf + 1.0))
            return (int64_t)kf;
    }
    return (int64_t)std::floor(lam);
}

/* collide(::PhotoEmission) + apply!(::MultiplePhotonOutcome) (electron.jl:141-144,
 * collisions.jl:125-141): the electron is unchanged; rand(Poisson(w / multiplier /
 * photon_weight)) photons at its position, each with randsphere() * c, nu = exp(log_numin +
 * (log_numax - log_numin) rand()), weight photon_weight, nextcoll() and the electron's
 * active flag.  No charge is tracked. */
void photo_emit(StepCtx& c, const Event& rng, int row, const double x[3], double w, uint8_t active) {
    const orc_table* t = c.tab;
    const uint64_t seed = (uint64_t)rng.key[0] | ((uint64_t)rng.key[1] << 32);
    const uint32_t jev = rng.j - 1;
    Stream cnt(seed, rng.c0, rng.c1, ORC_TAG_PHOTON_COUNT | jev);
    const int64_t n = poisson_sample(cnt, w / t->pe_mult / t->pe_pw);
    Stream ps(seed, rng.c0, rng.c1, ORC_TAG_PHOTON_DRAW | jev);
    const double lmin = t->pe_lmin[row], lmax = t->pe_lmax[row];
    for (int64_t p = 0; p < n; ++p) {
        PhotonOut ph;
        const double uphi = ps.next(), uu = ps.next();
        double d[3];
        randsphere(uphi, uu, d);
        for (int q = 0; q < 3; ++q) { ph.x[q] = x[q]; ph.v[q] = d[q] * SPEED_OF_LIGHT; }
        ph.nu = std::exp(lmin + (lmax - lmin) * ps.next());
        ph.w = t->pe_pw;
        ph.s = -std::log(ps.next());
        ph.active = active;
        c.photons->push_back(ph);
    }
}

/* do_one_collision!: JuMC/src/collisions.jl:159-192 with collide (electron.jl:108-139),
 * track (collisions.jl:151, gridfields.jl:215-224) and apply! (collisions.jl:96-123). */
void do_one_collision(StepCtx& c, Event& rng, double x[3], double v[3], double& w, double& s,
                      uint8_t& active) {
    const orc_table* t = c.tab;
    const double eng = energy_of(v);
    int64_t k; double wk;
    c.status |= indweight(t, eng, &k, &wk, c.clamp);
    rng.begin();
    double xi = rng.u(U_XI) * t->maxrate;
    for (int j = 0; j < t->nrows; ++j) {
        const double nu = rate_at(t, j, k, wk);
        if (nu > xi) {
            const int kind = t->kind[j];
            const double par = t->param[j];
            if (kind == ORC_ELASTIC) {
                const double f = par / (1.0 + par);
                const double vcm[3] = {f * v[0], f * v[1], f * v[2]};
                const double dv[3] = {v[0] - vcm[0], v[1] - vcm[1], v[2] - vcm[2]};
                const double nrm = std::sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
                const double uphi = rng.u(U_PHI), ucos = rng.u(U_COS);
                double d[3]; randsphere(uphi, ucos, d);
                for (int q = 0; q < 3; ++q) v[q] = d[q] * nrm + vcm[q];
            } else if (kind == ORC_EXCITATION) {
                const double E1 = std::max(0.0, eng - par);
                const double vabs = std::sqrt(2.0 * E1 / ELECTRON_MASS);
                const double uphi = rng.u(U_PHI), ucos = rng.u(U_COS);
                double d[3]; randsphere(uphi, ucos, d);
                for (int q = 0; q < 3; ++q) v[q] = d[q] * vabs;
            } else if (kind == ORC_IONIZATION || kind == ORC_IONIZATION_UNIFORM) {
                double va1, va2;
                if (kind == ORC_IONIZATION) {
                    const double E1 = std::max(0.0, eng - par) / 2.0;
                    va1 = va2 = std::sqrt(2.0 * E1 / ELECTRON_MASS);
                } else {
                    /* Extension (not in JuMC): secondary energy uniform on [0, eps-th]. */
                    const double Ea = std::max(0.0, eng - par);
                    const double E2 = rng.u(U_SHARE) * Ea;
                    const double E1 = Ea - E2;
                    va1 = std::sqrt(2.0 * E1 / ELECTRON_MASS);
                    va2 = std::sqrt(2.0 * E2 / ELECTRON_MASS);
                }
                double d1[3], d2[3];
                const double uphi1 = rng.u(U_PHI), ucos1 = rng.u(U_COS);
                randsphere(uphi1, ucos1, d1);
                const double uphi2 = rng.u(U_PHI2), ucos2 = rng.u(U_COS2);
                randsphere(uphi2, ucos2, d2);
                Secondary sec;
                for (int q = 0; q < 3; ++q) { sec.x[q] = x[q]; sec.v[q] = d2[q] * va2; }
                sec.w = w;
                sec.s = nextcoll(rng.u(U_S2));
                sec.active = active;
                track_charge(c.trk, x, w, c.cyl_local);       /* NewParticleOutcome: +w */
                for (int q = 0; q < 3; ++q) v[q] = d1[q] * va1;
                c.out->push_back(sec);
            } else if (kind == ORC_ATTACHMENT) {
                track_charge(c.trk, x, -w, c.cyl_local);      /* RemoveParticleOutcome: -w */
                active = 0;
            } else if (kind == ORC_PHOTOEMISSION) {
                if (c.photons) photo_emit(c, rng, j, x, w, active);
                else c.status |= F_UNSUPPORTED;
            }
            /* ORC_NULL: NullOutcome, nothing */
            return;
        }
        xi -= nu;
    }
}

void run_chunks(int64_t n, int nthreads, const std::function<void(int, int64_t, int64_t)>& f) {
    if (nthreads < 1) nthreads = 1;
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthreads) schedule(static, 1)
#endif
    for (int t = 0; t < nthreads; ++t) {
        const int64_t lo = n * t / nthreads, hi = n * (t + 1) / nthreads;
        f(t, lo, hi);
    }
}

/* Shared driver for advance! and collisions!: runs per-particle work in contiguous
 * chunks, then appends secondaries in chunk order (== serial parent order). */
int drive(orc_pop* pop, const orc_table* tab, const orc_field* fld, orc_tracker* trk,
          int nthreads, int clamp,
          const std::function<void(StepCtx&, int64_t)>& per_particle, orc_photons* ph_out = nullptr) {
    if (nthreads < 1) nthreads = 1;
    const int64_t n_entry = pop->n;
    std::vector<std::vector<Secondary>> outs(nthreads);
    std::vector<std::vector<PhotonOut>> phs(nthreads);
    std::vector<std::vector<double>> cyl(nthreads);
    std::vector<int> status(nthreads, 0);
    const bool is_cyl = trk && trk->type == ORC_TRACK_CYL;
    run_chunks(n_entry, nthreads, [&](int t, int64_t lo, int64_t hi) {
        if (is_cyl) cyl[t].assign((size_t)(trk->M + 2) * (trk->N + 2), 0.0);
        StepCtx c{tab, fld, trk, &cyl[t], &outs[t], clamp, 0, ph_out ? &phs[t] : nullptr};
        for (int64_t i = lo; i < hi; ++i) per_particle(c, i);
        status[t] = c.status;
    });
    /* photons in serial parent order (add_particle!(photons, p2), collisions.jl:138) */
    if (ph_out)
        for (int t = 0; t < nthreads; ++t)
            for (const PhotonOut& ph : phs[t]) {
                if (ph_out->n >= ph_out->cap) { status[t] |= F_CAP; continue; }
                const int64_t m = ph_out->n++;
                for (int q = 0; q < 3; ++q) { ph_out->x[3 * m + q] = ph.x[q]; ph_out->v[3 * m + q] = ph.v[q]; }
                ph_out->nu[m] = ph.nu; ph_out->w[m] = ph.w; ph_out->s[m] = ph.s; ph_out->active[m] = ph.active;
            }
    int st = 0;
    for (int t = 0; t < nthreads; ++t) st |= status[t];
    if (is_cyl) {
        const size_t m = (size_t)(trk->M + 2) * (trk->N + 2);
        for (int t = 0; t < nthreads; ++t)
            for (size_t q = 0; q < m; ++q) trk->qcyl[q] += cyl[t][q];
    }
    /* add_particle!: JuMC/src/population.jl:88-97 (capacity assert :90) */
    int64_t n = n_entry;
    for (int t = 0; t < nthreads; ++t) {
        for (const Secondary& s : outs[t]) {
            if (n >= pop->cap) { st |= F_CAP; continue; }
            for (int q = 0; q < 3; ++q) { pop->x[3 * n + q] = s.x[q]; pop->v[3 * n + q] = s.v[q]; }
            pop->w[n] = s.w; pop->s[n] = s.s; pop->active[n] = s.active;
            ++n;
        }
    }
    pop->n = n;
    pop->step += 1;
    return status_code(st);
}
}  // namespace

extern "C" {

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    philox10(ctr, key, out);
}

double orc_uniform(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t tag, uint32_t k) {
    Stream s(seed, c0, c1, tag);
    double u = 0.0;
    for (uint32_t i = 0; i <= k; ++i) u = s.next();
    return u;
}

void orc_efield(const orc_field* fld, const double x[3], double e[3]) { efield_any(fld, x, e); }

int orc_indweight(const orc_table* tab, double eng, int64_t* k, double* w) {
    return indweight(tab, eng, k, w, 0);
}

void orc_yoshida(const orc_field* fld, double x[3], double v[3], double dt) { yoshida(fld, x, v, dt); }

/* advance!: JuMC/src/mixed_population.jl:24-54 */
static int advance_electrons(orc_pop* pop, const orc_table* tab, const orc_field* fld, double dt,
                             orc_tracker* trk, int nthreads, int clamp_energy, orc_photons* ph_out,
                             const Injected* inj = nullptr) {
    const uint64_t seed = pop->seed;
    const uint32_t step = pop->step;
    return drive(pop, tab, fld, trk, nthreads, clamp_energy, [&](StepCtx& c, int64_t i) {
        if (!pop->active[i]) return;                 /* l.active || continue */
        Event rng(seed, (uint32_t)i, step, ORC_TAG_ADVANCE);
        rng.inject(inj, i, &c.status);
        double x[3] = {pop->x[3 * i], pop->x[3 * i + 1], pop->x[3 * i + 2]};
        double v[3] = {pop->v[3 * i], pop->v[3 * i + 1], pop->v[3 * i + 2]};
        double w = pop->w[i], s = pop->s[i];
        uint8_t active = pop->active[i];
        double trem = dt;
        while (trem > 0) {
            const double tnext = s / tab->maxrate;
            double t;
            bool collides;
            if (trem > tnext) { t = tnext; collides = true; }
            else { t = trem; collides = false; s -= t * tab->maxrate; }
            c.status |= yoshida(fld, x, v, t);
            if (collides) {
                do_one_collision(c, rng, x, v, w, s, active);
                s = nextcoll(rng.u(U_S));
            }
            trem -= t;
        }
        rng.finish(i);
        for (int q = 0; q < 3; ++q) { pop->x[3 * i + q] = x[q]; pop->v[3 * i + q] = v[q]; }
        pop->w[i] = w; pop->s[i] = s; pop->active[i] = active;
    }, ph_out);
}

int orc_advance(orc_pop* pop, const orc_table* tab, const orc_field* fld, double dt,
                orc_tracker* trk, int nthreads, int clamp_energy) {
    return advance_electrons(pop, tab, fld, dt, trk, nthreads, clamp_energy, nullptr);
}

int orc_advance_injected(orc_pop* pop, const orc_table* tab, const orc_field* fld, double dt,
                         orc_tracker* trk, int nthreads, int clamp_energy, const double* u, int64_t* pos,
                         const int64_t* end, int64_t nslots) {
    const Injected inj{u, pos, end, nslots};
    return advance_electrons(pop, tab, fld, dt, trk, nthreads, clamp_energy, nullptr, &inj);
}

/* advance! of the photon population (mixed_population.jl:24-54 with the
 * ZhelezniakCollisions table, photon.jl:27-56): straight flight x + t v; at a collision
 * xi = rand() * numax and PhotoIonization when nu > xi: the tracker adds +w at the photon
 * (gridfields.jl:219-222), the photon is removed and an electron at rest with its weight,
 * nextcoll() and the photon's active flag is added.  A removed photon keeps sub-stepping to
 * the end of the step, as the reference's loop does, so it can photo-ionize again. */
int orc_photon_advance(orc_photons* ph, orc_pop* e, double dt, orc_tracker* trk, int nthreads) {
    if (nthreads < 1) nthreads = 1;
    const int64_t n_entry = ph->n;
    std::vector<std::vector<Secondary>> outs(nthreads);
    std::vector<std::vector<double>> cyl(nthreads);
    const bool is_cyl = trk && trk->type == ORC_TRACK_CYL;
    const double numax = ph->numax;
    run_chunks(n_entry, nthreads, [&](int t, int64_t lo, int64_t hi) {
        if (is_cyl) cyl[t].assign((size_t)(trk->M + 2) * (trk->N + 2), 0.0);
        for (int64_t i = lo; i < hi; ++i) {
            if (!ph->active[i]) continue;
            Event rng(ph->seed, (uint32_t)i, ph->step, ORC_TAG_PHOTON);
            double x[3] = {ph->x[3 * i], ph->x[3 * i + 1], ph->x[3 * i + 2]};
            const double v[3] = {ph->v[3 * i], ph->v[3 * i + 1], ph->v[3 * i + 2]};
            const double nu = ph->nu[i], w = ph->w[i];
            double s = ph->s[i];
            uint8_t active = 1;
            double trem = dt;
            while (trem > 0) {
                const double tnext = s / numax;
                double tt;
                bool collides;
                if (trem > tnext) { tt = tnext; collides = true; }
                else { tt = trem; collides = false; s -= tt * numax; }
                for (int q = 0; q < 3; ++q) x[q] = x[q] + tt * v[q];   /* advance_free, photon.jl:54-56 */
                if (collides) {
                    rng.begin();
                    const double xi = rng.u(U_XI) * numax;
                    if (nu > xi) {
                        track_charge(trk, x, w, &cyl[t]);
                        Secondary sec;
                        for (int q = 0; q < 3; ++q) { sec.x[q] = x[q]; sec.v[q] = 0.0; }
                        sec.w = w;
                        sec.s = nextcoll(rng.u(U_PHI));
                        sec.active = active;
                        outs[t].push_back(sec);
                        active = 0;
                    }
                    s = nextcoll(rng.u(U_S));
                }
                trem -= tt;
            }
            for (int q = 0; q < 3; ++q) ph->x[3 * i + q] = x[q];
            ph->s[i] = s;
            ph->active[i] = active;
        }
    });
    int st = 0;
    if (is_cyl) {
        const size_t m = (size_t)(trk->M + 2) * (trk->N + 2);
        for (int t = 0; t < nthreads; ++t)
            for (size_t q = 0; q < m; ++q) trk->qcyl[q] += cyl[t][q];
    }
    int64_t n = e->n;
    for (int t = 0; t < nthreads; ++t)
        for (const Secondary& sc : outs[t]) {
            if (n >= e->cap) { st |= F_CAP; continue; }
            for (int q = 0; q < 3; ++q) { e->x[3 * n + q] = sc.x[q]; e->v[3 * n + q] = sc.v[q]; }
            e->w[n] = sc.w; e->s[n] = sc.s; e->active[n] = sc.active;
            ++n;
        }
    e->n = n;
    ph->step += 1;
    return status_code(st);
}

int orc_advance_mixed(orc_pop* e, orc_photons* ph, const orc_table* tab, const orc_field* fld, double dt,
                      orc_tracker* trk, int nthreads, int clamp_energy) {
    const int st = advance_electrons(e, tab, fld, dt, trk, nthreads, clamp_energy, ph);
    const int st2 = orc_photon_advance(ph, e, dt, trk, nthreads);
    return st ? st : st2;
}

/* collisions!: JuMC/src/mixed_population.jl:61-77 (fixed-step variant, no push) */
int orc_collisions(orc_pop* pop, const orc_table* tab, double dt, orc_tracker* trk,
                   int nthreads, int clamp_energy) {
    const uint64_t seed = pop->seed;
    const uint32_t step = pop->step;
    orc_field none{};
    none.type = ORC_FIELD_UNIFORM;
    return drive(pop, tab, &none, trk, nthreads, clamp_energy, [&](StepCtx& c, int64_t i) {
        if (!pop->active[i]) return;
        double s = pop->s[i] - dt * tab->maxrate;
        if (s <= 0) {
            Event rng(seed, (uint32_t)i, step, ORC_TAG_COLLISIONS);
            double x[3] = {pop->x[3 * i], pop->x[3 * i + 1], pop->x[3 * i + 2]};
            double v[3] = {pop->v[3 * i], pop->v[3 * i + 1], pop->v[3 * i + 2]};
            double w = pop->w[i];
            uint8_t active = pop->active[i];
            do_one_collision(c, rng, x, v, w, s, active);
            s = nextcoll(rng.u(U_S));
            for (int q = 0; q < 3; ++q) pop->v[3 * i + q] = v[q];
            pop->active[i] = active;
        }
        pop->s[i] = s;
    });
}

/* repack!: JuMC/src/population.jl:191-215.  The reference throws a BoundsError when
 * no particle is active; here the population becomes empty instead. */
int orc_repack(orc_pop* pop) {
    int64_t l = pop->n - 1;
    if (pop->n == 0) return 0;
    while (l >= 0 && !pop->active[l]) --l;
    if (l < 0) { pop->n = 0; return 0; }
    auto copy = [&](int64_t dst, int64_t src) {
        for (int q = 0; q < 3; ++q) { pop->x[3 * dst + q] = pop->x[3 * src + q]; pop->v[3 * dst + q] = pop->v[3 * src + q]; }
        pop->w[dst] = pop->w[src]; pop->s[dst] = pop->s[src]; pop->active[dst] = pop->active[src];
    };
    int64_t i = 0;
    while (i <= l) {
        if (!pop->active[i]) {
            copy(i, l);
            --l;
            while (!pop->active[l]) --l;
        }
        ++i;
    }
    pop->n = l + 1;
    return 0;
}

/* repack!(photons): the same loop over the photon arrays. */
int orc_photons_repack(orc_photons* ph) {
    if (ph->n == 0) return 0;
    int64_t l = ph->n - 1;
    while (l >= 0 && !ph->active[l]) --l;
    if (l < 0) { ph->n = 0; return 0; }
    auto copy = [&](int64_t dst, int64_t src) {
        for (int q = 0; q < 3; ++q) { ph->x[3 * dst + q] = ph->x[3 * src + q]; ph->v[3 * dst + q] = ph->v[3 * src + q]; }
        ph->nu[dst] = ph->nu[src]; ph->w[dst] = ph->w[src]; ph->s[dst] = ph->s[src]; ph->active[dst] = ph->active[src];
    };
    int64_t i = 0;
    while (i <= l) {
        if (!ph->active[i]) {
            copy(i, l);
            --l;
            while (!ph->active[l]) --l;
        }
        ++i;
    }
    ph->n = l + 1;
    return 0;
}

/* Swarm.resample!: Swarm/src/Swarm.jl:193-223 */
int orc_swarm_resample(orc_pop* pop, int64_t n0, double tol) {
    int64_t ncur = 0;
    for (int64_t i = 0; i < pop->n; ++i) ncur += pop->active[i] ? 1 : 0;
    if (std::fabs((double)(ncur - n0) / (double)n0) < tol) return 0;
    const int64_t n_entry = pop->n;
    int st = 0;
    if (ncur > n0) {
        const double pdrop = (double)(ncur - n0) / (double)ncur;
        for (int64_t i = 0; i < n_entry; ++i) {
            if (!pop->active[i]) continue;
            Stream rng(pop->seed, (uint32_t)i, pop->step, ORC_TAG_SWARM_RESAMPLE);
            if (rng.next() < pdrop) pop->active[i] = 0;
        }
    } else {
        const double lam = (double)(n0 - ncur) / (double)ncur;
        for (int64_t i = 0; i < n_entry; ++i) {
            if (!pop->active[i]) continue;
            Stream rng(pop->seed, (uint32_t)i, pop->step, ORC_TAG_SWARM_RESAMPLE);
            const int64_t nnew = poisson_sample(rng, lam);
            for (int64_t j = 0; j < nnew; ++j) {
                if (pop->n >= pop->cap) { st = 3; break; }
                const int64_t d = pop->n++;
                for (int q = 0; q < 3; ++q) { pop->x[3 * d + q] = pop->x[3 * i + q]; pop->v[3 * d + q] = pop->v[3 * i + q]; }
                pop->w[d] = pop->w[i]; pop->s[d] = pop->s[i]; pop->active[d] = pop->active[i];
            }
        }
    }
    return st;
}

/* Moments: the per-step Swarm estimators (Swarm/src/Swarm.jl:126-127,152,156,242-248)
 * and JuMC diagnostics (population.jl:114-183).  Layout (doubles):
 *  0 n_active, 1 sum w, 2-4 sum x, 5-7 sum x^2, 8-10 sum v, 11 sum eps, 12 sum w*eps,
 *  13 max eps over ALL particles (population.jl:156-158 iterates eachparticle),
 *  14-16 sum w*x, 17 sum w*|x|^2, 18.. sum of rate_j(eps) over actives (collrate). */
void orc_moments(const orc_pop* pop, const orc_table* tab, double* out) {
    const int nm = 18 + (tab ? tab->nrows : 0);
    for (int q = 0; q < nm; ++q) out[q] = 0.0;
    out[13] = -INFINITY;
    for (int64_t i = 0; i < pop->n; ++i) {
        const double* v = &pop->v[3 * i];
        const double eng = energy_of(v);
        out[13] = std::max(out[13], eng);
        if (!pop->active[i]) continue;
        const double* x = &pop->x[3 * i];
        const double w = pop->w[i];
        out[0] += 1.0;
        out[1] += w;
        for (int q = 0; q < 3; ++q) {
            out[2 + q] += x[q];
            out[5 + q] += x[q] * x[q];
            out[8 + q] += v[q];
            out[14 + q] += w * x[q];
        }
        out[11] += eng;
        out[12] += w * eng;
        out[17] += w * (x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
        if (tab) {
            int64_t k; double wk;
            indweight(tab, eng, &k, &wk, 1);
            for (int j = 0; j < tab->nrows; ++j) out[18 + j] += rate_at(tab, j, k, wk);
        }
    }
}

/* Cell key: MCStreamer/src/grid.jl:84-90 (cyl, array p over (0:M+1, 0:N+1)) or the
 * 3-D mesh analogue (cells 0..n-1 per axis). */
int64_t orc_cell_key(const orc_field* g, const double x[3]) {
    if (g->type == ORC_FIELD_CART3D) {
        int64_t ic[3]; double fr[3];
        if (!cart3d_locate(g->nx, g->ny, g->nz, g->h, g->x0, g->y0, g->z0, x, ic, fr, false)) return -1;
        return ic[0] + (int64_t)g->nx * (ic[1] + (int64_t)g->ny * ic[2]);
    }
    const double rho = std::sqrt(x[0] * x[0] + x[1] * x[1]);
    const double fi = julia_fld(rho - 0.0, g->R / g->M) + 1.0;
    const double fj = julia_fld(x[2] - 0.0, g->L / g->N) + 1.0;
    if (!(fi >= 0.0 && fi <= g->M + 1.0 && fj >= 0.0 && fj <= g->N + 1.0)) return -1;
    return (int64_t)fi + (int64_t)(g->M + 2) * (int64_t)fj;
}

int orc_sort_cells(orc_pop* pop, const orc_field* g) {
    const int64_t n = pop->n;
    std::vector<int64_t> key(n), idx(n);
    for (int64_t i = 0; i < n; ++i) {
        /* inactive and out-of-grid particles go last */
        int64_t k = pop->active[i] ? orc_cell_key(g, &pop->x[3 * i]) : -1;
        key[i] = k < 0 ? INT64_MAX : k;
        idx[i] = i;
    }
    std::stable_sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) { return key[a] < key[b]; });
    std::vector<double> x(3 * n), v(3 * n), w(n), s(n);
    std::vector<uint8_t> a(n);
    for (int64_t i = 0; i < n; ++i) {
        const int64_t j = idx[i];
        for (int q = 0; q < 3; ++q) { x[3 * i + q] = pop->x[3 * j + q]; v[3 * i + q] = pop->v[3 * j + q]; }
        w[i] = pop->w[j]; s[i] = pop->s[j]; a[i] = pop->active[j];
    }
    std::memcpy(pop->x, x.data(), sizeof(double) * 3 * n);
    std::memcpy(pop->v, v.data(), sizeof(double) * 3 * n);
    std::memcpy(pop->w, w.data(), sizeof(double) * n);
    std::memcpy(pop->s, s.data(), sizeof(double) * n);
    std::memcpy(pop->active, a.data(), n);
    return 0;
}

/* resample!: MCStreamer/src/resample.jl:7-77, samplemin :84.  Uniforms come from one
 * Philox stream per cell (ctr = {cell key, call, k/4, TAG_CELL_RESAMPLE}). */
int orc_resample_cells(orc_pop* pop, const orc_field* g, int ntarget, int nmax, uint32_t call) {
    struct Cell { int64_t p = 0, pk = 0; double wtotal = 0, wcum = 0, x = 0; Stream* rng = nullptr; };
    std::vector<int64_t> key(pop->n);
    std::vector<Cell> cells;
    std::vector<Stream> streams;
    /* map key -> dense index */
    std::vector<std::pair<int64_t, int64_t>> kv;
    for (int64_t i = 0; i < pop->n; ++i) {
        key[i] = pop->active[i] ? orc_cell_key(g, &pop->x[3 * i]) : -1;
        if (key[i] >= 0) kv.push_back({key[i], i});
    }
    std::sort(kv.begin(), kv.end());
    std::vector<int64_t> dense(pop->n, -1);
    std::vector<int64_t> cellkey;
    for (size_t q = 0; q < kv.size(); ++q) {
        if (q == 0 || kv[q].first != kv[q - 1].first) cellkey.push_back(kv[q].first);
        dense[kv[q].second] = (int64_t)cellkey.size() - 1;
    }
    cells.resize(cellkey.size());
    streams.reserve(cellkey.size());
    for (size_t c = 0; c < cellkey.size(); ++c) {
        streams.emplace_back(pop->seed, (uint32_t)cellkey[c], call, ORC_TAG_CELL_RESAMPLE);
        cells[c].rng = &streams[c];
    }
    auto samplemin = [](Stream& r, double m) { return 1.0 - std::pow(1.0 - r.next(), 1.0 / m); };
    /* pass 1 (serial, index order): resample.jl:16-29 */
    for (int64_t i = 0; i < pop->n; ++i) {
        if (dense[i] < 0) continue;
        Cell& C = cells[dense[i]];
        C.p += 1;
        C.wtotal += pop->w[i];
        if (C.p == nmax) C.x = samplemin(*C.rng, (double)ntarget);
    }
    /* pass 2: resample.jl:31-76 (per cell in index order; new particles not revisited) */
    const int64_t n_entry = pop->n;
    int st = 0;
    auto clone = [&](int64_t i) -> int64_t {
        if (pop->n >= pop->cap) { st = 3; return -1; }
        const int64_t d = pop->n++;
        for (int q = 0; q < 3; ++q) { pop->x[3 * d + q] = pop->x[3 * i + q]; pop->v[3 * d + q] = pop->v[3 * i + q]; }
        pop->w[d] = pop->w[i]; pop->s[d] = pop->s[i]; pop->active[d] = pop->active[i];
        return d;
    };
    for (int64_t i = 0; i < n_entry; ++i) {
        if (dense[i] < 0) continue;
        Cell& C = cells[dense[i]];
        if (C.p > nmax) {
            while (C.wtotal * C.x < C.wcum + pop->w[i] && C.pk < ntarget) {
                C.pk += 1;
                const int64_t d = clone(i);
                if (d >= 0) pop->w[d] = C.wtotal / (double)ntarget;
                if (C.pk < ntarget) C.x += samplemin(*C.rng, (double)(ntarget - C.pk)) * (1.0 - C.x);
            }
            C.wcum += pop->w[i];
            pop->active[i] = 0;
        } else if (C.p < ntarget && pop->w[i] > 2) {
            const double wnew = std::nearbyint(pop->w[i] / 2.0);
            const int64_t d = clone(i);
            if (d >= 0) pop->w[d] = wnew;
            pop->w[i] = pop->w[i] - wnew;
            C.p += 1;
        }
    }
    return st;
}

/* density!: MCStreamer/src/poisson.jl:65-84 (cyl NGP, val/dV) and the 3-D CIC analogue
 * (int64, 2^-32 fixed point).  quantize_f32 rounds in-cell fractions to float exactly
 * like the device population layout does at upload. */
void orc_deposit(const orc_pop* pop, orc_tracker* trk, double val, int quantize_f32) {
    std::vector<double> cyl;
    if (trk->type == ORC_TRACK_CYL) cyl.assign((size_t)(trk->M + 2) * (trk->N + 2), 0.0);
    for (int64_t i = 0; i < pop->n; ++i) {
        if (!pop->active[i]) continue;
        const double* x = &pop->x[3 * i];
        if (trk->type == ORC_TRACK_CART3D) {
            int64_t ic[3]; double fr[3];
            if (!cart3d_locate(trk->nx, trk->ny, trk->nz, trk->h, trk->x0, trk->y0, trk->z0, x,
                               ic, fr, quantize_f32 != 0))
                continue;
            double wv = pop->w[i];
            if (quantize_f32) wv = (double)(float)wv;
            cic_fixed(trk->qnodes, trk->nx, trk->ny, ic, fr, wv * val);
        } else {
            track_charge(trk, x, pop->w[i] * val, &cyl);
        }
    }
    if (trk->type == ORC_TRACK_CYL)
        for (size_t q = 0; q < cyl.size(); ++q) trk->qcyl[q] += cyl[q];
}

}  // extern "C"

/* ---------------- initfromfiles!: MCStreamer/src/initdens.jl:64-159 ---------------- */
namespace {

struct CellSample {
    int64_t nume;
    double qf, w;
};

/* randround: initdens.jl:145-159 */
int64_t randround(Stream& rng, double x) {
    const double m = std::floor(x);
    const double f = x - m;
    return rng.next() > f ? (int64_t)m : (int64_t)m + 1;
}

/* nsample(::NoiselessInitSampling) :109-127 and nsample(::PoissonInitSampling) :130-142 */
CellSample nsample(int method, int64_t p, double ne, double q, double V, Stream& rng) {
    CellSample c{};
    const double pf = (double)p;
    if (method == ORC_INIT_NOISELESS) {
        const double n = ne * V;
        if (n < 1) {
            c.nume = poisson_sample(rng, n);
            c.w = 1.0;
        } else if (n < pf) {
            c.nume = randround(rng, n);
            c.w = 1.0;
        } else {
            c.nume = p;
            c.w = n / pf;
        }
        c.qf = q / ELEMENTARY_CHARGE + c.w * (double)c.nume / V;
    } else {
        const double a = ne * V / pf;
        c.w = (a > 1.0 || std::isnan(a)) ? a : 1.0;                 /* max(1, ...) */
        c.nume = poisson_sample(rng, ne * V / c.w);
        const double ni = ne + q / ELEMENTARY_CHARGE;
        const double b = std::fabs(ni) * V / pf;
        const double wi = (b > 1.0 || std::isnan(b)) ? b : 1.0;
        const int64_t numi = poisson_sample(rng, std::fabs(ni) * V / wi);
        const double sg = ni > 0 ? 1.0 : (ni < 0 ? -1.0 : ni);       /* sign(ni) */
        c.qf = sg * (double)numi * wi / V;
    }
    return c;
}

}  // namespace

extern "C" {

int64_t orc_init_from_density(int M, int N, double R, double L, const double* ne, const double* q, int method,
                              int64_t p, double fluid_threshold, uint64_t seed, int64_t cap, double* x, double* w,
                              double* s, double* qfd, double* ne_fluid) {
    const double dr = R / M, dz = L / N;
    int64_t n = 0;
    for (int j = 1; j <= N; ++j)
        for (int i = 1; i <= M; ++i) {
            const uint32_t c = (uint32_t)((i - 1) + (int64_t)(j - 1) * M);
            const double rc = ((double)(i - 1) + 0.5) * dr;
            const double V = 2.0 * M_PI * rc * dr * dz;                  /* dV(grid, i), grid.jl:76 */
            const double nec = ne[c], qc = q[c];
            if (nec > fluid_threshold) {
                ne_fluid[(i + 1) + (int64_t)(j + 1) * (M + 4)] = nec;
                qfd[i + (int64_t)j * (M + 2)] = qc / ELEMENTARY_CHARGE + nec;
                continue;
            }
            Stream rng(seed, c, 0u, ORC_TAG_DENSITY);
            const CellSample cs = nsample(method, p, nec, qc, V, rng);
            qfd[i + (int64_t)j * (M + 2)] = cs.qf;
            for (int64_t k = 0; k < cs.nume; ++k) {
                if (n >= cap) return -1;                                   /* "Particle limit reached" */
                Stream pr(seed, c, (uint32_t)k, ORC_TAG_DENSITY | ORC_TAG_DENSITY_PARTICLE);
                const double r = dr * pr.next() + (double)(i - 1) * dr;   /* rf[i] = (i - 1) dr */
                const double z = dz * pr.next() + (double)(j - 1) * dz;
                const double phi = 2.0 * M_PI * pr.next();
                x[3 * n] = r * std::cos(phi);
                x[3 * n + 1] = r * std::sin(phi);
                x[3 * n + 2] = z;
                w[n] = cs.w;
                s[n] = -std::log(pr.next());                               /* nextcoll() */
                ++n;
            }
        }
    return n;
}

}  // extern "C"
