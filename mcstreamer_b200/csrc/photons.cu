// photons.cu -- MCStreamer's photon population (PhotonState, JuMC/src/photon.jl:11-18) and
// advance! over electrons and photons (JuMC/src/mixed_population.jl:24-54).
//
// advance!(mpopl, efield, dt, tracker) runs the electrons first.  Their photo-emission
// collisions (electron.jl:141-144) add photons (collisions.jl:125-141), which the photon
// loop then advances too.  Photons fly straight (photon.jl:54-56) with null collisions at
// numax (ZhelezniakCollisions, photon.jl:27-43).  A real one (nu > xi, nu the photon's own
// absorption rate) is photo-ionization (photon.jl:45-51): the tracker adds +w
// (gridfields.jl:219-222), the photon goes and an electron at rest takes its place.
//
// Parents emit in parallel, and the populations grow in serial parent order, as the oracle
// grows them.
//   * Photons.  The step kernel records each photo-emission event with the count of photons
//     its parent emitted before it in the step, and the parent's total.  An exclusive scan
//     of the totals places every photon, and k_photon_emit makes it from its own counter-based
//     random block.
//   * Electrons.  k_photon_step records each photo-ionization the same way, and
//     k_ion_scatter appends the electrons after the electron step's own secondaries.
//
// Built with -fmad=false, so the flights x + t v are the oracle's unfused arithmetic.
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <vector>

#include "../../include/mcs.h"
#include "host_util.h"
#include "mcs_device.cuh"
#include "mcs_internal.h"
#include "pop_ops.h"
#include "scan.cuh"
#include "step.cuh"

namespace mcs {
namespace {

constexpr double kSpeedOfLight = 299792458.0;   // co.c (Constants/src/Constants.jl:39)

struct PhotonView {
    double* x[3];
    double* v[3];
    double* nu;
    double* w;
    double* s;
    uint8_t* act;
};

// One photo-ionization: electron k (in collision order) of photon `slot`.
struct IonEvent {
    double x, y, z, w, s;
    uint32_t slot, k, act;
};

__device__ __forceinline__ long long gid() { return (long long)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ long long gstride() { return (long long)gridDim.x * blockDim.x; }


// ---------------------------------------------------------------------------------------
// Photons from the recorded photo-emission events: photon p of event (slot, jev) takes
// block {slot, step, p, TAG_PHOTON_DRAW | jev}: randsphere() from words 0, 1, the log-nu
// fraction from word 2 and nextcoll() from word 3 (collisions.jl:134-138).
// ---------------------------------------------------------------------------------------
__global__ void k_photon_emit(PhotonView P, const PhotoEvent* ev, const uint32_t* nev_dev, uint32_t ev_cap,
                              const unsigned long long* pbase, long long n0, long long cap, TableView tab,
                              unsigned long long seed, uint32_t step, uint32_t slot_base, uint32_t* status) {
    const uint32_t nev = min(*nev_dev, ev_cap);
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    for (long long e = gid(); e < nev; e += gstride()) {
        const PhotoEvent E = ev[e];
        const double lmin = tab.pe_lmin[E.row], lmax = tab.pe_lmax[E.row];
        const long long d0 = n0 + (long long)pbase[E.slot] + E.poff;
        for (uint32_t p = 0; p < E.nphot; ++p) {
            const long long d = d0 + p;
            if (d >= cap) {
                atomicOr(status, ST_CAPACITY);
                break;
            }
            const U4 b = philox10(U4{E.slot + slot_base, step, p, TAG_PHOTON_DRAW | E.jev}, k0, k1);
            double ux, uy, uz;
            M<double>::dir(uni64(b.x), uni64(b.y), ux, uy, uz);
            P.x[0][d] = E.x; P.x[1][d] = E.y; P.x[2][d] = E.z;
            P.v[0][d] = ux * kSpeedOfLight; P.v[1][d] = uy * kSpeedOfLight; P.v[2][d] = uz * kSpeedOfLight;
            P.nu[d] = exp(lmin + (lmax - lmin) * uni64(b.z));
            P.w[d] = tab.pe_pw;
            P.s[d] = -log(uni64(b.w));
            P.act[d] = (uint8_t)E.act;
        }
    }
}

// ---------------------------------------------------------------------------------------
// advance! of the photons: the sub-step loop of mixed_population.jl:31-51 with
// advance_free = x + t v and do_one_collision! of the ZhelezniakCollisions table.  Event j of
// photon i draws block {i, step, j, TAG_PHOTON}: xi (x), the photon's new s (y), the new
// electron's nextcoll() (z).  A removed photon keeps sub-stepping, as in the reference.
// ---------------------------------------------------------------------------------------
__global__ void k_photon_step(PhotonView P, long long n_entry, double numax, double dt, unsigned long long seed,
                              uint32_t step, GridView tg, IonEvent* iev, uint32_t* iev_count, uint32_t iev_cap,
                              uint32_t* per_slot, uint32_t* status) {
    const bool tracking = tg.type != 0 && tg.qfixed != nullptr;
    for (long long i = gid(); i < n_entry; i += gstride()) {
        uint32_t k = 0;
        if (P.act[i]) {
            Event rng;
            rng.init(seed, (uint32_t)i, step, TAG_PHOTON);
            double x = P.x[0][i], y = P.x[1][i], z = P.x[2][i];
            const double vx = P.v[0][i], vy = P.v[1][i], vz = P.v[2][i];
            const double nu = P.nu[i], w = P.w[i];
            double s = P.s[i];
            uint32_t act = 1;
            double trem = dt;
            while (trem > 0) {
                const double tn = s / numax;
                double t;
                bool collides;
                if (trem > tn) { t = tn; collides = true; }
                else { t = trem; collides = false; s -= t * numax; }
                x = x + t * vx;
                y = y + t * vy;
                z = z + t * vz;
                if (collides) {
                    rng.begin();
                    const double xi = uni64(rng.b.x) * numax;
                    if (nu > xi) {
                        if (tracking) track_abs(tg, x, y, z, w, status);
                        const uint32_t e = atomicAdd(iev_count, 1u);
                        if (e < iev_cap) {
                            IonEvent E;
                            E.x = x; E.y = y; E.z = z; E.w = w;
                            E.s = -log(uni64(rng.b.z));
                            E.slot = (uint32_t)i; E.k = k; E.act = act;
                            iev[e] = E;
                        } else {
                            atomicOr(status, ST_OVERFLOW);
                        }
                        ++k;
                        act = 0;
                    }
                    s = -log(uni64(rng.b.y));
                }
                trem -= t;
            }
            P.x[0][i] = x; P.x[1][i] = y; P.x[2][i] = z;
            P.s[i] = s;
            if (!act) P.act[i] = 0;
        }
        per_slot[i] = k;
    }
}

// The photo-ionization electrons, appended after `n0` in serial photon order: at rest, the
// photon's position and weight, their own nextcoll() and the photon's active flag
// (photon.jl:45-51).
template <typename T>
__global__ void k_ion_scatter(PopView<T> E, const IonEvent* ev, const uint32_t* nev_dev, uint32_t ev_cap,
                              const unsigned long long* ibase, long long n0, uint32_t* status) {
    const uint32_t nev = min(*nev_dev, ev_cap);
    for (long long e = gid(); e < nev; e += gstride()) {
        const IonEvent V = ev[e];
        const long long d = n0 + (long long)ibase[V.slot] + V.k;
        if (d >= E.cap) {
            atomicOr(status, ST_CAPACITY);
            continue;
        }
        E.f[0][d] = (T)V.x; E.f[1][d] = (T)V.y; E.f[2][d] = (T)V.z;
        E.f[3][d] = (T)0; E.f[4][d] = (T)0; E.f[5][d] = (T)0;
        E.f[6][d] = (T)V.w; E.f[7][d] = (T)V.s;
        E.act[d] = (uint8_t)V.act;
    }
}

__global__ void k_set_count(long long* n, long long v) { *n = v; }

constexpr int kDiagBlocks = 592, kDiagThreads = 256;

// actives(photons) and weight(photons) (JuMC/src/population.jl:114-131): per-block partials
// over a fixed grid, then one block sums them in a fixed order, so the totals do not depend
// on timing.
__device__ __forceinline__ void block_sum2(double& a, double& b, double* sh) {
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { sh[2 * warp] = a; sh[2 * warp + 1] = b; }
    __syncthreads();
    if (warp == 0) {
        a = lane < (int)(blockDim.x >> 5) ? sh[2 * lane] : 0.0;
        b = lane < (int)(blockDim.x >> 5) ? sh[2 * lane + 1] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
    }
}

__global__ void __launch_bounds__(kDiagThreads) k_photon_sums(const double* __restrict__ w,
                                                              const uint8_t* __restrict__ act, long long n,
                                                              double* __restrict__ part) {
    __shared__ double sh[2 * (kDiagThreads / 32)];
    double cnt = 0.0, wt = 0.0;
    for (long long i = blockIdx.x * (long long)kDiagThreads + threadIdx.x; i < n;
         i += (long long)gridDim.x * kDiagThreads)
        if (act[i]) { cnt += 1.0; wt += w[i]; }
    block_sum2(cnt, wt, sh);
    if (threadIdx.x == 0) { part[2 * blockIdx.x] = cnt; part[2 * blockIdx.x + 1] = wt; }
}

__global__ void __launch_bounds__(kDiagThreads) k_photon_sums_final(double* part, int nb) {
    __shared__ double sh[2 * (kDiagThreads / 32)];
    double cnt = 0.0, wt = 0.0;
    for (int b = threadIdx.x; b < nb; b += kDiagThreads) { cnt += part[2 * b]; wt += part[2 * b + 1]; }
    block_sum2(cnt, wt, sh);
    if (threadIdx.x == 0) { part[2 * nb] = cnt; part[2 * nb + 1] = wt; }
}

// repack! of the photon population (JuMC/src/population.jl:191-215): with A actives, the
// k-th hole below A (ascending) takes the k-th active at or above A counted from the end.
// From the exclusive scan base[] of the active flags: a hole i < A has rank i - base[i], an
// active i >= A has rank A - 1 - base[i].
__global__ void k_photon_flags(const uint8_t* act, long long n, uint32_t* flags) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        flags[i] = act[i] ? 1u : 0u;
}

__global__ void k_photon_holes(const uint8_t* act, const unsigned long long* base, const unsigned long long* total,
                               uint32_t* hole_at) {
    const long long A = (long long)*total;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < A; i += (long long)gridDim.x * blockDim.x)
        if (!act[i]) hole_at[i - (long long)base[i]] = (uint32_t)i;
}

struct PhotonRaw {
    double* f[9];
    uint8_t* act;
};

__global__ void k_photon_fill(PhotonRaw P, const unsigned long long* base, const unsigned long long* total, long long n,
                              const uint32_t* hole_at) {
    const long long A = (long long)*total;
    for (long long i = A + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        if (!P.act[i]) continue;
        const long long h = hole_at[A - 1 - (long long)base[i]];
#pragma unroll
        for (int q = 0; q < 9; ++q) P.f[q][h] = P.f[q][i];
        P.act[h] = 1;
    }
}

}  // namespace
}  // namespace mcs

using namespace mcs;

struct mcs_photons {
    mcs_ctx* ctx = nullptr;
    long long cap = 0, n = 0;
    double numax = 0.0;
    unsigned long long seed = 0;
    uint32_t step = 0;
    double* d_f[9] = {};          // x, y, z, vx, vy, vz, nu, w, s
    uint8_t* d_act = nullptr;
    // work buffers: photo-emission events (room: cap photons) and per-electron-slot
    // photon counts; photo-ionization events and per-photon electron counts
    PhotoEvent* d_pev = nullptr;
    uint32_t* d_pslot = nullptr;
    long long pslot_cap = 0;
    IonEvent* d_iev = nullptr;
    long long iev_cap = 0;
    uint32_t* d_islot = nullptr;
    unsigned long long* d_base = nullptr;   // scan output (max of both slot counts)
    long long base_cap = 0;
    unsigned long long* d_sums = nullptr;
    long long sums_cap = 0;
    uint32_t* d_counts = nullptr;           // [0] photo-emission events, [1] photo-ionizations
    unsigned long long* d_total = nullptr;
    unsigned long long* h_total = nullptr;  // pinned
    double* d_diag = nullptr;               // per-block (count, weight) partials, then the totals
    cudaEvent_t ev[4] = {};                 // around k_photon_emit and k_photon_step
    float emit_ms = 0.0f, step_ms = 0.0f;   // of the last mixed advance
    long long last_emitted = 0, last_entry = 0;
};

namespace {

PhotonView photon_view(mcs_photons* ph) {
    PhotonView v;
    for (int q = 0; q < 3; ++q) { v.x[q] = ph->d_f[q]; v.v[q] = ph->d_f[3 + q]; }
    v.nu = ph->d_f[6];
    v.w = ph->d_f[7];
    v.s = ph->d_f[8];
    v.act = ph->d_act;
    return v;
}

template <typename T>
int dalloc_n(mcs_ctx* c, T** p, size_t count) {
    void* d = nullptr;
    if (cudaMalloc(&d, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        return set_err(c, MCS_ERR_NOMEM, "photons: device allocation failed");
    }
    *p = static_cast<T*>(d);
    return MCS_OK;
}

template <typename T>
int grow(mcs_ctx* c, T** p, long long* have, long long need) {
    if (*have >= need) return MCS_OK;
    cudaFree(*p);
    *p = nullptr;
    *have = 0;
    if (int e = dalloc_n(c, p, (size_t)need)) return e;
    *have = need;
    return MCS_OK;
}

int blocks_for(mcs_ctx* c, long long n, int block) {
    const long long b = (n + block - 1) / block;
    return (int)std::max(1LL, std::min(b, (long long)c->num_sms * 16));
}

// bases[0..n) = exclusive scan of counts[0..n); the total lands in ph->h_total after a sync.
int scan_counts(mcs_photons* ph, const uint32_t* counts, long long n, cudaStream_t st) {
    mcs_ctx* c = ph->ctx;
    MCS_CK(c, cudaStreamSynchronize(st));   // no queued kernel still reads a buffer regrown here
    const long long nb = std::max(1LL, (n + kScanTile - 1) / kScanTile);
    if (int e = grow(c, &ph->d_sums, &ph->sums_cap, nb)) return e;
    if (int e = grow(c, &ph->d_base, &ph->base_cap, std::max(1LL, n))) return e;
    k_scan_sums<<<(int)nb, kScanThreads, 0, st>>>(counts, n, ph->d_sums);
    k_scan_top<<<1, kScanThreads, 0, st>>>(ph->d_sums, (int)nb, ph->d_total);
    k_scan_apply<<<(int)nb, kScanThreads, 0, st>>>(counts, n, ph->d_sums, ph->d_base);
    MCS_CK_LAUNCH(c);
    MCS_CK(c, cudaMemcpyAsync(ph->h_total, ph->d_total, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    MCS_CK(c, cudaStreamSynchronize(st));
    return MCS_OK;
}

// The population's current count (after the work queued on the context's stream).
long long pop_count(mcs_pop* p, int* err) {
    long long n = 0;
    cudaStream_t st = p->ctx->stream;
    *err = (cudaMemcpyAsync(&n, p->d_n + p->cur, sizeof(n), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
            cudaStreamSynchronize(st) == cudaSuccess)
               ? MCS_OK
               : MCS_ERR_CUDA;
    return n;
}

// The photon half of advance! (photons, then their electrons into e).
int photon_half(mcs_photons* ph, mcs_pop* e, double dt, mcs_grid* tracker) {
    mcs_ctx* c = ph->ctx;
    cudaStream_t st = c->stream;
    const long long n_entry = ph->n;
    MCS_CK(c, cudaStreamSynchronize(st));   // k_photon_emit may still read the scan buffers
    if (int er = grow(c, &ph->d_iev, &ph->iev_cap, std::max(1LL, e->cap))) return er;
    MCS_CK(c, cudaMemsetAsync(ph->d_counts + 1, 0, sizeof(uint32_t), st));
    ph->last_entry = n_entry;
    ph->step_ms = 0.0f;
    if (n_entry > 0) {
        cudaEventRecord(ph->ev[2], st);
        k_photon_step<<<blocks_for(c, n_entry, 256), 256, 0, st>>>(
            photon_view(ph), n_entry, ph->numax, dt, ph->seed, ph->step, grid_view(tracker), ph->d_iev,
            ph->d_counts + 1, (uint32_t)std::min<long long>(ph->iev_cap, 0xffffffffLL), ph->d_islot, c->d_status);
        cudaEventRecord(ph->ev[3], st);
        MCS_CK_LAUNCH(c);
        if (int er = scan_counts(ph, ph->d_islot, n_entry, st)) return er;
        cudaEventElapsedTime(&ph->step_ms, ph->ev[2], ph->ev[3]);
        const unsigned long long added = *ph->h_total;
        if (added > 0) {
            int er = MCS_OK;
            const long long n0 = pop_count(e, &er);
            if (er) return set_err(c, er, "photons: count read failed");
            const int blocks = blocks_for(c, (long long)added, 256);
            if (e->precision == MCS_FP32)
                k_ion_scatter<float><<<blocks, 256, 0, st>>>(pop_view<float>(e), ph->d_iev, ph->d_counts + 1,
                                                             (uint32_t)std::min<long long>(ph->iev_cap, 0xffffffffLL),
                                                             ph->d_base, n0, c->d_status);
            else
                k_ion_scatter<double><<<blocks, 256, 0, st>>>(pop_view<double>(e), ph->d_iev, ph->d_counts + 1,
                                                              (uint32_t)std::min<long long>(ph->iev_cap, 0xffffffffLL),
                                                              ph->d_base, n0, c->d_status);
            k_set_count<<<1, 1, 0, st>>>(e->d_n + e->cur, std::min(n0 + (long long)added, e->cap));
            MCS_CK_LAUNCH(c);
        }
    }
    ph->step += 1;
    return MCS_OK;
}

bool has_photo_rows(const mcs_table* t) {
    for (int j = 0; j < t->v.nrows; ++j)
        if (t->v.kind[j] == K_PHOTOEMISSION) return true;
    return false;
}

}  // namespace

extern "C" {

MCS_API int mcs_photons_create(mcs_ctx* c, int64_t capacity, double numax, uint64_t seed, mcs_photons** out) {
    if (!c || !out || capacity < 1 || !(numax > 0)) return MCS_ERR_ARG;
    *out = nullptr;
    MCS_CK(c, cudaSetDevice(c->device));
    mcs_photons* ph = new (std::nothrow) mcs_photons();
    if (!ph) return MCS_ERR_NOMEM;
    ph->ctx = c;
    ph->cap = capacity;
    ph->numax = numax;
    ph->seed = seed;
    int e = MCS_OK;
    for (int q = 0; q < 9 && !e; ++q) e = dalloc_n(c, &ph->d_f[q], (size_t)capacity);
    if (!e) e = dalloc_n(c, &ph->d_act, (size_t)capacity);
    if (!e) e = dalloc_n(c, &ph->d_pev, (size_t)capacity);
    if (!e) e = dalloc_n(c, &ph->d_islot, (size_t)capacity);
    if (!e) e = dalloc_n(c, &ph->d_counts, 2);
    if (!e) e = dalloc_n(c, &ph->d_total, 1);
    if (!e) e = dalloc_n(c, &ph->d_diag, (size_t)(2 * kDiagBlocks + 2));
    if (!e && cudaMallocHost(&ph->h_total, sizeof(unsigned long long)) != cudaSuccess)
        e = set_err(c, MCS_ERR_NOMEM, "photons: pinned allocation failed");
    if (!e && cudaMemset(ph->d_act, 0, (size_t)capacity) != cudaSuccess) e = MCS_ERR_CUDA;
    for (int q = 0; q < 4 && !e; ++q)
        if (cudaEventCreate(&ph->ev[q]) != cudaSuccess) e = MCS_ERR_CUDA;
    if (e) {
        mcs_photons_destroy(ph);
        return e;
    }
    *out = ph;
    return MCS_OK;
}

MCS_API int mcs_photons_destroy(mcs_photons* ph) {
    if (!ph) return MCS_ERR_ARG;
    if (ph->ctx && ph->ctx->stream) cudaStreamSynchronize(ph->ctx->stream);
    for (double* f : ph->d_f) cudaFree(f);
    cudaFree(ph->d_act);
    cudaFree(ph->d_pev);
    cudaFree(ph->d_pslot);
    cudaFree(ph->d_iev);
    cudaFree(ph->d_islot);
    cudaFree(ph->d_base);
    cudaFree(ph->d_sums);
    cudaFree(ph->d_counts);
    cudaFree(ph->d_total);
    cudaFree(ph->d_diag);
    if (ph->h_total) cudaFreeHost(ph->h_total);
    for (cudaEvent_t v : ph->ev)
        if (v) cudaEventDestroy(v);
    delete ph;
    return MCS_OK;
}

// Host arrays in the Julia layout: x, v 3 doubles per photon (interleaved), nu, w, s one
// double each, active one byte.
MCS_API int mcs_photons_upload(mcs_photons* ph, const double* x, const double* v, const double* nu,
                               const double* w, const double* s, const uint8_t* active, int64_t n) {
    if (!ph || n < 0 || n > ph->cap || (n > 0 && (!x || !v || !nu || !w || !s || !active))) return MCS_ERR_ARG;
    mcs_ctx* c = ph->ctx;
    MCS_CK(c, cudaSetDevice(c->device));
    MCS_CK(c, cudaStreamSynchronize(c->stream));
    std::vector<double> tmp((size_t)n);
    for (int q = 0; q < 3; ++q) {
        for (int64_t i = 0; i < n; ++i) tmp[i] = x[3 * i + q];
        MCS_CK(c, cudaMemcpy(ph->d_f[q], tmp.data(), n * sizeof(double), cudaMemcpyHostToDevice));
        for (int64_t i = 0; i < n; ++i) tmp[i] = v[3 * i + q];
        MCS_CK(c, cudaMemcpy(ph->d_f[3 + q], tmp.data(), n * sizeof(double), cudaMemcpyHostToDevice));
    }
    MCS_CK(c, cudaMemcpy(ph->d_f[6], nu, n * sizeof(double), cudaMemcpyHostToDevice));
    MCS_CK(c, cudaMemcpy(ph->d_f[7], w, n * sizeof(double), cudaMemcpyHostToDevice));
    MCS_CK(c, cudaMemcpy(ph->d_f[8], s, n * sizeof(double), cudaMemcpyHostToDevice));
    MCS_CK(c, cudaMemcpy(ph->d_act, active, (size_t)n, cudaMemcpyHostToDevice));
    ph->n = n;
    return MCS_OK;
}

MCS_API int mcs_photons_download(mcs_photons* ph, double* x, double* v, double* nu, double* w, double* s,
                                 uint8_t* active, int64_t capacity, int64_t* n_out) {
    if (!ph || !n_out) return MCS_ERR_ARG;
    mcs_ctx* c = ph->ctx;
    MCS_CK(c, cudaSetDevice(c->device));
    const int st = sync_status(c);
    const int64_t n = ph->n;
    *n_out = n;
    if (n > capacity) return set_err(c, MCS_ERR_ARG, "photons: host arrays too small");
    if (n > 0 && (!x || !v || !nu || !w || !s || !active)) return MCS_ERR_ARG;
    std::vector<double> tmp((size_t)n);
    for (int q = 0; q < 3; ++q) {
        MCS_CK(c, cudaMemcpy(tmp.data(), ph->d_f[q], n * sizeof(double), cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < n; ++i) x[3 * i + q] = tmp[i];
        MCS_CK(c, cudaMemcpy(tmp.data(), ph->d_f[3 + q], n * sizeof(double), cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < n; ++i) v[3 * i + q] = tmp[i];
    }
    MCS_CK(c, cudaMemcpy(nu, ph->d_f[6], n * sizeof(double), cudaMemcpyDeviceToHost));
    MCS_CK(c, cudaMemcpy(w, ph->d_f[7], n * sizeof(double), cudaMemcpyDeviceToHost));
    MCS_CK(c, cudaMemcpy(s, ph->d_f[8], n * sizeof(double), cudaMemcpyDeviceToHost));
    MCS_CK(c, cudaMemcpy(active, ph->d_act, (size_t)n, cudaMemcpyDeviceToHost));
    return st;
}

// dst <- src on the device (the first src->n photons and the count).
MCS_API int mcs_photons_copy(mcs_photons* dst, const mcs_photons* src) {
    if (!dst || !src || dst->ctx != src->ctx) return MCS_ERR_ARG;
    mcs_ctx* c = dst->ctx;
    if (src->n > dst->cap) return set_err(c, MCS_ERR_CAPACITY, "photons: destination too small");
    MCS_CK(c, cudaSetDevice(c->device));
    const size_t n = (size_t)src->n;
    for (int q = 0; q < 9; ++q)
        MCS_CK(c, cudaMemcpyAsync(dst->d_f[q], src->d_f[q], n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    MCS_CK(c, cudaMemcpyAsync(dst->d_act, src->d_act, n, cudaMemcpyDeviceToDevice, c->stream));
    dst->n = src->n;
    dst->step = src->step;
    return MCS_OK;
}

// Device times (CUDA events on the context's stream) of the last mixed advance's photon
// kernels, with the photons they handled: k_photon_emit (emitted) and k_photon_step (entry
// count of the photon half).
MCS_API int mcs_photons_last_timing(mcs_photons* ph, float* emit_ms, int64_t* emitted, float* step_ms,
                                    int64_t* stepped) {
    if (!ph) return MCS_ERR_ARG;
    if (ph->last_emitted > 0) cudaEventElapsedTime(&ph->emit_ms, ph->ev[0], ph->ev[1]);
    if (emit_ms) *emit_ms = ph->emit_ms;
    if (emitted) *emitted = ph->last_emitted;
    if (step_ms) *step_ms = ph->step_ms;
    if (stepped) *stepped = ph->last_entry;
    return MCS_OK;
}

MCS_API int mcs_photons_count(mcs_photons* ph, int64_t* n) {
    if (!ph || !n) return MCS_ERR_ARG;
    *n = ph->n;
    return MCS_OK;
}

MCS_API int mcs_photons_repack(mcs_photons* ph) {
    if (!ph) return MCS_ERR_ARG;
    mcs_ctx* c = ph->ctx;
    if (ph->n == 0) return MCS_OK;
    MCS_CK(c, cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    const long long n = ph->n;
    const int g = blocks_for(c, n, 256);
    k_photon_flags<<<g, 256, 0, st>>>(ph->d_act, n, ph->d_islot);
    MCS_CK_LAUNCH(c);
    if (int e = scan_counts(ph, ph->d_islot, n, st)) return e;   // bases in d_base, A in *h_total
    const long long A = (long long)*ph->h_total;
    if (A < n) {
        if (int e = grow(c, &ph->d_pslot, &ph->pslot_cap, std::max(1LL, A))) return e;
        k_photon_holes<<<g, 256, 0, st>>>(ph->d_act, ph->d_base, ph->d_total, ph->d_pslot);
        PhotonRaw R;
        for (int q = 0; q < 9; ++q) R.f[q] = ph->d_f[q];
        R.act = ph->d_act;
        k_photon_fill<<<g, 256, 0, st>>>(R, ph->d_base, ph->d_total, n, ph->d_pslot);
        MCS_CK_LAUNCH(c);
    }
    ph->n = A;
    return sync_status(c);
}

MCS_API int mcs_photons_moments(mcs_photons* ph, double* out) {
    if (!ph || !out) return MCS_ERR_ARG;
    mcs_ctx* c = ph->ctx;
    out[0] = out[1] = 0.0;
    if (ph->n == 0) return MCS_OK;
    MCS_CK(c, cudaSetDevice(c->device));
    const int nb = (int)std::min<long long>(kDiagBlocks, (ph->n + kDiagThreads - 1) / kDiagThreads);
    k_photon_sums<<<nb, kDiagThreads, 0, c->stream>>>(ph->d_f[7], ph->d_act, ph->n, ph->d_diag);
    k_photon_sums_final<<<1, kDiagThreads, 0, c->stream>>>(ph->d_diag, nb);
    MCS_CK(c, cudaGetLastError());
    MCS_CK(c, cudaMemcpyAsync(out, ph->d_diag + 2 * nb, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    MCS_CK(c, cudaStreamSynchronize(c->stream));
    return MCS_OK;
}

MCS_API int mcs_table_set_photoemission(mcs_table* t, const double* log_numin, const double* log_numax,
                                        double photon_multiplier, double photon_weight) {
    if (!t || !log_numin || !log_numax || !(photon_multiplier > 0) || !(photon_weight > 0)) return MCS_ERR_ARG;
    TableView& v = t->v;
    for (int j = 0; j < v.nrows; ++j) {
        v.pe_lmin[j] = log_numin[j];
        v.pe_lmax[j] = log_numax[j];
    }
    v.pe_mult = photon_multiplier;
    v.pe_pw = photon_weight;
    v.has_pe = has_photo_rows(t) ? 1 : 0;
    return MCS_OK;
}

// advance!(mpopl, efield, dt, tracker) with an electron and a photon population.
MCS_API int mcs_advance_mixed(mcs_pop* e, mcs_photons* ph, const mcs_table* t, const mcs_field* f, double dt,
                              mcs_grid* tracker) {
    if (!e || !ph || !t || !f) return MCS_ERR_ARG;
    mcs_ctx* c = e->ctx;
    if (ph->ctx != c) return set_err(c, MCS_ERR_ARG, "electrons and photons on different contexts");
    if (!(dt >= 0)) return set_err(c, MCS_ERR_ARG, "dt must be >= 0");
    if (f->type == FIELD_GRID && !f->grid) return MCS_ERR_ARG;
    if (e->cells) return set_err(c, MCS_ERR_UNSUPPORTED, "photo-emission needs absolute positions (no cell layout)");
    if (has_photo_rows(t) && !t->v.has_pe)
        return set_err(c, MCS_ERR_ARG, "photo-emission rows without mcs_table_set_photoemission");
    MCS_CK(c, cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    int er = MCS_OK;
    const long long ne0 = pop_count(e, &er);
    if (er) return set_err(c, er, "photons: count read failed");
    if (int q = grow(c, &ph->d_pslot, &ph->pslot_cap, std::max(1LL, ne0))) return q;
    MCS_CK(c, cudaMemsetAsync(ph->d_counts, 0, sizeof(uint32_t), st));
    // the electrons, recording their photo-emission events
    e->photo.events = ph->d_pev;
    e->photo.count = ph->d_counts;
    e->photo.cap = (uint32_t)std::min<long long>(ph->cap, 0xffffffffLL);
    e->photo.per_slot = ph->d_pslot;
    const uint32_t estep = e->step, ebase = e->slot_base;
    int s1 = e->precision == MCS_FP32 ? launch_step_abs<float>(e, t, f, dt, tracker, log_slot(e))
                                      : launch_step_abs<double>(e, t, f, dt, tracker, log_slot(e));
    e->photo = PhotoOut{};
    if (s1) return s1;
    e->cur ^= 1;
    e->step += 1;
    // their photons, in serial parent order
    ph->emit_ms = 0.0f;
    ph->last_emitted = 0;
    if (ne0 > 0) {
        if (int q = scan_counts(ph, ph->d_pslot, ne0, st)) return q;
        const unsigned long long added = *ph->h_total;
        if (added > 0) {
            cudaEventRecord(ph->ev[0], st);
            k_photon_emit<<<blocks_for(c, (long long)added, 256), 256, 0, st>>>(
                photon_view(ph), ph->d_pev, ph->d_counts, (uint32_t)std::min<long long>(ph->cap, 0xffffffffLL),
                ph->d_base, ph->n, ph->cap, t->v, e->seed, estep, ebase, c->d_status);
            cudaEventRecord(ph->ev[1], st);
            MCS_CK_LAUNCH(c);
            ph->n = std::min(ph->n + (long long)added, ph->cap);
            ph->last_emitted = (long long)added;
        }
    }
    // every photon, the new ones included
    if (int q = photon_half(ph, e, dt, tracker)) return q;
    return sync_status(c);
}

MCS_API int mcs_photon_advance(mcs_photons* ph, mcs_pop* e, double dt, mcs_grid* tracker) {
    if (!ph || !e) return MCS_ERR_ARG;
    mcs_ctx* c = ph->ctx;
    if (!(dt >= 0)) return set_err(c, MCS_ERR_ARG, "dt must be >= 0");
    if (e->cells) return set_err(c, MCS_ERR_UNSUPPORTED, "photo-ionization needs absolute positions");
    MCS_CK(c, cudaSetDevice(c->device));
    if (int q = photon_half(ph, e, dt, tracker)) return q;
    return sync_status(c);
}

}  // extern "C"
