// host_step.cu -- advance! + density! of a population that lives in host memory (the Julia
// StructArray itself), with the transfers hidden behind the step.
//
// The population is cut into chunks.  Chunk c's upload (H2D), its step and its download
// (D2H) run on three streams, so the upload of chunk c+1 and the download of chunk c-1 overlap
// the step of chunk c, and the H2D and D2H directions of the host link run at the same time.
// Each chunk is stepped by the fused mesh step with its random streams keyed by the
// particles' global slots (slot_base), the int64 deposits are order-independent sums, and
// each chunk's secondaries are written after all earlier chunks' secondaries, so the result
// is the same as uploading the whole population, one step, and downloading it.
#include <algorithm>
#include <vector>

#include "host_util.h"
#include "pop_ops.h"

namespace mcs {

// Workspace of mcs_advance_deposit_host, kept in the population between calls and grown
// when a call needs more: two Julia-layout staging buffers each way, pinned per-chunk
// counts and weight flags, the copy streams and per-chunk events; and the bytes the last
// call copied each way.
struct HostStepBuffers {
    double* in[2] = {nullptr, nullptr};    // a chunk's input
    double* out[2] = {nullptr, nullptr};   // a chunk's output (the chunk and its secondaries)
    long long* cnt = nullptr;              // pinned: particles after each chunk's step
    unsigned int* wl = nullptr;            // pinned: 1 when a chunk's weights changed on upload
    unsigned int* d_wl = nullptr;          // the flags on the device
    size_t in_bytes = 0, out_bytes = 0;
    int nch = 0;
    long long h2d = 0, d2h = 0;            // bytes copied by the last call
    cudaStream_t s_in = nullptr, s_out = nullptr;
    std::vector<cudaEvent_t> ev;
    ~HostStepBuffers() {
        for (int q = 0; q < 2; ++q) { cudaFree(in[q]); cudaFree(out[q]); }
        if (cnt) cudaFreeHost(cnt);
        if (wl) cudaFreeHost(wl);
        cudaFree(d_wl);
        if (s_in) cudaStreamDestroy(s_in);
        if (s_out) cudaStreamDestroy(s_out);
        for (auto e : ev) cudaEventDestroy(e);
    }
};

void free_host_step(HostStepBuffers* b) { delete b; }

namespace {

__global__ void k_set_count(long long* p, long long v) { *p = v; }

int ensure_host_step(mcs_pop* p, size_t in_bytes, size_t out_bytes, int nch) {
    mcs_ctx* c = p->ctx;
    if (!p->host_step) p->host_step = new HostStepBuffers();
    HostStepBuffers& B = *p->host_step;
    for (int q = 0; q < 2; ++q) {
        if (B.in_bytes < in_bytes) {
            cudaFree(B.in[q]);
            B.in[q] = nullptr;
            if (cudaMalloc(&B.in[q], in_bytes) != cudaSuccess) return set_err(c, MCS_ERR_NOMEM, "host-step staging");
        }
        if (B.out_bytes < out_bytes) {
            cudaFree(B.out[q]);
            B.out[q] = nullptr;
            if (cudaMalloc(&B.out[q], out_bytes) != cudaSuccess) return set_err(c, MCS_ERR_NOMEM, "host-step staging");
        }
    }
    B.in_bytes = std::max(B.in_bytes, in_bytes);
    B.out_bytes = std::max(B.out_bytes, out_bytes);
    if (B.nch < nch) {
        if (B.cnt) cudaFreeHost(B.cnt);
        if (B.wl) cudaFreeHost(B.wl);
        cudaFree(B.d_wl);
        B.cnt = nullptr;
        B.wl = nullptr;
        B.d_wl = nullptr;
        if (cudaHostAlloc(&B.cnt, sizeof(long long) * nch, cudaHostAllocDefault) != cudaSuccess ||
            cudaHostAlloc(&B.wl, sizeof(unsigned int) * nch, cudaHostAllocDefault) != cudaSuccess ||
            cudaMalloc(&B.d_wl, sizeof(unsigned int) * nch) != cudaSuccess)
            return set_err(c, MCS_ERR_NOMEM, "host-step counts");
        while ((int)B.ev.size() < 3 * nch) {
            cudaEvent_t e;
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return MCS_ERR_CUDA;
            B.ev.push_back(e);
        }
        B.nch = nch;
    }
    if (!B.s_in && (cudaStreamCreateWithFlags(&B.s_in, cudaStreamNonBlocking) != cudaSuccess ||
                    cudaStreamCreateWithFlags(&B.s_out, cudaStreamNonBlocking) != cudaSuccess))
        return set_err(c, MCS_ERR_CUDA, "host-step streams");
    return MCS_OK;
}

// Julia layout of m particles in one buffer: x (3m), v (3m), w (m), s (m), active (m bytes).
constexpr long long kJuliaBytes = 8 * sizeof(double) + 1;   // one particle, 65 bytes
constexpr long long kJuliaBytesNoW = kJuliaBytes - (long long)sizeof(double);
struct JView {
    double *x, *v, *w, *s;
    uint8_t* a;
};
JView jview(double* base, long long m) {
    JView j;
    j.x = base;
    j.v = base + 3 * m;
    j.w = base + 6 * m;
    j.s = base + 7 * m;
    j.a = reinterpret_cast<uint8_t*>(base + 8 * m);
    return j;
}

}  // namespace
}  // namespace mcs

using namespace mcs;

extern "C" {

MCS_API int mcs_advance_deposit_host(mcs_pop* p, const mcs_table* t, const mcs_field* f, double dt, mcs_grid* tracker,
                                     mcs_grid* deposit, double val, double* x, double* v, double* w, double* s,
                                     uint8_t* active, int64_t* n_io, int64_t capacity, int chunks) {
    if (!p || !t || !f || !deposit || !x || !v || !w || !s || !active || !n_io || chunks < 1) return MCS_ERR_ARG;
    mcs_ctx* c = p->ctx;
    if (!p->cells || deposit != p->cells || f->type != FIELD_GRID || f->grid != p->cells ||
        (tracker && tracker != p->cells))
        return set_err(c, MCS_ERR_UNSUPPORTED, "fused step+deposit needs a cell-layout population on one mesh");
    const long long n0 = *n_io;
    if (n0 < 0 || n0 > capacity || !(dt >= 0)) return MCS_ERR_ARG;
    if (cudaSetDevice(c->device) != cudaSuccess) return MCS_ERR_CUDA;
    if (p->host_step) p->host_step->h2d = p->host_step->d2h = 0;
    if (n0 == 0) return MCS_OK;
    const long long chunk = (n0 + chunks - 1) / chunks;
    const int nch = (int)((n0 + chunk - 1) / chunk);
    // the device population holds one chunk and its secondaries
    if (chunk > p->cap) return set_err(c, MCS_ERR_CAPACITY, "a chunk does not fit the device population");
    if (int st = sync_status(c)) return st;

    const long long out_m = p->cap;   // a chunk plus the secondaries its step may append
    const size_t in_bytes = (size_t)chunk * 8 * sizeof(double) + (size_t)chunk;
    const size_t out_bytes = (size_t)out_m * 8 * sizeof(double) + (size_t)out_m;
    if (int r = ensure_host_step(p, in_bytes, out_bytes, nch)) return r;
    HostStepBuffers& B = *p->host_step;
    B.h2d = B.d2h = 0;
    // per chunk events: uploaded, stepped (staging_in free, outputs staged), downloaded
    auto ev_in = [&](int k) { return B.ev[3 * k]; };
    auto ev_comp = [&](int k) { return B.ev[3 * k + 1]; };
    auto ev_out = [&](int k) { return B.ev[3 * k + 2]; };

    const uint32_t step0 = p->step;
    long long sec_total = 0;
    int st = MCS_OK;

    auto enqueue_in = [&](int k) -> int {
        const long long a = (long long)k * chunk, m = std::min(chunk, n0 - a);
        const JView d = jview(B.in[k & 1], chunk);
        if (k >= 2) cudaStreamWaitEvent(B.s_in, ev_comp(k - 2), 0);   // staging_in[k&1] consumed
        cudaError_t e = cudaMemcpyAsync(d.x, x + 3 * a, 3 * m * sizeof(double), cudaMemcpyHostToDevice, B.s_in);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d.v, v + 3 * a, 3 * m * sizeof(double), cudaMemcpyHostToDevice, B.s_in);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d.w, w + a, m * sizeof(double), cudaMemcpyHostToDevice, B.s_in);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d.s, s + a, m * sizeof(double), cudaMemcpyHostToDevice, B.s_in);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d.a, active + a, (size_t)m, cudaMemcpyHostToDevice, B.s_in);
        if (e == cudaSuccess) e = cudaEventRecord(ev_in(k), B.s_in);
        B.h2d += m * kJuliaBytes;
        return e == cudaSuccess ? MCS_OK : set_err(c, MCS_ERR_CUDA, cudaGetErrorString(e));
    };
    auto enqueue_comp = [&](int k) -> int {
        const long long a = (long long)k * chunk, m = std::min(chunk, n0 - a);
        const JView d = jview(B.in[k & 1], chunk);
        const JView o = jview(B.out[k & 1], out_m);
        cudaStreamWaitEvent(c->stream, ev_in(k), 0);
        if (k >= 2) cudaStreamWaitEvent(c->stream, ev_out(k - 2), 0);   // staging_out[k&1] downloaded
        if (cudaMemsetAsync(B.d_wl + k, 0, sizeof(unsigned int), c->stream) != cudaSuccess)
            return set_err(c, MCS_ERR_CUDA, "host-step flag");
        if (int r = launch_upload(p, d.x, d.v, d.w, d.s, d.a, m, B.d_wl + k)) return r;
        k_set_count<<<1, 1, 0, c->stream>>>(p->d_n + p->cur, m);
        p->step = step0;
        p->slot_base = (uint32_t)a;
        const int r = p->precision == MCS_FP32 ? launch_step_mesh<float>(p, t, dt, tracker != nullptr, val, nullptr)
                                               : launch_step_mesh<double>(p, t, dt, tracker != nullptr, val, nullptr);
        p->slot_base = 0;
        if (r) return r;
        p->cur ^= 1;
        if (int r2 = launch_download(p, o.x, o.v, o.w, o.s, o.a)) return r2;
        cudaError_t e = cudaMemcpyAsync(B.cnt + k, p->d_n + p->cur, sizeof(long long), cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(B.wl + k, B.d_wl + k, sizeof(unsigned int), cudaMemcpyDeviceToHost, c->stream);
        B.d2h += sizeof(long long) + sizeof(unsigned int);
        if (e == cudaSuccess) e = cudaEventRecord(ev_comp(k), c->stream);
        return e == cudaSuccess ? MCS_OK : set_err(c, MCS_ERR_CUDA, cudaGetErrorString(e));
    };
    auto enqueue_out = [&](int k) -> int {
        // chunk k's stepped particles back in place, its secondaries after all earlier ones
        if (cudaEventSynchronize(ev_comp(k)) != cudaSuccess) return set_err(c, MCS_ERR_CUDA, "host-step wait");
        const long long a = (long long)k * chunk, m = std::min(chunk, n0 - a);
        const long long nsec = B.cnt[k] - m;
        const JView o = jview(B.out[k & 1], out_m);
        if (n0 + sec_total + nsec > capacity) return set_err(c, MCS_ERR_CAPACITY, "Maximum number of particles reached");
        cudaStreamWaitEvent(B.s_out, ev_comp(k), 0);
        const long long ds = n0 + sec_total;
        cudaError_t e = cudaSuccess;
        // The step never changes the weight of a particle it is given (its secondaries carry
        // their own), so the chunk's weights come back only when the upload rounded one.
        const struct { long long dst, src, cnt; bool w; } parts[2] = {{a, 0, m, B.wl[k] != 0u}, {ds, m, nsec, true}};
        for (const auto& q : parts) {
            if (q.cnt <= 0) continue;
            if (e == cudaSuccess) e = cudaMemcpyAsync(x + 3 * q.dst, o.x + 3 * q.src, 3 * q.cnt * sizeof(double),
                                                      cudaMemcpyDeviceToHost, B.s_out);
            if (e == cudaSuccess) e = cudaMemcpyAsync(v + 3 * q.dst, o.v + 3 * q.src, 3 * q.cnt * sizeof(double),
                                                      cudaMemcpyDeviceToHost, B.s_out);
            if (e == cudaSuccess && q.w) e = cudaMemcpyAsync(w + q.dst, o.w + q.src, q.cnt * sizeof(double),
                                                             cudaMemcpyDeviceToHost, B.s_out);
            if (e == cudaSuccess) e = cudaMemcpyAsync(s + q.dst, o.s + q.src, q.cnt * sizeof(double),
                                                      cudaMemcpyDeviceToHost, B.s_out);
            if (e == cudaSuccess) e = cudaMemcpyAsync(active + q.dst, o.a + q.src, (size_t)q.cnt,
                                                      cudaMemcpyDeviceToHost, B.s_out);
            B.d2h += q.cnt * (q.w ? kJuliaBytes : kJuliaBytesNoW);
        }
        if (e == cudaSuccess) e = cudaEventRecord(ev_out(k), B.s_out);
        sec_total += nsec;
        return e == cudaSuccess ? MCS_OK : set_err(c, MCS_ERR_CUDA, cudaGetErrorString(e));
    };

    // software pipeline: in(k+1) and comp(k+1) are queued before the host waits for comp(k)
    st = enqueue_in(0);
    if (!st) st = enqueue_comp(0);
    for (int k = 0; k < nch && !st; ++k) {
        if (k + 1 < nch) {
            st = enqueue_in(k + 1);
            if (!st) st = enqueue_comp(k + 1);
        }
        if (!st) st = enqueue_out(k);
    }
    cudaStreamSynchronize(B.s_in);
    cudaStreamSynchronize(B.s_out);
    cudaStreamSynchronize(c->stream);
    p->step = step0 + 1;
    if (st) return st;
    *n_io = n0 + sec_total;
    return sync_status(c);
}

MCS_API int mcs_pop_host_step_bytes(const mcs_pop* p, int64_t* h2d, int64_t* d2h) {
    if (!p || !h2d || !d2h) return MCS_ERR_ARG;
    *h2d = p->host_step ? p->host_step->h2d : 0;
    *d2h = p->host_step ? p->host_step->d2h : 0;
    return MCS_OK;
}

}  // extern "C"
