// api.cu -- the extern "C" entry points declared in include/mcs.h.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "host_util.h"
#include "pop_ops.h"
#include "step.cuh"

using namespace mcs;

namespace mcs {

int map_status(uint32_t st) {
    if (st & ST_UNSUPPORTED) return MCS_ERR_UNSUPPORTED;
    if (st & ST_TIMEOUT) return MCS_ERR_TIMEOUT;
    if (st & ST_CAPACITY) return MCS_ERR_CAPACITY;
    if (st & ST_OVERFLOW) return MCS_ERR_OVERFLOW;
    if (st & ST_ENERGY) return MCS_ERR_ENERGY_RANGE;
    if (st & ST_FIELD) return MCS_ERR_FIELD_TOO_HIGH;
    if (st & ST_NONFINITE) return MCS_ERR_NONFINITE;
    if (st & ST_UNIFORMS) return MCS_ERR_UNIFORMS;
    if (st & ST_CHARGE) return MCS_ERR_CHARGE_RANGE;
    return MCS_OK;
}

const char* status_text(int code) {
    switch (code) {
    case MCS_ERR_TIMEOUT: return "a bounded device-side wait gave up";
    case MCS_ERR_CAPACITY: return "Maximum number of particles reached";
    case MCS_ERR_OVERFLOW: return "a tile produced more secondaries than its staging holds";
    case MCS_ERR_ENERGY_RANGE: return "particle energy outside the collision table";
    case MCS_ERR_FIELD_TOO_HIGH: return "Too high electric field";
    case MCS_ERR_NONFINITE: return "non-finite particle state";
    case MCS_ERR_UNSUPPORTED: return "a process the kernel does not apply (photo-emission needs mcs_advance_mixed)";
    case MCS_ERR_UNIFORMS: return "a particle needed more injected uniforms than it was given";
    case MCS_ERR_CHARGE_RANGE: return "a charge beyond the int64 fixed-point range (2^30 e per particle or node)";
    default: return "";
    }
}

int use_device(mcs_ctx* c) {
    MCS_CK(c, cudaSetDevice(c->device));
    return MCS_OK;
}

template <typename T>
int dalloc(mcs_ctx* c, T** p, size_t count) {
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        return set_err(c, MCS_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    return MCS_OK;
}

int sync_status(mcs_ctx* c) {
    MCS_CK(c, cudaStreamSynchronize(c->stream));
    uint32_t st = 0;
    MCS_CK(c, cudaMemcpy(&st, c->d_status, sizeof(st), cudaMemcpyDeviceToHost));
    if (st) {
        MCS_CK(c, cudaMemset(c->d_status, 0, sizeof(uint32_t)));
        const int code = map_status(st);
        return set_err(c, code, status_text(code));
    }
    return MCS_OK;
}

}  // namespace mcs

namespace {

// First and last node of a charge array holding a nonzero value (range[0] = min, range[1] =
// max; untouched when every node is zero): one min and one max per CTA go to global atomics.
__global__ void __launch_bounds__(256) k_nonzero_range(const long long* __restrict__ q, long long n,
                                                       unsigned long long* range) {
    __shared__ unsigned long long s_lo, s_hi;
    if (threadIdx.x == 0) { s_lo = ~0ull; s_hi = 0; }
    __syncthreads();
    unsigned long long lo = ~0ull, hi = 0;
    bool any = false;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        if (q[i] != 0) {
            if (!any) lo = (unsigned long long)i;
            hi = (unsigned long long)i;
            any = true;
        }
    if (any) {
        atomicMin(&s_lo, lo);
        atomicMax(&s_hi, hi);
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_lo != ~0ull) {
        atomicMin(&range[0], s_lo);
        atomicMax(&range[1], s_hi);
    }
}

int ensure_staging(mcs_pop* p, size_t bytes) {
    if (p->staging_bytes >= bytes) return MCS_OK;
    if (p->staging) cudaFree(p->staging);
    p->staging = nullptr;
    p->staging_bytes = 0;
    void* s = nullptr;
    int st = dalloc(p->ctx, reinterpret_cast<char**>(&s), bytes);
    if (st) return st;
    p->staging = s;
    p->staging_bytes = bytes;
    return MCS_OK;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Slot of the per-step moments log for the step about to run (nullptr when disabled).
}  // namespace

namespace mcs {
double* log_slot(mcs_pop* p) {
    if (!p->d_log || p->log_cap < 1) return nullptr;
    const uint32_t k = (p->step - p->log_step0) % (uint32_t)p->log_cap;
    return p->d_log + (size_t)k * kStepMoments;
}
}  // namespace mcs

extern "C" {

MCS_API int mcs_version(void) { return 1; }

MCS_API int mcs_ctx_create(int device, mcs_ctx** out) {
    if (!out) return MCS_ERR_ARG;
    *out = nullptr;
    mcs_ctx* c = new (std::nothrow) mcs_ctx();
    if (!c) return MCS_ERR_NOMEM;
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess) { delete c; return MCS_ERR_CUDA; }
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return MCS_ERR_CUDA; }
    c->own_stream = true;
    if (cudaMalloc(&c->d_status, sizeof(uint32_t)) != cudaSuccess) { cudaStreamDestroy(c->stream); delete c; return MCS_ERR_NOMEM; }
    cudaMemset(c->d_status, 0, sizeof(uint32_t));
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaDeviceSynchronize() != cudaSuccess) { cudaFree(c->d_status); cudaStreamDestroy(c->stream); delete c; return MCS_ERR_CUDA; }
    *out = c;
    return MCS_OK;
}

MCS_API int mcs_ctx_destroy(mcs_ctx* c) {
    if (!c) return MCS_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    cudaFree(c->d_status);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
    return MCS_OK;
}

MCS_API const char* mcs_last_error(const mcs_ctx* c) { return c ? c->err.c_str() : "null context"; }

MCS_API int mcs_ctx_set_stream(mcs_ctx* c, void* stream) {
    if (!c) return MCS_ERR_ARG;
    if (c->own_stream) { cudaStreamSynchronize(c->stream); cudaStreamDestroy(c->stream); }
    c->stream = static_cast<cudaStream_t>(stream);
    c->own_stream = false;
    return MCS_OK;
}

MCS_API void* mcs_ctx_stream(mcs_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

MCS_API int mcs_ctx_set_flags(mcs_ctx* c, uint32_t flags) {
    if (!c) return MCS_ERR_ARG;
    c->flags = flags;
    return MCS_OK;
}

MCS_API int mcs_ctx_set_option(mcs_ctx* c, int option, int value) {
    if (!c) return MCS_ERR_ARG;
    if (option == MCS_OPT_MESH_SHAPE) {
        if (value < 0 || value >= MCS_MESH_SHAPES) return set_err(c, MCS_ERR_ARG, "no such mesh kernel shape");
        c->mesh_shape = value;
        return MCS_OK;
    }
    return set_err(c, MCS_ERR_ARG, "unknown option");
}

MCS_API int mcs_ctx_get_option(mcs_ctx* c, int option, int* value) {
    if (!c || !value) return MCS_ERR_ARG;
    if (option == MCS_OPT_MESH_SHAPE) { *value = c->mesh_shape; return MCS_OK; }
    return set_err(c, MCS_ERR_ARG, "unknown option");
}

MCS_API int mcs_mesh_shape(int shape, int* block, int* ppt, int* min_blocks) {
    if (!block || !ppt || !min_blocks) return MCS_ERR_ARG;
    return mesh_shape_info(shape, block, ppt, min_blocks);
}

MCS_API int mcs_sync(mcs_ctx* c) {
    if (!c) return MCS_ERR_ARG;
    if (int st = use_device(c)) return st;
    return sync_status(c);
}

// ---------------------------------------------------------------------------------------
MCS_API int mcs_table_create(mcs_ctx* c, int nrows, int neps, double e0, double emax, const double* rate,
                             const int* kind, const double* param, double maxrate, mcs_table** out) {
    if (!c || !out || !rate || !kind || !param) return MCS_ERR_ARG;
    *out = nullptr;
    if (nrows < 1 || nrows > kMaxRows) return set_err(c, MCS_ERR_ARG, "nrows must be in [1, 32]");
    if (neps < 2 || !(emax > e0) || !(maxrate > 0)) return set_err(c, MCS_ERR_ARG, "bad energy grid or maxrate");
    for (int j = 0; j < nrows; ++j)
        if (kind[j] < MCS_NULL || kind[j] > MCS_PHOTOEMISSION)
            return set_err(c, MCS_ERR_UNSUPPORTED, "unsupported collision process kind");
    if (int st = use_device(c)) return st;
    mcs_table* t = new (std::nothrow) mcs_table();
    if (!t) return MCS_ERR_NOMEM;
    t->ctx = c;
    TableView& v = t->v;
    v.nrows = nrows;
    v.nrp = (nrows + 4) & ~3;   // the total real rate, then the rows, padded to 4
    v.neps = neps;
    v.e0 = e0;
    v.emax = emax;
    v.step = (emax - e0) / (double)(neps - 1);
    v.maxrate = maxrate;
    v.inv_maxrate = 1.0 / maxrate;
    v.ke32 = (float)(0.5 * kElectronMass / v.step);
    v.e0n32 = (float)(e0 / v.step);
    v.maxrate32 = (float)maxrate;
    for (int j = 0; j < kMaxRows; ++j) {
        v.kind[j] = j < nrows ? kind[j] : MCS_NULL;
        v.param[j] = j < nrows ? param[j] : 0.0;
        if (j < nrows && kind[j] == MCS_PHOTOEMISSION) t->photo_rows = true;
    }
    const size_t n64 = (size_t)neps * nrows, n32 = (size_t)neps * v.nrp;
    int st = dalloc(c, &t->d_rate64, n64);
    if (!st) st = dalloc(c, &t->d_rate32, n32);
    if (st) { cudaFree(t->d_rate64); delete t; return st; }
    std::vector<float> r32(n32, 0.0f);
    for (int k = 0; k < neps; ++k) {
        double tot = 0.0;
        for (int j = 0; j < nrows; ++j) {
            tot += rate[(size_t)k * nrows + j];
            r32[(size_t)k * v.nrp + 1 + j] = (float)rate[(size_t)k * nrows + j];
        }
        r32[(size_t)k * v.nrp] = (float)tot;
    }
    cudaError_t e1 = cudaMemcpy(t->d_rate64, rate, n64 * sizeof(double), cudaMemcpyHostToDevice);
    cudaError_t e2 = cudaMemcpy(t->d_rate32, r32.data(), n32 * sizeof(float), cudaMemcpyHostToDevice);
    if (e1 != cudaSuccess || e2 != cudaSuccess) {
        cudaFree(t->d_rate64); cudaFree(t->d_rate32); delete t;
        return set_err(c, MCS_ERR_CUDA, "table upload failed");
    }
    v.rate64 = t->d_rate64;
    v.rate32 = t->d_rate32;
    *out = t;
    return MCS_OK;
}

MCS_API int mcs_table_destroy(mcs_table* t) {
    if (!t) return MCS_OK;
    cudaSetDevice(t->ctx->device);
    cudaStreamSynchronize(t->ctx->stream);
    cudaFree(t->d_rate64);
    cudaFree(t->d_rate32);
    delete t;
    return MCS_OK;
}

// ---------------------------------------------------------------------------------------
MCS_API int mcs_grid_create_cart3d(mcs_ctx* c, int nx, int ny, int nz, double h, double x0, double y0, double z0,
                                   int precision, mcs_grid** out) {
    if (!c || !out) return MCS_ERR_ARG;
    *out = nullptr;
    if (nx < 1 || ny < 1 || nz < 1 || !(h > 0)) return set_err(c, MCS_ERR_ARG, "bad mesh");
    if ((double)nx * ny * nz >= 4294967295.0) return set_err(c, MCS_ERR_ARG, "mesh has too many cells");
    if (precision != MCS_FP32 && precision != MCS_FP64) return set_err(c, MCS_ERR_ARG, "bad precision");
    if (int st = use_device(c)) return st;
    mcs_grid* g = new (std::nothrow) mcs_grid();
    if (!g) return MCS_ERR_NOMEM;
    g->ctx = c;
    g->precision = precision;
    GridView& v = g->v;
    v.type = GRID_CART3D;
    v.nx = nx; v.ny = ny; v.nz = nz;
    v.dnx = make_fastdiv((uint32_t)nx);
    v.dny = make_fastdiv((uint32_t)ny);
    v.h = h; v.inv_h = 1.0 / h; v.x0 = x0; v.y0 = y0; v.z0 = z0;
    const size_t nodes = (size_t)(nx + 1) * (ny + 1) * (nz + 1);
    g->nq = nodes;
    int st = MCS_OK;
    if (precision == MCS_FP32) st = dalloc(c, &g->d_e32, 4 * nodes);
    else st = dalloc(c, &g->d_e64, 3 * nodes);
    if (!st) st = dalloc(c, &g->d_q[0], nodes);
    if (!st) st = dalloc(c, &g->d_q[1], nodes);
    if (st) { cudaFree(g->d_e32); cudaFree(g->d_e64); cudaFree(g->d_q[0]); delete g; return st; }
    if (g->d_e32) cudaMemset(g->d_e32, 0, 4 * nodes * sizeof(float));
    if (g->d_e64) cudaMemset(g->d_e64, 0, 3 * nodes * sizeof(double));
    cudaMemset(g->d_q[0], 0, nodes * sizeof(long long));
    cudaMemset(g->d_q[1], 0, nodes * sizeof(long long));
    v.e32 = g->d_e32;
    v.e64 = g->d_e64;
    v.qfixed = g->d_q[0];
    v.qpart = g->d_q[1];
    *out = g;
    return MCS_OK;
}

MCS_API int mcs_grid_create_cyl(mcs_ctx* c, double R, double L, int M, int N, mcs_grid** out) {
    if (!c || !out) return MCS_ERR_ARG;
    *out = nullptr;
    if (M < 1 || N < 1 || !(R > 0) || !(L > 0)) return set_err(c, MCS_ERR_ARG, "bad cylindrical grid");
    if (int st = use_device(c)) return st;
    mcs_grid* g = new (std::nothrow) mcs_grid();
    if (!g) return MCS_ERR_NOMEM;
    g->ctx = c;
    g->precision = MCS_FP64;
    GridView& v = g->v;
    v.type = GRID_CYL;
    v.R = R; v.L = L; v.M = M; v.N = N;
    v.dr = R / M;
    v.dz = L / N;
    double zc0, zc1;
    centre_range(R, M, &v.rc0, &v.rc1, &v.drc);
    centre_range(L, N, &zc0, &zc1, &v.dzc);
    const size_t faces = (size_t)(M + 3) * (N + 3), cells = (size_t)(M + 2) * (N + 2);
    g->nq = cells;
    int st = dalloc(c, &g->d_er, faces);
    if (!st) st = dalloc(c, &g->d_ez, faces);
    if (!st) st = dalloc(c, &g->d_erz32, 2 * faces);
    if (!st) st = dalloc(c, &g->d_q[0], cells);
    if (!st) st = dalloc(c, &g->d_q[1], cells);
    if (st) {
        cudaFree(g->d_er); cudaFree(g->d_ez); cudaFree(g->d_erz32); cudaFree(g->d_q[0]); delete g;
        return st;
    }
    cudaMemset(g->d_er, 0, faces * sizeof(double));
    cudaMemset(g->d_ez, 0, faces * sizeof(double));
    cudaMemset(g->d_erz32, 0, 2 * faces * sizeof(float));
    v.er32 = g->d_erz32;
    v.ez32 = g->d_erz32 + faces;
    v.R32 = (float)R;
    v.L32 = (float)L;
    v.inv_dr32 = (float)(1.0 / v.drc);
    v.inv_dz32 = (float)(1.0 / v.dzc);
    cudaMemset(g->d_q[0], 0, cells * sizeof(long long));
    cudaMemset(g->d_q[1], 0, cells * sizeof(long long));
    v.er = g->d_er;
    v.ez = g->d_ez;
    v.qfixed = g->d_q[0];
    v.qpart = g->d_q[1];
    *out = g;
    return MCS_OK;
}

MCS_API int mcs_grid_destroy(mcs_grid* g) {
    if (!g) return MCS_OK;
    cudaSetDevice(g->ctx->device);
    cudaStreamSynchronize(g->ctx->stream);
    if (g->fluid) g->fluid->g = nullptr;
    cudaFree(g->d_e32); cudaFree(g->d_e64); cudaFree(g->d_er); cudaFree(g->d_ez); cudaFree(g->d_erz32);
    cudaFree(g->d_qfd);
    cudaFree(g->d_init_ws);
    cudaFree(g->d_q[0]); cudaFree(g->d_q[1]);
    cudaFree(g->d_range);
    delete g;
    return MCS_OK;
}

MCS_API int mcs_grid_set_efield(mcs_grid* g, const double* e) {
    if (!g || !e) return MCS_ERR_ARG;
    mcs_ctx* c = g->ctx;
    if (int st = use_device(c)) return st;
    MCS_CK(c, cudaStreamSynchronize(c->stream));
    if (g->v.type == GRID_CART3D) {
        const size_t nodes = g->nq;
        if (g->d_e32) {
            std::vector<float> tmp(4 * nodes);
            for (size_t i = 0; i < nodes; ++i) {
                tmp[4 * i] = (float)e[3 * i];
                tmp[4 * i + 1] = (float)e[3 * i + 1];
                tmp[4 * i + 2] = (float)e[3 * i + 2];
                tmp[4 * i + 3] = 0.0f;
            }
            MCS_CK(c, cudaMemcpy(g->d_e32, tmp.data(), tmp.size() * sizeof(float), cudaMemcpyHostToDevice));
        } else {
            MCS_CK(c, cudaMemcpy(g->d_e64, e, 3 * nodes * sizeof(double), cudaMemcpyHostToDevice));
        }
    } else {
        const size_t faces = (size_t)(g->v.M + 3) * (g->v.N + 3);
        MCS_CK(c, cudaMemcpy(g->d_er, e, faces * sizeof(double), cudaMemcpyHostToDevice));
        MCS_CK(c, cudaMemcpy(g->d_ez, e + faces, faces * sizeof(double), cudaMemcpyHostToDevice));
        std::vector<float> tmp(2 * faces);
        for (size_t i = 0; i < 2 * faces; ++i) tmp[i] = (float)e[i];
        MCS_CK(c, cudaMemcpy(g->d_erz32, tmp.data(), tmp.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    return MCS_OK;
}

MCS_API int mcs_grid_set_efield_range(mcs_grid* g, int64_t node0, int64_t count, const double* e) {
    if (!g || !e || node0 < 0 || count < 0) return MCS_ERR_ARG;
    mcs_ctx* c = g->ctx;
    if (g->v.type != GRID_CART3D) return set_err(c, MCS_ERR_ARG, "range upload needs a cart3d grid");
    if ((size_t)(node0 + count) > g->nq) return set_err(c, MCS_ERR_ARG, "node range beyond the mesh");
    if (int st = use_device(c)) return st;
    MCS_CK(c, cudaStreamSynchronize(c->stream));
    if (g->d_e32) {
        std::vector<float> tmp(4 * (size_t)count);
        for (int64_t i = 0; i < count; ++i) {
            tmp[4 * i] = (float)e[3 * i];
            tmp[4 * i + 1] = (float)e[3 * i + 1];
            tmp[4 * i + 2] = (float)e[3 * i + 2];
            tmp[4 * i + 3] = 0.0f;
        }
        MCS_CK(c, cudaMemcpy(g->d_e32 + 4 * node0, tmp.data(), tmp.size() * sizeof(float), cudaMemcpyHostToDevice));
    } else {
        MCS_CK(c, cudaMemcpy(g->d_e64 + 3 * node0, e, 3 * (size_t)count * sizeof(double), cudaMemcpyHostToDevice));
    }
    return MCS_OK;
}

MCS_API int mcs_grid_read_efield(mcs_grid* g, double* e) {
    if (!g || !e) return MCS_ERR_ARG;
    mcs_ctx* c = g->ctx;
    if (int st = use_device(c)) return st;
    MCS_CK(c, cudaStreamSynchronize(c->stream));
    if (g->v.type == GRID_CYL) {
        const size_t faces = (size_t)(g->v.M + 3) * (g->v.N + 3);
        MCS_CK(c, cudaMemcpy(e, g->d_er, faces * sizeof(double), cudaMemcpyDeviceToHost));
        MCS_CK(c, cudaMemcpy(e + faces, g->d_ez, faces * sizeof(double), cudaMemcpyDeviceToHost));
        return MCS_OK;
    }
    if (g->d_e32) {
        std::vector<float> tmp(4 * g->nq);
        MCS_CK(c, cudaMemcpy(tmp.data(), g->d_e32, tmp.size() * sizeof(float), cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < g->nq; ++i)
            for (int d = 0; d < 3; ++d) e[3 * i + d] = tmp[4 * i + d];
    } else {
        MCS_CK(c, cudaMemcpy(e, g->d_e64, 3 * g->nq * sizeof(double), cudaMemcpyDeviceToHost));
    }
    return MCS_OK;
}

MCS_API int mcs_grid_read_efield_range(mcs_grid* g, int64_t node0, int64_t count, double* e) {
    if (!g || !e || node0 < 0 || count < 0) return MCS_ERR_ARG;
    mcs_ctx* c = g->ctx;
    if (g->v.type != GRID_CART3D) return set_err(c, MCS_ERR_ARG, "range read needs a cart3d grid");
    if ((size_t)(node0 + count) > g->nq) return set_err(c, MCS_ERR_ARG, "node range beyond the mesh");
    if (int st = use_device(c)) return st;
    MCS_CK(c, cudaStreamSynchronize(c->stream));
    if (g->d_e32) {
        std::vector<float> tmp(4 * (size_t)count);
        MCS_CK(c, cudaMemcpy(tmp.data(), g->d_e32 + 4 * node0, tmp.size() * sizeof(float), cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < count; ++i)
            for (int d = 0; d < 3; ++d) e[3 * i + d] = tmp[4 * i + d];
    } else {
        MCS_CK(c, cudaMemcpy(e, g->d_e64 + 3 * node0, 3 * (size_t)count * sizeof(double), cudaMemcpyDeviceToHost));
    }
    return MCS_OK;
}

MCS_API int mcs_grid_read_fixed_range(mcs_grid* g, int which, int64_t node0, int64_t count, int64_t* out) {
    if (!g || !out || (which != MCS_Q_FIXED && which != MCS_Q_PART) || node0 < 0 || count < 0) return MCS_ERR_ARG;
    mcs_ctx* c = g->ctx;
    if ((size_t)(node0 + count) > g->nq) return set_err(c, MCS_ERR_ARG, "range beyond the charge array");
    if (int st = use_device(c)) return st;
    MCS_CK(c, cudaStreamSynchronize(c->stream));
    MCS_CK(c, cudaMemcpy(out, g->d_q[which] + node0, (size_t)count * sizeof(long long), cudaMemcpyDeviceToHost));
    return sync_status(c);
}

MCS_API int mcs_grid_fixed_plane_range(mcs_grid* g, int which, int64_t* z0, int64_t* z1) {
    if (!g || !z0 || !z1 || (which != MCS_Q_FIXED && which != MCS_Q_PART)) return MCS_ERR_ARG;
    mcs_ctx* c = g->ctx;
    if (g->v.type != GRID_CART3D) return set_err(c, MCS_ERR_UNSUPPORTED, "plane ranges are of cart3d grids");
    if (int st = use_device(c)) return st;
    if (!g->d_range && cudaMalloc(&g->d_range, 2 * sizeof(unsigned long long)) != cudaSuccess) {
        g->d_range = nullptr;
        return set_err(c, MCS_ERR_NOMEM, "plane range buffer");
    }
    MCS_CK(c, cudaMemsetAsync(g->d_range, 0xff, sizeof(unsigned long long), c->stream));
    MCS_CK(c, cudaMemsetAsync(g->d_range + 1, 0, sizeof(unsigned long long), c->stream));
    k_nonzero_range<<<c->num_sms * 4, 256, 0, c->stream>>>(g->d_q[which], (long long)g->nq, g->d_range);
    MCS_CK_LAUNCH(c);
    unsigned long long r[2] = {0, 0};
    MCS_CK(c, cudaMemcpyAsync(r, g->d_range, sizeof(r), cudaMemcpyDeviceToHost, c->stream));
    if (int st = sync_status(c)) return st;
    const long long plane = (long long)(g->v.nx + 1) * (g->v.ny + 1);
    if (r[0] == ~0ull) {
        *z0 = *z1 = 0;
    } else {
        *z0 = (int64_t)(r[0] / (unsigned long long)plane);
        *z1 = (int64_t)(r[1] / (unsigned long long)plane) + 1;
    }
    return MCS_OK;
}

MCS_API int mcs_grid_zero(mcs_grid* g, int which) {
    if (!g || (which != MCS_Q_FIXED && which != MCS_Q_PART)) return MCS_ERR_ARG;
    mcs_ctx* c = g->ctx;
    if (int st = use_device(c)) return st;
    MCS_CK(c, cudaMemsetAsync(g->d_q[which], 0, g->nq * sizeof(long long), c->stream));
    if (which == MCS_Q_FIXED && g->d_qfd)
        MCS_CK(c, cudaMemsetAsync(g->d_qfd, 0, (size_t)(g->v.M + 2) * (g->v.N + 2) * sizeof(double), c->stream));
    return MCS_OK;
}

MCS_API int mcs_grid_read_fixed(mcs_grid* g, int which, int64_t* out) {
    if (!g || !out || (which != MCS_Q_FIXED && which != MCS_Q_PART)) return MCS_ERR_ARG;
    mcs_ctx* c = g->ctx;
    if (int st = use_device(c)) return st;
    const int st = sync_status(c);
    MCS_CK(c, cudaMemcpy(out, g->d_q[which], g->nq * sizeof(long long), cudaMemcpyDeviceToHost));
    return st;
}

MCS_API int mcs_grid_write_fixed(mcs_grid* g, int which, const int64_t* in) {
    if (!g || !in || (which != MCS_Q_FIXED && which != MCS_Q_PART)) return MCS_ERR_ARG;
    mcs_ctx* c = g->ctx;
    if (int st = use_device(c)) return st;
    MCS_CK(c, cudaMemcpyAsync(g->d_q[which], in, g->nq * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
    MCS_CK(c, cudaStreamSynchronize(c->stream));
    return MCS_OK;
}

MCS_API int mcs_grid_charge_ptr(mcs_grid* g, int which, void** dptr, int64_t* count) {
    if (!g || !dptr || !count || (which != MCS_Q_FIXED && which != MCS_Q_PART)) return MCS_ERR_ARG;
    *dptr = g->d_q[which];
    *count = (int64_t)g->nq;
    return MCS_OK;
}

MCS_API int mcs_grid_read_density(mcs_grid* g, int which, double* out) {
    if (!g || !out || (which != MCS_Q_FIXED && which != MCS_Q_PART)) return MCS_ERR_ARG;
    std::vector<long long> q(g->nq);
    const int st = mcs_grid_read_fixed(g, which, reinterpret_cast<int64_t*>(q.data()));
    if (st == MCS_ERR_CUDA || st == MCS_ERR_ARG) return st;
    if (g->v.type == GRID_CART3D) {
        for (size_t i = 0; i < g->nq; ++i) out[i] = (double)q[i] * 0x1p-32;
    } else {
        const int M = g->v.M, N = g->v.N;
        for (int j = 0; j < N + 2; ++j)
            for (int i = 0; i < M + 2; ++i) {
                const size_t k = (size_t)i + (size_t)j * (M + 2);
                if (i < 1 || i > M) { out[k] = 0.0; continue; }
                const double rc = lerpi(i - 1, M > 1 ? M - 1 : 1, g->v.rc0, g->v.rc1);  // grid.rc[i]
                const double dV = 2.0 * M_PI * rc * g->v.drc * g->v.dzc;                 // grid.jl:76
                out[k] = (double)q[k] * 0x1p-32 / dV;
            }
    }
    return st;
}

// ---------------------------------------------------------------------------------------
MCS_API int mcs_field_uniform(mcs_ctx* c, double ex, double ey, double ez, mcs_field** out) {
    if (!c || !out) return MCS_ERR_ARG;
    mcs_field* f = new (std::nothrow) mcs_field();
    if (!f) return MCS_ERR_NOMEM;
    f->ctx = c;
    f->type = FIELD_UNIFORM;
    f->e[0] = ex; f->e[1] = ey; f->e[2] = ez;
    *out = f;
    return MCS_OK;
}

MCS_API int mcs_field_from_grid(mcs_grid* g, mcs_field** out) {
    if (!g || !out) return MCS_ERR_ARG;
    mcs_field* f = new (std::nothrow) mcs_field();
    if (!f) return MCS_ERR_NOMEM;
    f->ctx = g->ctx;
    f->type = FIELD_GRID;
    f->grid = g;
    *out = f;
    return MCS_OK;
}

MCS_API int mcs_field_destroy(mcs_field* f) {
    delete f;
    return MCS_OK;
}

// ---------------------------------------------------------------------------------------
MCS_API int mcs_pop_create(mcs_ctx* c, int64_t capacity, int precision, mcs_grid* cells, mcs_pop** out) {
    if (!c || !out) return MCS_ERR_ARG;
    *out = nullptr;
    if (capacity < 1 || capacity > 0xfffffff0LL) return set_err(c, MCS_ERR_ARG, "capacity must be in [1, 2^32-16]");
    if (precision != MCS_FP32 && precision != MCS_FP64) return set_err(c, MCS_ERR_ARG, "bad precision");
    if (cells && cells->v.type != GRID_CART3D) return set_err(c, MCS_ERR_ARG, "cell layout needs a cart3d grid");
    if (int st = use_device(c)) return st;
    mcs_pop* p = new (std::nothrow) mcs_pop();
    if (!p) return MCS_ERR_NOMEM;
    p->ctx = c;
    p->precision = precision;
    p->cells = cells;
    p->cap = capacity;
    p->esz = precision == MCS_FP32 ? 4 : 8;
    int st = MCS_OK;
    for (int q = 0; q < 8 && !st; ++q) st = dalloc(c, reinterpret_cast<char**>(&p->f[q]), (size_t)capacity * p->esz);
    if (!st) st = dalloc(c, &p->act, (size_t)capacity);
    if (!st && cells) st = dalloc(c, &p->cell, (size_t)capacity);
    if (!st) st = dalloc(c, &p->d_n, 2);
    p->max_tiles = (capacity + 127) / 128 + 1;
    if (!st) st = dalloc(c, &p->tile_status, (size_t)p->max_tiles);
    size_t npart = (size_t)p->max_tiles * kStepMoments;
    if (npart < (size_t)kMomentPartialsMin) npart = kMomentPartialsMin;
    if (!st) st = dalloc(c, &p->tile_partials, npart);
    if (!st) st = dalloc(c, &p->counters, kCounterWords);
    if (!st) st = dalloc(c, &p->d_moments, MCS_MOMENTS_BASE + kMaxRows);
    if (!st) st = dalloc(c, &p->u32a, (size_t)capacity);
    if (!st) st = dalloc(c, &p->u32b, (size_t)capacity);
    if (st) { mcs_pop_destroy(p); return st; }
    cudaMemset(p->d_n, 0, 2 * sizeof(long long));
    cudaMemset(p->tile_status, 0, (size_t)p->max_tiles * sizeof(unsigned long long));
    cudaMemset(p->counters, 0, kCounterWords * sizeof(uint32_t));
    cudaMemset(p->act, 0, (size_t)capacity);
    if (cudaDeviceSynchronize() != cudaSuccess) { mcs_pop_destroy(p); return set_err(c, MCS_ERR_CUDA, "pop init"); }
    *out = p;
    return MCS_OK;
}

MCS_API int mcs_pop_destroy(mcs_pop* p) {
    if (!p) return MCS_OK;
    cudaSetDevice(p->ctx->device);
    cudaStreamSynchronize(p->ctx->stream);
    for (int q = 0; q < 8; ++q) { cudaFree(p->f[q]); cudaFree(p->alt[q]); }
    cudaFree(p->act); cudaFree(p->cell); cudaFree(p->d_n); cudaFree(p->tile_status);
    cudaFree(p->tile_partials); cudaFree(p->counters); cudaFree(p->d_moments); cudaFree(p->staging);
    cudaFree(p->app_cnt); cudaFree(p->app_off); cudaFree(p->app_excl);
    cudaFree(p->u32a); cudaFree(p->u32b); cudaFree(p->alt_cell); cudaFree(p->alt_act); cudaFree(p->stage); cudaFree(p->d_log);
    for (int q = 0; q < 2; ++q) { cudaFree(p->sort_key[q]); cudaFree(p->sort_val[q]); }
    cudaFree(p->sort_hist); cudaFree(p->sort_hoff); cudaFree(p->seg_a); cudaFree(p->seg_b);
    cudaFree(p->d_inj_u); cudaFree(p->d_inj_pos); cudaFree(p->d_inj_end);
    free_host_step(p->host_step);
    delete p;
    return MCS_OK;
}

MCS_API int mcs_pop_set_seed(mcs_pop* p, uint64_t seed, uint32_t step) {
    if (!p) return MCS_ERR_ARG;
    p->seed = seed;
    p->step = step;
    return MCS_OK;
}

MCS_API int mcs_set_uniform_source(mcs_pop* p, int mode, const double* u, const int64_t* offsets, int64_t nslots) {
    if (!p) return MCS_ERR_ARG;
    mcs_ctx* c = p->ctx;
    if (mode == MCS_UNIFORMS_PHILOX) {
        p->inj = false;
        return MCS_OK;
    }
    if (mode != MCS_UNIFORMS_INJECTED || nslots < 0 || !offsets) return set_err(c, MCS_ERR_ARG, "uniform source mode");
    if (p->cells) return set_err(c, MCS_ERR_UNSUPPORTED, "injected uniforms on a mesh-layout population");
    if (offsets[0] < 0) return set_err(c, MCS_ERR_ARG, "negative uniform offset");
    for (int64_t i = 0; i < nslots; ++i)
        if (offsets[i + 1] < offsets[i]) return set_err(c, MCS_ERR_ARG, "uniform offsets must not decrease");
    const int64_t total = offsets[nslots];
    if (total > 0 && !u) return set_err(c, MCS_ERR_ARG, "no uniforms");
    if (int st = use_device(c)) return st;
    MCS_CK(c, cudaStreamSynchronize(c->stream));   // steps in flight still read the old values
    cudaFree(p->d_inj_u); cudaFree(p->d_inj_pos); cudaFree(p->d_inj_end);
    p->d_inj_u = nullptr; p->d_inj_pos = nullptr; p->d_inj_end = nullptr;
    p->inj = false;
    int st = dalloc(c, &p->d_inj_u, (size_t)std::max<int64_t>(total, 1));
    if (!st) st = dalloc(c, &p->d_inj_pos, (size_t)std::max<int64_t>(nslots, 1));
    if (!st) st = dalloc(c, &p->d_inj_end, (size_t)std::max<int64_t>(nslots, 1));
    if (st) return st;
    if (total > 0) MCS_CK(c, cudaMemcpy(p->d_inj_u, u, (size_t)total * sizeof(double), cudaMemcpyHostToDevice));
    if (nslots > 0) {
        MCS_CK(c, cudaMemcpy(p->d_inj_pos, offsets, (size_t)nslots * sizeof(int64_t), cudaMemcpyHostToDevice));
        MCS_CK(c, cudaMemcpy(p->d_inj_end, offsets + 1, (size_t)nslots * sizeof(int64_t), cudaMemcpyHostToDevice));
    }
    p->inj_n = nslots;
    p->inj = true;
    return MCS_OK;
}

MCS_API int mcs_pop_get_step(mcs_pop* p, uint32_t* step) {
    if (!p || !step) return MCS_ERR_ARG;
    *step = p->step;
    return MCS_OK;
}

MCS_API int mcs_pop_upload(mcs_pop* p, const double* x, const double* v, const double* w, const double* s,
                           const uint8_t* active, int64_t n) {
    if (!p || n < 0 || (n > 0 && (!x || !v || !w || !s || !active))) return MCS_ERR_ARG;
    mcs_ctx* c = p->ctx;
    if (n > p->cap) return set_err(c, MCS_ERR_CAPACITY, "Maximum number of particles reached");
    if (int st = use_device(c)) return st;
    const size_t o_v = align256(3 * n * sizeof(double)), o_w = o_v + align256(3 * n * sizeof(double));
    const size_t o_s = o_w + align256(n * sizeof(double)), o_a = o_s + align256(n * sizeof(double));
    const size_t bytes = o_a + align256((size_t)n);
    if (int st = ensure_staging(p, bytes)) return st;
    char* b = static_cast<char*>(p->staging);
    if (n > 0) {
        MCS_CK(c, cudaMemcpyAsync(b, x, 3 * n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        MCS_CK(c, cudaMemcpyAsync(b + o_v, v, 3 * n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        MCS_CK(c, cudaMemcpyAsync(b + o_w, w, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        MCS_CK(c, cudaMemcpyAsync(b + o_s, s, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        MCS_CK(c, cudaMemcpyAsync(b + o_a, active, (size_t)n, cudaMemcpyHostToDevice, c->stream));
        if (int st = launch_upload(p, reinterpret_cast<double*>(b), reinterpret_cast<double*>(b + o_v),
                                   reinterpret_cast<double*>(b + o_w), reinterpret_cast<double*>(b + o_s),
                                   reinterpret_cast<uint8_t*>(b + o_a), n))
            return st;
    }
    const long long nn = n;
    MCS_CK(c, cudaMemcpyAsync(p->d_n + p->cur, &nn, sizeof(nn), cudaMemcpyHostToDevice, c->stream));
    MCS_CK(c, cudaStreamSynchronize(c->stream));  // nn and the host buffers are caller-owned
    return MCS_OK;
}

MCS_API int mcs_pop_init_maxwellian(mcs_pop* p, int64_t n, double mean_energy_ev) {
    if (!p || n < 0 || !(mean_energy_ev >= 0)) return MCS_ERR_ARG;
    mcs_ctx* c = p->ctx;
    if (p->cells) return set_err(c, MCS_ERR_UNSUPPORTED, "swarm initialisation of a cell-layout population");
    if (n > p->cap) return set_err(c, MCS_ERR_CAPACITY, "Maximum number of particles reached");
    if (int st = use_device(c)) return st;
    if (n > 0)
        if (int st = launch_init_maxwellian(p, n, maxwellian_sigma(mean_energy_ev))) return st;
    const long long nn = n;
    MCS_CK(c, cudaMemcpyAsync(p->d_n + p->cur, &nn, sizeof(nn), cudaMemcpyHostToDevice, c->stream));
    MCS_CK(c, cudaStreamSynchronize(c->stream));
    return MCS_OK;
}

MCS_API int mcs_pop_init_cloud(mcs_pop* p, int64_t n, double cx, double cy, double cz, double sigma,
                               double energy_ev, double wmin, double wmax) {
    if (!p || n < 0 || !(sigma >= 0) || !(energy_ev >= 0) || !(wmin > 0) || !(wmax >= wmin)) return MCS_ERR_ARG;
    mcs_ctx* c = p->ctx;
    if (n > p->cap) return set_err(c, MCS_ERR_CAPACITY, "Maximum number of particles reached");
    if (int st = use_device(c)) return st;
    const double ctr[3] = {cx, cy, cz};
    if (n > 0)
        if (int st = launch_init_cloud(p, n, ctr, sigma, sqrt(2.0 * energy_ev * kElementaryCharge / kElectronMass),
                                       wmin, wmax))
            return st;
    const long long nn = n;
    MCS_CK(c, cudaMemcpyAsync(p->d_n + p->cur, &nn, sizeof(nn), cudaMemcpyHostToDevice, c->stream));
    MCS_CK(c, cudaStreamSynchronize(c->stream));
    return MCS_OK;
}

MCS_API int mcs_grid_set_efield_gaussian(mcs_grid* g, double cx, double cy, double cz, double sigma, double rho_peak,
                                         double ebx, double eby, double ebz) {
    if (!g || !(sigma > 0)) return MCS_ERR_ARG;
    mcs_ctx* c = g->ctx;
    if (g->v.type != GRID_CART3D) return set_err(c, MCS_ERR_ARG, "the Gaussian field needs a cart3d grid");
    if (int st = use_device(c)) return st;
    const double ctr[3] = {cx, cy, cz}, eb[3] = {ebx, eby, ebz};
    if (int st = launch_efield_gaussian(g, ctr, sigma, rho_peak, eb)) return st;
    MCS_CK(c, cudaStreamSynchronize(c->stream));
    return MCS_OK;
}

MCS_API int mcs_pop_copy(mcs_pop* dst, const mcs_pop* src) {
    if (!dst || !src || dst->ctx != src->ctx) return MCS_ERR_ARG;
    mcs_ctx* c = dst->ctx;
    if (dst->precision != src->precision || dst->cells != src->cells)
        return set_err(c, MCS_ERR_ARG, "populations differ in precision or layout");
    if (dst->cap < src->cap) return set_err(c, MCS_ERR_CAPACITY, "destination capacity below source capacity");
    if (int st = use_device(c)) return st;
    const size_t n = (size_t)src->cap;
    for (int q = 0; q < 8; ++q)
        MCS_CK(c, cudaMemcpyAsync(dst->f[q], src->f[q], n * src->esz, cudaMemcpyDeviceToDevice, c->stream));
    MCS_CK(c, cudaMemcpyAsync(dst->act, src->act, n, cudaMemcpyDeviceToDevice, c->stream));
    if (src->cell)
        MCS_CK(c, cudaMemcpyAsync(dst->cell, src->cell, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, c->stream));
    MCS_CK(c, cudaMemcpyAsync(dst->d_n + dst->cur, src->d_n + src->cur, sizeof(long long), cudaMemcpyDeviceToDevice,
                              c->stream));
    dst->seed = src->seed;
    dst->step = src->step;
    return MCS_OK;
}

MCS_API int mcs_pop_nparticles(mcs_pop* p, int64_t* n) {
    if (!p || !n) return MCS_ERR_ARG;
    mcs_ctx* c = p->ctx;
    if (int st = use_device(c)) return st;
    long long v = 0;
    MCS_CK(c, cudaMemcpyAsync(&v, p->d_n + p->cur, sizeof(v), cudaMemcpyDeviceToHost, c->stream));
    const int st = sync_status(c);
    *n = v;
    return st;
}

MCS_API int mcs_pop_download(mcs_pop* p, double* x, double* v, double* w, double* s, uint8_t* active, int64_t cap,
                             int64_t* n_out) {
    if (!p || !n_out) return MCS_ERR_ARG;
    mcs_ctx* c = p->ctx;
    int64_t n = 0;
    int st = mcs_pop_nparticles(p, &n);
    if (st == MCS_ERR_CUDA) return st;
    *n_out = n;
    if (n > cap) return set_err(c, MCS_ERR_ARG, "host buffers too small");
    if (n == 0) return st;
    if (!x || !v || !w || !s || !active) return MCS_ERR_ARG;
    const size_t o_v = align256(3 * n * sizeof(double)), o_w = o_v + align256(3 * n * sizeof(double));
    const size_t o_s = o_w + align256(n * sizeof(double)), o_a = o_s + align256(n * sizeof(double));
    const size_t bytes = o_a + align256((size_t)n);
    if (int e = ensure_staging(p, bytes)) return e;
    char* b = static_cast<char*>(p->staging);
    if (int e = launch_download(p, reinterpret_cast<double*>(b), reinterpret_cast<double*>(b + o_v),
                                reinterpret_cast<double*>(b + o_w), reinterpret_cast<double*>(b + o_s),
                                reinterpret_cast<uint8_t*>(b + o_a)))
        return e;
    MCS_CK(c, cudaMemcpyAsync(x, b, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    MCS_CK(c, cudaMemcpyAsync(v, b + o_v, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    MCS_CK(c, cudaMemcpyAsync(w, b + o_w, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    MCS_CK(c, cudaMemcpyAsync(s, b + o_s, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    MCS_CK(c, cudaMemcpyAsync(active, b + o_a, (size_t)n, cudaMemcpyDeviceToHost, c->stream));
    MCS_CK(c, cudaStreamSynchronize(c->stream));
    return st;
}

// ---------------------------------------------------------------------------------------
MCS_API int mcs_advance(mcs_pop* p, const mcs_table* t, const mcs_field* f, double dt, mcs_grid* tracker) {
    if (!p || !t || !f) return MCS_ERR_ARG;
    mcs_ctx* c = p->ctx;
    if (t->photo_rows) return set_err(c, MCS_ERR_UNSUPPORTED, "photo-emission needs mcs_advance_mixed");
    if (!(dt >= 0)) return set_err(c, MCS_ERR_ARG, "dt must be >= 0");
    if (f->type == FIELD_GRID && !f->grid) return MCS_ERR_ARG;
    if (int st = use_device(c)) return st;
    int st;
    if (p->cells) {
        if (f->type != FIELD_GRID || f->grid != p->cells)
            return set_err(c, MCS_ERR_UNSUPPORTED, "a cell-layout population needs the field of its own mesh");
        if (tracker && tracker != p->cells)
            return set_err(c, MCS_ERR_UNSUPPORTED, "a cell-layout population tracks onto its own mesh");
        st = p->precision == MCS_FP32 ? launch_step_mesh<float>(p, t, dt, tracker != nullptr, 0.0, log_slot(p))
                                      : launch_step_mesh<double>(p, t, dt, tracker != nullptr, 0.0, log_slot(p));
    } else {
        st = p->precision == MCS_FP32 ? launch_step_abs<float>(p, t, f, dt, tracker, log_slot(p))
                                      : launch_step_abs<double>(p, t, f, dt, tracker, log_slot(p));
    }
    if (st) return st;
    p->cur ^= 1;
    p->step += 1;
    return MCS_OK;
}

MCS_API int mcs_advance_deposit(mcs_pop* p, const mcs_table* t, const mcs_field* f, double dt, mcs_grid* tracker,
                                mcs_grid* deposit, double val) {
    if (!p || !t || !f || !deposit) return MCS_ERR_ARG;
    mcs_ctx* c = p->ctx;
    if (t->photo_rows) return set_err(c, MCS_ERR_UNSUPPORTED, "photo-emission needs mcs_advance_mixed");
    if (!p->cells || deposit != p->cells || f->type != FIELD_GRID || f->grid != p->cells ||
        (tracker && tracker != p->cells))
        return set_err(c, MCS_ERR_UNSUPPORTED, "fused step+deposit needs a cell-layout population on one mesh");
    if (!(dt >= 0)) return set_err(c, MCS_ERR_ARG, "dt must be >= 0");
    if (int st = use_device(c)) return st;
    const int st = p->precision == MCS_FP32 ? launch_step_mesh<float>(p, t, dt, tracker != nullptr, val, log_slot(p))
                                            : launch_step_mesh<double>(p, t, dt, tracker != nullptr, val, log_slot(p));
    if (st) return st;
    p->cur ^= 1;
    p->step += 1;
    return MCS_OK;
}

MCS_API int mcs_collisions(mcs_pop* p, const mcs_table* t, double dt, mcs_grid* tracker) {
    if (!p || !t) return MCS_ERR_ARG;
    mcs_ctx* c = p->ctx;
    if (p->cells) return set_err(c, MCS_ERR_UNSUPPORTED, "collisions! on a cell-layout population");
    if (t->photo_rows) return set_err(c, MCS_ERR_UNSUPPORTED, "photo-emission needs mcs_advance_mixed");
    if (int st = use_device(c)) return st;
    const int st = p->precision == MCS_FP32 ? launch_collisions<float>(p, t, dt, tracker)
                                            : launch_collisions<double>(p, t, dt, tracker);
    if (st) return st;
    p->cur ^= 1;
    p->step += 1;
    return MCS_OK;
}

MCS_API int mcs_deposit(mcs_pop* p, mcs_grid* g, double val) {
    if (!p || !g) return MCS_ERR_ARG;
    if (p->cells && p->cells != g) return set_err(p->ctx, MCS_ERR_UNSUPPORTED, "deposit onto another mesh");
    if (int st = use_device(p->ctx)) return st;
    return launch_deposit(p, g, val);
}

MCS_API int mcs_repack(mcs_pop* p) {
    if (!p) return MCS_ERR_ARG;
    if (int st = use_device(p->ctx)) return st;
    return launch_repack(p);
}

MCS_API int mcs_swarm_resample(mcs_pop* p, int64_t n0, double tol) {
    if (!p || n0 < 1) return MCS_ERR_ARG;
    if (int st = use_device(p->ctx)) return st;
    return launch_swarm_resample(p, n0, tol);
}

MCS_API int mcs_moments(mcs_pop* p, const mcs_table* t, double* out, int nout) {
    if (!p || !out) return MCS_ERR_ARG;
    mcs_ctx* c = p->ctx;
    const int nm = MCS_MOMENTS_BASE + (t ? t->v.nrows : 0);
    if (nout < nm) return set_err(c, MCS_ERR_ARG, "moments buffer too small");
    if (int st = use_device(c)) return st;
    if (int st = launch_moments(p, t, p->d_moments, nm)) return st;
    MCS_CK(c, cudaMemcpyAsync(out, p->d_moments, nm * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return sync_status(c);
}

MCS_API int mcs_pop_step_log(mcs_pop* p, int capacity) {
    if (!p || capacity < 0) return MCS_ERR_ARG;
    mcs_ctx* c = p->ctx;
    if (int st = use_device(c)) return st;
    MCS_CK(c, cudaStreamSynchronize(c->stream));
    cudaFree(p->d_log);
    p->d_log = nullptr;
    p->log_cap = 0;
    if (capacity == 0) return MCS_OK;
    if (int st = dalloc(c, &p->d_log, (size_t)capacity * kStepMoments)) return st;
    MCS_CK(c, cudaMemset(p->d_log, 0, (size_t)capacity * kStepMoments * sizeof(double)));
    p->log_cap = capacity;
    p->log_step0 = p->step;
    return MCS_OK;
}

MCS_API int mcs_pop_read_step_log(mcs_pop* p, double* out, int nsteps) {
    if (!p || !out || nsteps < 0) return MCS_ERR_ARG;
    mcs_ctx* c = p->ctx;
    if (nsteps > p->log_cap) return set_err(c, MCS_ERR_ARG, "more steps than the log holds");
    if (int st = use_device(c)) return st;
    if (nsteps > 0)
        MCS_CK(c, cudaMemcpyAsync(out, p->d_log, (size_t)nsteps * kStepMoments * sizeof(double),
                                  cudaMemcpyDeviceToHost, c->stream));
    return sync_status(c);
}

MCS_API int mcs_swarm_run(mcs_pop* p, const mcs_table* t, const mcs_field* f, double dt, int nsteps, int64_t n0,
                          double tol, int repack_every, double* moments_out) {
    if (!p || !t || !f || nsteps < 0) return MCS_ERR_ARG;
    mcs_ctx* c = p->ctx;
    if (p->cells) return set_err(c, MCS_ERR_UNSUPPORTED, "swarm loop on a cell-layout population");
    if (t->photo_rows) return set_err(c, MCS_ERR_UNSUPPORTED, "photo-emission needs mcs_advance_mixed");
    if (int st = use_device(c)) return st;
    double* d_out = nullptr;
    if (int st = dalloc(c, &d_out, (size_t)(nsteps > 0 ? nsteps : 1) * kStepMoments)) return st;
    int st = MCS_OK;
    for (int i = 0; i < nsteps && !st; ++i) {
        double* mo = d_out + (size_t)i * kStepMoments;
        st = p->precision == MCS_FP32 ? launch_step_abs<float>(p, t, f, dt, nullptr, mo)
                                      : launch_step_abs<double>(p, t, f, dt, nullptr, mo);
        if (st) break;
        p->cur ^= 1;
        p->step += 1;
        if (n0 > 0) st = launch_swarm_resample(p, n0, tol);
        if (!st && repack_every > 0 && (i + 1) % repack_every == 0) st = launch_repack(p);
    }
    if (!st && moments_out && nsteps > 0) {
        cudaError_t e = cudaMemcpyAsync(moments_out, d_out, (size_t)nsteps * kStepMoments * sizeof(double),
                                        cudaMemcpyDeviceToHost, c->stream);
        if (e != cudaSuccess) st = set_err(c, MCS_ERR_CUDA, cudaGetErrorString(e));
    }
    const int st2 = sync_status(c);
    cudaFree(d_out);
    return st ? st : st2;
}

}  // extern "C"
