// host_util.h -- host helpers shared by the translation units of the library.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <string>

#include "mcs_internal.h"

namespace mcs {

inline int set_err(mcs_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

#define MCS_CK(ctx, call)                                                                   \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) {                                                            \
            return ::mcs::set_err((ctx), MCS_ERR_CUDA,                                      \
                                  std::string(#call) + ": " + cudaGetErrorString(e_));      \
        }                                                                                   \
    } while (0)

#define MCS_CK_LAUNCH(ctx) MCS_CK(ctx, cudaGetLastError())

template <typename T>
inline PopView<T> pop_view(mcs_pop* p) {
    PopView<T> v;
    for (int q = 0; q < 8; ++q) v.f[q] = static_cast<T*>(p->f[q]);
    v.cell = p->cell;
    v.act = p->act;
    v.n_in = p->d_n + p->cur;
    v.n_out = p->d_n + (p->cur ^ 1);
    v.cap = p->cap;
    return v;
}

// Julia's LinRange arithmetic, which MCStreamer's Grid relies on (grid.jl:33-41): getindex
// r[j+1] = lerpi(j, lendiv, start, stop) = (1 - j/lendiv) start + (j/lendiv) stop, and
// step(r) = (stop - start) / lendiv with lendiv = max(1, len - 1).
inline double lerpi(long long j, long long d, double a, double b) {
    const double t = (double)j / (double)d;
    return (1.0 - t) * a + t * b;
}

// The cell-centre range of one axis: faces f = LinRange(0, len, m + 1) and
// c = 0.5 * (f[2:end] + f[1:end-1]), a LinRange from 0.5 (f[2] + f[1]) to 0.5 (f[m+1] + f[m])
// of m points.  Returns its first and last point and step(c) (dr(grid) / dz(grid)).
inline void centre_range(double len, int m, double* first, double* last, double* step) {
    const double f1 = lerpi(0, m, 0.0, len), f2 = lerpi(1, m, 0.0, len);
    const double fm = lerpi(m - 1, m, 0.0, len), fm1 = lerpi(m, m, 0.0, len);
    *first = 0.5 * (f2 + f1);
    *last = 0.5 * (fm1 + fm);
    *step = (*last - *first) / (double)(m > 1 ? m - 1 : 1);
}

// Same arithmetic as the oracle's Yoshida constants (JuMC/src/electron.jl:38-46).
struct YoshidaHost {
    double c1, c2, c3, c4, d1, d2, d3;
    YoshidaHost() {
        const double cb = std::pow(2.0, 1.0 / 3.0);
        const double w0 = -cb / (2.0 - cb);
        const double w1 = 1.0 / (2.0 - cb);
        c1 = w1 / 2.0;
        c2 = (w0 + w1) / 2.0;
        c3 = c2;
        c4 = c1;
        d1 = w1;
        d2 = w0;
        d3 = d1;
    }
};

inline StepCtl step_ctl(mcs_pop* p, double dt, uint32_t tag, double* moments_out) {
    mcs_ctx* c = p->ctx;
    StepCtl s;
    s.seed = p->seed;
    s.step = p->step;
    s.tag = tag;
    s.flags = c->flags;
    c->epoch += 1;
    if ((c->epoch & 0x3fffffffu) == 0) c->epoch += 1;
    s.epoch = c->epoch;
    s.status = c->d_status;
    s.tile_status = p->tile_status;
    s.counters = p->counters;
    s.tile_partials = p->tile_partials;
    s.moments_out = moments_out;
    s.dt = dt;
    s.slot_base = p->slot_base;
    s.photo = p->photo;
    s.inj_u = p->inj ? p->d_inj_u : nullptr;
    s.inj_pos = p->inj ? p->d_inj_pos : nullptr;
    s.inj_end = p->inj ? p->d_inj_end : nullptr;
    s.inj_n = p->inj ? p->inj_n : 0;
    return s;
}

inline GridView grid_view(const mcs_grid* g) {
    if (!g) {
        GridView v{};
        v.type = 0;
        return v;
    }
    return g->v;
}

// Persistent grid: enough CTAs to fill the GPU, never more than there can be tiles.
template <typename K>
inline int persistent_grid(mcs_ctx* c, K kernel, int block, long long max_tiles) {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, block, 0) != cudaSuccess || occ < 1) occ = 1;
    long long g = (long long)occ * c->num_sms;
    if (g > max_tiles) g = max_tiles;
    if (g < 1) g = 1;
    return (int)g;
}

// Launch functions defined per precision translation unit.
template <typename T>
int launch_step_abs(mcs_pop* p, const mcs_table* t, const mcs_field* f, double dt, mcs_grid* trk,
                    double* moments_out);
template <typename T>
int launch_step_mesh(mcs_pop* p, const mcs_table* t, double dt, bool tracking, double dep_val, double* moments_out);
template <typename T>
int launch_collisions(mcs_pop* p, const mcs_table* t, double dt, mcs_grid* trk);

}  // namespace mcs
