// step_launch.cuh -- host launchers of the step kernels, instantiated per precision by
// step_f32.cu and step_f64.cu.
#pragma once
#include <type_traits>

#include "host_util.h"
#include "pop_ops.h"
#include "step_kernel.cuh"

namespace mcs {

// Secondary staging of one launch: `grid` CTAs, each with room for 4*TILE + 2048 entries
// (eight or more secondaries per particle and step before MCS_ERR_OVERFLOW).
template <typename T, int TILE>
int attach_stage(mcs_pop* p, int grid, StepCtl& C) {
    const uint32_t cap = 4 * TILE + 2048;
    const size_t stride = ((size_t)cap * (8 * sizeof(T) + 9) + 255) & ~(size_t)255;
    const size_t bytes = stride * (size_t)grid;
    if (p->stage_bytes < bytes) {
        if (p->stage) cudaFree(p->stage);
        p->stage = nullptr;
        p->stage_bytes = 0;
        cudaError_t e = cudaMalloc(&p->stage, bytes);
        if (e != cudaSuccess) return set_err(p->ctx, MCS_ERR_NOMEM, std::string("staging: ") + cudaGetErrorString(e));
        p->stage_bytes = bytes;
    }
    C.stage = static_cast<char*>(p->stage);
    C.stage_stride = stride;
    C.stage_cap = cap;
    return MCS_OK;
}

template <typename T, int BLOCK, int PPT, class Field, bool CLOSED, class Ev = Event>
int launch_abs_variant(mcs_pop* p, const mcs_table* t, const GridView& fg, const GridView& tg, const Field& fld,
                       double dt, double ax, double ay, double az, double* mom) {
    if constexpr (std::is_same<Ev, Event>::value) {
        if (p->inj)   // the same kernel reading the caller's uniforms (mcs_set_uniform_source)
            return launch_abs_variant<T, BLOCK, PPT, Field, CLOSED, EventInj>(p, t, fg, tg, fld, dt, ax, ay, az, mom);
    }
    mcs_ctx* c = p->ctx;
    constexpr int TILE = BLOCK * PPT;
    auto kern = k_step_abs<T, BLOCK, PPT, Field, CLOSED, Ev>;
    const long long max_tiles = (p->cap + TILE - 1) / TILE;
    const int grid = persistent_grid(c, kern, BLOCK, max_tiles);
    YoshidaHost yh;
    YoshidaC Y{yh.c1, yh.c2, yh.c3, yh.c4, yh.d1, yh.d2, yh.d3, (-kElementaryCharge) / kElectronMass};
    StepCtl C = step_ctl(p, dt, TAG_ADVANCE, mom);
    if (int st = attach_stage<T, TILE>(p, grid, C)) return st;
    kern<<<grid, BLOCK, 0, c->stream>>>(pop_view<T>(p), t->v, fg, tg, C, fld, Y, ax, ay, az);
    MCS_CK_LAUNCH(c);
    return MCS_OK;
}

template <typename T, int BLOCK, int PPT>
int launch_step_abs_impl(mcs_pop* p, const mcs_table* t, const mcs_field* f, double dt, mcs_grid* trk,
                         double* mom) {
    const GridView tg = grid_view(trk);
    const double qm = (-kElementaryCharge) / kElectronMass;
    if (f->type == FIELD_UNIFORM) {
        FieldUniform fu{f->e[0], f->e[1], f->e[2]};
        const GridView none = grid_view(nullptr);
        if constexpr (sizeof(T) == 4)
            return launch_abs_variant<T, BLOCK, PPT, FieldUniform, true>(p, t, none, tg, fu, dt, qm * f->e[0],
                                                                         qm * f->e[1], qm * f->e[2], mom);
        else
            return launch_abs_variant<T, BLOCK, PPT, FieldUniform, false>(p, t, none, tg, fu, dt, 0, 0, 0, mom);
    }
    const GridView fg = grid_view(f->grid);
    if (f->grid->v.type == GRID_CYL)
        return launch_abs_variant<T, BLOCK, PPT, FieldCyl, false>(p, t, fg, tg, FieldCyl{}, dt, 0, 0, 0, mom);
    return launch_abs_variant<T, BLOCK, PPT, FieldCartAbs, false>(p, t, fg, tg, FieldCartAbs{}, dt, 0, 0, 0, mom);
}

template <typename T, int BLOCK, int PPT, int MINB = 1, int REFILL = 8>
int launch_step_mesh_impl(mcs_pop* p, const mcs_table* t, double dt, bool tracking, double dep_val, double* mom) {
    mcs_ctx* c = p->ctx;
    if (p->inj) return set_err(c, MCS_ERR_UNSUPPORTED, "injected uniforms on a mesh-layout population");
    constexpr int TILE = BLOCK * PPT;
    auto kern = k_step_mesh<T, BLOCK, PPT, MINB, REFILL>;
    const int grid = persistent_grid(c, kern, BLOCK, (p->cap + TILE - 1) / TILE);
    YoshidaHost yh;
    YoshidaC Y{yh.c1, yh.c2, yh.c3, yh.c4, yh.d1, yh.d2, yh.d3, (-kElementaryCharge) / kElectronMass};
    StepCtl C = step_ctl(p, dt, TAG_ADVANCE, mom);
    if (int st = attach_stage<T, TILE>(p, grid, C)) return st;
    if (int st = reserve_mesh_pool(p)) return st;
    for (int q = 0; q < 8; ++q) C.pool_f[q] = p->alt[q];
    C.pool_cell = p->alt_cell;
    C.pool_act = p->alt_act;
    C.pool_top = reinterpret_cast<unsigned long long*>(p->counters + 16);
    C.app_cnt = p->app_cnt;
    C.app_off = p->app_off;
    const PopView<T> P = pop_view<T>(p);
    kern<<<grid, BLOCK, 0, c->stream>>>(P, t->v, p->cells->v, tracking ? 1 : 0, C, Y, dep_val);
    MCS_CK_LAUNCH(c);
    k_pool_scan<1024><<<1, 1024, 0, c->stream>>>(P.n_in, P.n_out, P.cap, TILE, p->app_cnt, p->app_excl, C.pool_top,
                                                C.status);
    MCS_CK_LAUNCH(c);
    k_pool_copy<T><<<c->num_sms * 8, 128, 0, c->stream>>>(P, C, TILE, p->app_excl);
    MCS_CK_LAUNCH(c);
    return MCS_OK;
}

template <typename T, int BLOCK, int PPT, class Ev = Event>
int launch_collisions_impl(mcs_pop* p, const mcs_table* t, double dt, mcs_grid* trk) {
    if constexpr (std::is_same<Ev, Event>::value) {
        if (p->inj) return launch_collisions_impl<T, BLOCK, PPT, EventInj>(p, t, dt, trk);
    }
    mcs_ctx* c = p->ctx;
    constexpr int TILE = BLOCK * PPT;
    auto kern = k_collisions<T, BLOCK, PPT, Ev>;
    const int grid = persistent_grid(c, kern, BLOCK, (p->cap + TILE - 1) / TILE);
    StepCtl C = step_ctl(p, dt, TAG_COLLISIONS, nullptr);
    if (int st = attach_stage<T, TILE>(p, grid, C)) return st;
    kern<<<grid, BLOCK, 0, c->stream>>>(pop_view<T>(p), t->v, grid_view(trk), C);
    MCS_CK_LAUNCH(c);
    return MCS_OK;
}

}  // namespace mcs
