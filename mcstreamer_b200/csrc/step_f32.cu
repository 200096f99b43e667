// step_f32.cu -- FP32 instantiations of the step kernels (push and collision sampling in
// FP32; time accumulation, deposits and moments in FP64 / int64).
#include "step_launch.cuh"

namespace mcs {
template <>
int launch_step_abs<float>(mcs_pop* p, const mcs_table* t, const mcs_field* f, double dt, mcs_grid* trk,
                           double* mom) {
    return launch_step_abs_impl<float, 256, 2>(p, t, f, dt, trk, mom);
}
template <>
int launch_collisions<float>(mcs_pop* p, const mcs_table* t, double dt, mcs_grid* trk) {
    return launch_collisions_impl<float, 256, 2>(p, t, dt, trk);
}
// Kernel shapes of the FP32 mesh step: (threads per block, particles per thread, resident
// CTAs per SM the register budget is set for).  Shape 0 is the default.
const int kMeshShapes[][3] = {{256, 8, 3}, {256, 8, 4}, {256, 16, 3}, {256, 16, 4},
                              {128, 16, 6}, {128, 16, 8}, {512, 8, 2}, {256, 32, 3}};
constexpr int kNumMeshShapes = sizeof(kMeshShapes) / sizeof(kMeshShapes[0]);
static_assert(kNumMeshShapes == MCS_MESH_SHAPES, "shape table and header disagree");

template <>
int launch_step_mesh<float>(mcs_pop* p, const mcs_table* t, double dt, bool tracking, double dep_val, double* mom) {
    switch (p->ctx->mesh_shape) {
    case 1: return launch_step_mesh_impl<float, 256, 8, 4>(p, t, dt, tracking, dep_val, mom);
    case 2: return launch_step_mesh_impl<float, 256, 16, 3>(p, t, dt, tracking, dep_val, mom);
    case 3: return launch_step_mesh_impl<float, 256, 16, 4>(p, t, dt, tracking, dep_val, mom);
    case 4: return launch_step_mesh_impl<float, 128, 16, 6>(p, t, dt, tracking, dep_val, mom);
    case 5: return launch_step_mesh_impl<float, 128, 16, 8>(p, t, dt, tracking, dep_val, mom);
    case 6: return launch_step_mesh_impl<float, 512, 8, 2>(p, t, dt, tracking, dep_val, mom);
    case 7: return launch_step_mesh_impl<float, 256, 32, 3>(p, t, dt, tracking, dep_val, mom);
    default: return launch_step_mesh_impl<float, 256, 8, 3>(p, t, dt, tracking, dep_val, mom);
    }
}

int mesh_shape_info(int shape, int* block, int* ppt, int* minb) {
    if (shape < 0 || shape >= kNumMeshShapes) return MCS_ERR_ARG;
    *block = kMeshShapes[shape][0];
    *ppt = kMeshShapes[shape][1];
    *minb = kMeshShapes[shape][2];
    return MCS_OK;
}
}  // namespace mcs
