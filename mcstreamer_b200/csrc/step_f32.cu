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
template <>
int launch_step_mesh<float>(mcs_pop* p, const mcs_table* t, double dt, bool tracking, double dep_val, double* mom) {
    return launch_step_mesh_impl<float, 256, 8, 3>(p, t, dt, tracking, dep_val, mom);
}
}  // namespace mcs
