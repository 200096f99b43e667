// step_f64.cu -- FP64 instantiations of the step kernels.  Built with -fmad=false so the
// arithmetic is the reference's unfused sequence (parity mode).
#include "step_launch.cuh"

namespace mcs {
template <>
int launch_step_abs<double>(mcs_pop* p, const mcs_table* t, const mcs_field* f, double dt, mcs_grid* trk,
                            double* mom) {
    return launch_step_abs_impl<double, 128, 1>(p, t, f, dt, trk, mom);
}
template <>
int launch_collisions<double>(mcs_pop* p, const mcs_table* t, double dt, mcs_grid* trk) {
    return launch_collisions_impl<double, 128, 1>(p, t, dt, trk);
}
template <>
int launch_step_mesh<double>(mcs_pop* p, const mcs_table* t, double dt, bool tracking, double dep_val, double* mom) {
    return launch_step_mesh_impl<double, 128, 8>(p, t, dt, tracking, dep_val, mom);
}
}  // namespace mcs
