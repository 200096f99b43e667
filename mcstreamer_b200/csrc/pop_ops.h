// pop_ops.h -- launchers of the population-level kernels (pop_ops.cu).
#pragma once
#include <cmath>

#include "mcs_device.cuh"
#include "mcs_internal.h"

namespace mcs {
int launch_scan(mcs_pop* p, const uint32_t* in, uint32_t* out, const long long* n_dev, long long* total);
int launch_repack(mcs_pop* p);
int launch_swarm_resample(mcs_pop* p, long long n0, double tol);
int launch_moments(mcs_pop* p, const mcs_table* t, double* d_out, int nm);
int launch_deposit(mcs_pop* p, mcs_grid* g, double val);
// w_lossy (device word, optional) is set to 1 when some uploaded weight changes in the
// population's precision (FP32 only), so that a download must bring the weights back.
int launch_upload(mcs_pop* p, const double* dx, const double* dv, const double* dw, const double* ds,
                  const uint8_t* da, long long n, unsigned int* w_lossy = nullptr);
int launch_download(mcs_pop* p, double* dx, double* dv, double* dw, double* ds, uint8_t* da);
int grid_for(mcs_ctx* c, long long n, int block);
int launch_init_maxwellian(mcs_pop* p, long long n, double sigma);
int launch_init_cloud(mcs_pop* p, long long n, const double c[3], double sigma, double vabs, double wmin, double wmax);
int launch_efield_gaussian(mcs_grid* g, const double c[3], double sigma, double rho_peak, const double eb[3]);
// Standard deviation of each velocity component of a Maxwellian with mean energy mean_ev.
inline double maxwellian_sigma(double mean_ev) {
    return sqrt((2.0 / 3.0) * mean_ev * kElementaryCharge / kElectronMass);
}
int map_status(uint32_t st);
const char* status_text(int code);
// Wait for the context's stream and turn the sticky device status into an error code.
int sync_status(mcs_ctx* c);
// The slot of the population's per-step sums for its next step (nullptr: no log).
double* log_slot(mcs_pop* p);
// (threads per block, particles per thread, CTAs per SM) of an FP32 mesh-step shape.
int mesh_shape_info(int shape, int* block, int* ppt, int* minb);
// The population's second set of arrays (cap slots), allocated on first use.
int reserve_alt(mcs_pop* p);
// That and the per-tile tables of the mesh step's secondary pool.
int reserve_mesh_pool(mcs_pop* p);
constexpr int kMomentPartialsMin = 148 * 2 * (MCS_MOMENTS_BASE + kMaxRows);
}  // namespace mcs
