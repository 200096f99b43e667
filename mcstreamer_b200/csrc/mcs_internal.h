// mcs_internal.h -- host-side objects behind the opaque handles of include/mcs.h and the
// plain-data views that kernels receive by value.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/mcs.h"

namespace mcs {

constexpr int kMaxRows = 32;      // table rows (processes incl. null)
constexpr int kStepMoments = 12;  // fused per-step moments, see StepMoment
// device counter words of a population: [0..1] step tiles, [2..3] scan, [4..7] repack and
// swarm resample, [8..9] sort, [10..15] resample, [16..17] the mesh step's secondary pool
constexpr int kCounterWords = 32;
enum StepMoment { SM_COUNT = 0, SM_W, SM_X, SM_Y, SM_Z, SM_XX, SM_YY, SM_ZZ, SM_VX, SM_VY, SM_VZ, SM_E };

enum GridType { GRID_CART3D = 1, GRID_CYL = 2 };
enum FieldType { FIELD_UNIFORM = 0, FIELD_GRID = 1 };

// ---- kernel-side views (trivially copyable) ----
struct TableView {
    const double* rate64;   // [neps][nrows]
    const float* rate32;    // [neps][nrp]: the total real rate, then the rows (nrp = nrows + 1 rounded up to 4)
    int nrows, nrp, neps;
    double e0, emax, step, maxrate, inv_maxrate;
    float ke32, e0n32, maxrate32;  // u = v^2*ke32 - e0n32 in grid units
    int kind[kMaxRows];
    double param[kMaxRows];
    // PhotoEmission rows (electron.jl:88-105): log(nu_min), log(nu_max) per row,
    // photon_multiplier, photon_weight; has_pe = 0 when the table has no such row
    int has_pe;
    double pe_mult, pe_pw;
    double pe_lmin[kMaxRows], pe_lmax[kMaxRows];
};

// One photo-emission event of a step: `nphot` photons of parent slot `slot` (local to the
// launch), collision event `jev`, at positions [poff, poff + nphot) among that parent's
// photons of the step.
struct PhotoEvent {
    double x, y, z;
    uint32_t slot, jev, poff, nphot;
    int row;
    uint32_t act;
};

// Where a step kernel records photo-emission (all null: photo-emission is unsupported).
struct PhotoOut {
    PhotoEvent* events;
    uint32_t* count;     // events recorded (device counter)
    uint32_t cap;        // events room
    uint32_t* per_slot;  // photons per parent slot (n_entry entries)
};

// Unsigned 32-bit division by an invariant divisor with one multiply-high (Granlund &
// Montgomery, "Division by invariant integers using multiplication", PLDI 1994, fig. 4.1):
// q = (t + ((n - t) >> s1)) >> s2 with t = umulhi(m, n), exact for every n < 2^32.
struct FastDiv {
    uint32_t d, m, s1, s2;
};
inline FastDiv make_fastdiv(uint32_t d) {
    int l = 0;
    while (l < 32 && (1ull << l) < d) ++l;   // ceil(log2 d)
    FastDiv f;
    f.d = d;
    f.m = (uint32_t)((((1ull << 32) * ((1ull << l) - d)) / d + 1) & 0xffffffffull);
    f.s1 = l < 1 ? (uint32_t)l : 1u;
    f.s2 = l > 1 ? (uint32_t)(l - 1) : 0u;
    return f;
}
#ifdef __CUDACC__
__device__ __forceinline__ uint32_t fast_div(uint32_t n, const FastDiv& f) {
    const uint32_t t = __umulhi(f.m, n);
    return (t + ((n - t) >> f.s1)) >> f.s2;
}
#endif

struct GridView {
    int type;               // 0 none, GRID_CART3D, GRID_CYL
    int nx, ny, nz;         // cart3d cells
    FastDiv dnx, dny;       // division by nx, ny (cell index -> ix, iy, iz)
    double h, inv_h, x0, y0, z0;
    const float* e32;       // cart3d node field, 4 floats per node (Ex,Ey,Ez,0)
    const double* e64;      // cart3d node field, 3 doubles per node
    double R, L, dr, dz;    // cyl: R / M, L / N (step(grid.rf), step(grid.zf): cellindex)
    double drc, dzc;        // cyl: step(grid.rc), step(grid.zc) in Julia's LinRange arithmetic (FieldInterp, dV)
    double rc0, rc1;        // cyl: first and last cell centre of grid.rc (rc[i] by lerpi, for dV)
    int M, N;
    const double* er; const double* ez;  // cyl faces (M+3)x(N+3)
    const float* er32; const float* ez32;  // their FP32 copies (the FP32 push gathers these)
    float R32, L32, inv_dr32, inv_dz32;
    long long* qfixed;      // tracker deposits (int64, 2^-32 e)
    long long* qpart;       // particle deposits
};

#ifdef __CUDACC__
// Linear cell index -> (ix, iy, iz), x fastest.
__device__ __forceinline__ void cell_split(const GridView& g, uint32_t cell, uint32_t& ix, uint32_t& iy, uint32_t& iz) {
    const uint32_t r = fast_div(cell, g.dnx);
    ix = cell - r * (uint32_t)g.nx;
    iz = fast_div(r, g.dny);
    iy = r - iz * (uint32_t)g.ny;
}
#endif

template <typename T>
struct PopView {
    T* f[8];                // x y z vx vy vz w s   (mesh layout: ox oy oz = in-cell offsets)
    uint32_t* cell;         // mesh layout only
    uint8_t* act;
    const long long* n_in;  // particles at entry
    long long* n_out;       // particles at exit (double-buffered count)
    long long cap;
};

struct StepCtl {
    unsigned long long seed;
    uint32_t step, tag, flags, epoch;
    uint32_t* status;         // sticky status word
    unsigned long long* tile_status;
    uint32_t* counters;       // [0] tile ticket, [1] CTA done count (kCounterWords words)
    double* tile_partials;    // [tile][kStepMoments]
    double* moments_out;      // kStepMoments doubles or nullptr
    double dt;
    char* stage;              // per-CTA secondary staging, stage_stride bytes per CTA
    unsigned long long stage_stride;
    uint32_t stage_cap;       // entries per CTA
    uint32_t slot_base;       // added to the slot index that keys a particle's random stream
    PhotoOut photo;           // photo-emission output (k_step_abs only)
    // injected uniforms (mcs_set_uniform_source): slot i reads inj_u[inj_pos[i] .. inj_end[i])
    const double* inj_u;
    long long* inj_pos;
    const long long* inj_end;
    long long inj_n;          // slots with a range
    // secondary pool of the mesh step: each tile reserves app_cnt[tile] entries at
    // app_off[tile] (from pool_top), in the order of its parents; k_pool_scan/k_pool_copy
    // then append them after the population in tile order
    void* pool_f[8];
    uint32_t* pool_cell;
    uint8_t* pool_act;
    unsigned long long* pool_top;
    uint32_t* app_cnt;
    unsigned long long* app_off;
};

}  // namespace mcs

// ---- opaque handle types ----
struct mcs_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    uint32_t flags = 0;
    int mesh_shape = 0;            // kernel shape of the FP32 mesh step (MCS_OPT_MESH_SHAPE)
    uint32_t* d_status = nullptr;
    uint32_t epoch = 1;
    int num_sms = 148;
    std::string err;
};

struct mcs_table {
    mcs_ctx* ctx = nullptr;
    mcs::TableView v{};
    bool photo_rows = false;   // has MCS_PHOTOEMISSION rows (only mcs_advance_mixed applies them)
    double* d_rate64 = nullptr;
    float* d_rate32 = nullptr;
};

struct mcs_grid {
    mcs_ctx* ctx = nullptr;
    mcs::GridView v{};
    int precision = MCS_FP32;
    float* d_e32 = nullptr;
    double* d_e64 = nullptr;
    double* d_er = nullptr;
    double* d_ez = nullptr;
    float* d_erz32 = nullptr;   // cyl: FP32 er faces then ez faces
    long long* d_q[2] = {nullptr, nullptr};
    size_t nq = 0;          // entries per charge array
    struct mcs_fluid* fluid = nullptr;   // cyl: the electron fluid on this grid, if any
    double* d_qfd = nullptr;  // cyl: FP64 density part of qfixed, (M+2)x(N+2), made on first use
    void* d_init_ws = nullptr;   // initfromfiles! workspace (counts, bases, scan sums), kept
    size_t init_ws_bytes = 0;
    unsigned long long* d_range = nullptr;   // mcs_grid_fixed_plane_range: first, last nonzero node
};

// The electron fluid of MCStreamer (fluid.jl) on a cylindrical grid: density ne and its
// derivative dne with two ghost layers ((M+4)x(N+4), (i, j) at (i+1) + (j+1)(M+4)), double
// buffered for the fused setdne! + euler!.  setneedle! adds to the grid's d_qfd.
struct mcs_fluid {
    mcs_ctx* ctx = nullptr;
    mcs_grid* g = nullptr;
    int M = 0, N = 0;
    double* ne[2] = {nullptr, nullptr};
    int cur = 0;
    double* dne = nullptr;
    long long launches = 0;
};

namespace mcs {
// The grid's FP64 density part of qfixed, allocated (zeroed) on first use; nullptr on failure
// with the context's error set.
double* grid_qfd(mcs_grid* g);
}  // namespace mcs

struct mcs_field {
    mcs_ctx* ctx = nullptr;
    int type = mcs::FIELD_UNIFORM;
    double e[3] = {0, 0, 0};
    mcs_grid* grid = nullptr;
};

namespace mcs { struct HostStepBuffers; void free_host_step(HostStepBuffers*); }

struct mcs_pop {
    mcs::HostStepBuffers* host_step = nullptr;   // cached workspace of mcs_advance_deposit_host
    mcs_ctx* ctx = nullptr;
    int precision = MCS_FP64;
    mcs_grid* cells = nullptr;     // mesh layout when non-null
    long long cap = 0;
    size_t esz = 8;                // bytes per float field
    uint32_t slot_base = 0;        // stream slot of slot 0 (a chunk of a larger population)
    mcs::PhotoOut photo{};         // set by mcs_advance_mixed for the duration of its step
    void* f[8] = {};
    uint32_t* cell = nullptr;
    uint8_t* act = nullptr;
    long long* d_n = nullptr;      // [2] double-buffered count
    int cur = 0;
    unsigned long long seed = 0;
    uint32_t step = 0;
    uint32_t resample_calls = 0;
    // scratch
    unsigned long long* tile_status = nullptr;
    long long max_tiles = 0;
    double* tile_partials = nullptr;
    uint32_t* counters = nullptr;  // kCounterWords words
    double* d_moments = nullptr;   // kStepMoments
    void* staging = nullptr;       // host<->device transfer staging
    size_t staging_bytes = 0;
    uint32_t* u32a = nullptr;      // per-particle scratch (cap)
    uint32_t* u32b = nullptr;      // per-particle scratch (cap)
    void* alt[8] = {};             // permutation double buffer
    uint32_t* alt_cell = nullptr;
    uint8_t* alt_act = nullptr;
    void* stage = nullptr;         // secondary staging of the step kernels
    size_t stage_bytes = 0;
    uint32_t* sort_key[2] = {nullptr, nullptr};   // radix sort ping-pong (cap entries)
    uint32_t* sort_val[2] = {nullptr, nullptr};
    uint32_t* sort_hist = nullptr;                // [256][tiles] counts, then offsets
    uint32_t* sort_hoff = nullptr;
    uint32_t* seg_a = nullptr;                    // resample segment scratch (cap entries)
    uint32_t* seg_b = nullptr;
    uint32_t* app_cnt = nullptr;             // mesh step: secondaries per tile
    unsigned long long* app_off = nullptr;   // their pool offset
    unsigned long long* app_excl = nullptr;  // and their offset after the population
    long long app_tiles = 0;
    double* d_log = nullptr;       // per-step fused moments, log_cap entries of kStepMoments
    int log_cap = 0;
    uint32_t log_step0 = 0;
    // injected uniforms (mcs_set_uniform_source)
    bool inj = false;
    double* d_inj_u = nullptr;
    long long* d_inj_pos = nullptr;   // next value of each slot
    long long* d_inj_end = nullptr;   // end of each slot's range
    long long inj_n = 0;
};
