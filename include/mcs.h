/*
 * mcs.h -- C ABI of mcstreamer-b200, the B200 (sm_100a) implementation of JuMC's electron
 * step (aluque/mcstreamer).  Plain pointers and sizes only; every entry point returns an
 * int status (MCS_OK == 0) and mcs_last_error(ctx) gives the message of the last failure.
 *
 * The reference has no FFI: its "plugin API" is Julia multiple dispatch.  Each entry point
 * below names the reference function it replaces (file:line inside the reference project);
 * a Julia caller binds them with ccall.
 *
 * Host buffer layouts equal the Julia memory layouts so Julia arrays pass without copies:
 *   x, v   : 3 doubles per particle, interleaved   (Vector{SVector{3,Float64}})
 *   w, s   : 1 double per particle                 (Vector{Float64})
 *   active : 1 byte per particle (0/1)             (Vector{Bool})
 *   rate   : neps columns of nrows doubles, process index fastest
 *            (CollisionTable.rate, Matrix{Float64} of size (nrows, neps))
 *
 * Work is queued on the context's CUDA stream; calls that return data to the host
 * (download, read, nparticles, moments, mcs_sync) synchronise and report the sticky
 * device status (capacity, energy range, field magnitude, overflow, timeout) raised by
 * earlier queued kernels.  A context is not thread-safe (the reference's advance! is
 * likewise called from one task).
 */
#ifndef MCS_H
#define MCS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MCS_API __attribute__((visibility("default")))

/* ---- status codes ---- */
enum {
    MCS_OK = 0,
    MCS_ERR_ARG = 1,            /* invalid argument */
    MCS_ERR_CUDA = 2,           /* CUDA runtime error */
    MCS_ERR_CAPACITY = 3,       /* "Maximum number of particles reached" (population.jl:90) */
    MCS_ERR_ENERGY_RANGE = 4,   /* energy beyond the table (util.jl:28 @assert 0 <= w <= 1) */
    MCS_ERR_FIELD_TOO_HIGH = 5, /* |E| > 1e8 V/m (gridfields.jl:179-187) */
    MCS_ERR_NONFINITE = 6,      /* NaN / Inf in particle state */
    MCS_ERR_UNSUPPORTED = 7,    /* combination not implemented (e.g. user-defined process) */
    MCS_ERR_OVERFLOW = 8,       /* a tile produced more secondaries than its staging holds */
    MCS_ERR_NOMEM = 9,          /* device allocation failed */
    MCS_ERR_TIMEOUT = 10,       /* a bounded device-side wait gave up */
    MCS_ERR_UNIFORMS = 11,      /* a particle needed more injected uniforms than it was given */
    MCS_ERR_CHARGE_RANGE = 12   /* a charge beyond the int64 fixed-point range of the deposits
                                   (2^-32 e units): |w * val| >= 2^30 e for one particle, or a
                                   node / cell sum of 2^30 e or more (within a factor 2 of the
                                   2^31 e where the sums would wrap) */
};

/* ---- collision process kinds (JuMC/src/electron.jl:70-84, collisions.jl:3) ---- */
enum {
    MCS_NULL = 0,
    MCS_ELASTIC = 1,             /* param = mass_ratio                           */
    MCS_EXCITATION = 2,          /* param = threshold (J)                         */
    MCS_IONIZATION = 3,          /* param = threshold (J), equal energy sharing   */
    MCS_ATTACHMENT = 4,          /* param = threshold (J), unused                 */
    MCS_IONIZATION_UNIFORM = 5,  /* param = threshold (J), secondary energy uniform on
                                    [0, eps - threshold]; no counterpart in JuMC */
    MCS_PHOTOEMISSION = 6        /* PhotoEmission (electron.jl:88-105, 141-144): param unused;
                                    the band and weights by mcs_table_set_photoemission */
};

enum { MCS_FP64 = 0, MCS_FP32 = 1 };

/* context flags */
enum { MCS_FLAG_CLAMP_ENERGY = 1 }; /* energies beyond the table use the last column
                                       instead of raising MCS_ERR_ENERGY_RANGE */

/* charge arrays of a grid */
enum { MCS_Q_FIXED = 0, /* tracker deposits: CollisionTracker -> fields.qfixed */
       MCS_Q_PART = 1   /* particle deposits: density! -> fields.qpart */ };

/* layout of the moments vector filled by mcs_moments (length MCS_MOMENTS_BASE + nrows) */
enum {
    MCS_M_COUNT = 0,   /* number of active particles */
    MCS_M_W = 1,       /* sum w                         (population.jl:114-124 weight) */
    MCS_M_X = 2,       /* sum x, y, z (2..4)            (Swarm.jl:126)              */
    MCS_M_X2 = 5,      /* sum x^2, y^2, z^2 (5..7)      (Swarm.jl:127)              */
    MCS_M_V = 8,       /* sum vx, vy, vz (8..10)        (Swarm.jl:152)              */
    MCS_M_E = 11,      /* sum energy                                               */
    MCS_M_WE = 12,     /* sum w*energy                  (population.jl:136-150)     */
    MCS_M_EMAX = 13,   /* max energy over ALL particles (population.jl:156-158)     */
    MCS_M_WX = 14,     /* sum w*x, w*y, w*z (14..16)    (population.jl:164-183)     */
    MCS_M_WX2 = 17,    /* sum w*|x|^2                                              */
    MCS_MOMENTS_BASE = 18 /* then sum of rate_j(energy) per table row (Swarm.jl:242-248) */
};

typedef struct mcs_ctx mcs_ctx;
typedef struct mcs_table mcs_table;
typedef struct mcs_grid mcs_grid;
typedef struct mcs_field mcs_field;
typedef struct mcs_pop mcs_pop;
typedef struct mcs_batch mcs_batch;
typedef struct mcs_poisson mcs_poisson;
typedef struct mcs_fluid mcs_fluid;
typedef struct mcs_photons mcs_photons;

/* ---- context ---- */
MCS_API int mcs_version(void);
/* Creates a context on `device` with its own CUDA stream. */
MCS_API int mcs_ctx_create(int device, mcs_ctx** out);
MCS_API int mcs_ctx_destroy(mcs_ctx* ctx);
MCS_API const char* mcs_last_error(const mcs_ctx* ctx);
/* Use an external CUDA stream (cudaStream_t) instead of the context's own. */
MCS_API int mcs_ctx_set_stream(mcs_ctx* ctx, void* stream);
MCS_API void* mcs_ctx_stream(mcs_ctx* ctx);
MCS_API int mcs_ctx_set_flags(mcs_ctx* ctx, uint32_t flags);
/* Failure-detection self-test (no counterpart in the reference): launches the bounded waits
 * of the ordered-append look-back, in its one-thread and whole-warp forms, on predecessors
 * that never publish, with at most max_spins checks each (1 .. 2^20).  Returns
 * MCS_ERR_TIMEOUT when both waits gave up, raised the status and returned, as every wait in
 * the library does; the context stays usable. */
MCS_API int mcs_diag_wait_timeout(mcs_ctx* ctx, uint32_t max_spins);
/* Tuning options of a context (no counterpart in the reference, which has no kernels).
 * MCS_OPT_MESH_SHAPE selects the kernel shape of the FP32 mesh step (0 .. MCS_MESH_SHAPES-1,
 * 0 = default); every shape computes the same result. */
enum { MCS_OPT_MESH_SHAPE = 1, MCS_MESH_SHAPES = 8 };
MCS_API int mcs_ctx_set_option(mcs_ctx* ctx, int option, int value);
MCS_API int mcs_ctx_get_option(mcs_ctx* ctx, int option, int* value);
/* (threads per block, particles per thread, resident CTAs per SM) of a mesh-step shape. */
MCS_API int mcs_mesh_shape(int shape, int* block, int* ppt, int* min_blocks);
/* Waits for queued work; returns (and clears) the sticky device status. */
MCS_API int mcs_sync(mcs_ctx* ctx);

/* ---- collision table: CollisionTable (JuMC/src/collisions.jl:9-22) as built by
 *      load_lxcat (JuMC/src/lxcat.jl:17-134).  Energy grid LinRange(e0, emax, neps). ---- */
MCS_API int mcs_table_create(mcs_ctx* ctx, int nrows, int neps, double e0, double emax,
                             const double* rate, const int* kind, const double* param,
                             double maxrate, mcs_table** out);
MCS_API int mcs_table_destroy(mcs_table* t);

/* ---- grids ---- */
/* 3-D uniform mesh of nx*ny*nz cubic cells of side h, lower corner (x0,y0,z0).  Node
 * field E: 3 values per node, (nx+1)(ny+1)(nz+1) nodes, x fastest.  Charge: int64 per
 * node at 2^-32 elementary charges (cloud-in-cell).  `precision` selects the device copy
 * of the node field (MCS_FP32 / MCS_FP64). */
MCS_API int mcs_grid_create_cart3d(mcs_ctx* ctx, int nx, int ny, int nz, double h, double x0,
                                   double y0, double z0, int precision, mcs_grid** out);
/* Cylindrical Grid(R, L, M, N) (MCStreamer/src/grid.jl:4-42).  Face fields er, ez of
 * (M+3)x(N+3) doubles indexed i + j*(M+3) (calloc_faces, grid.jl:71-72).  Charge arrays
 * are cell densities (M+2)x(N+2), index i + j*(M+2) (calloc_centers, grid.jl:55-57). */
MCS_API int mcs_grid_create_cyl(mcs_ctx* ctx, double R, double L, int M, int N, mcs_grid** out);
MCS_API int mcs_grid_destroy(mcs_grid* g);
/* cart3d: 3 doubles per node.  cyl: er followed by ez. */
MCS_API int mcs_grid_set_efield(mcs_grid* g, const double* e);
/* cart3d only: nodes [node0, node0 + count) of the node field (3 doubles per node), so a
 * large field can be streamed from the host in pieces. */
MCS_API int mcs_grid_set_efield_range(mcs_grid* g, int64_t node0, int64_t count, const double* e);
/* Zero a charge array; MCS_Q_FIXED also zeroes qfixed's FP64 density part on a cylindrical grid. */
MCS_API int mcs_grid_zero(mcs_grid* g, int which);
/* int64 at 2^-32 e: per node (cart3d) or per cell, index i + j*(M+2) (cyl). */
MCS_API int mcs_grid_read_fixed(mcs_grid* g, int which, int64_t* out);
/* Overwrite a charge array with host int64 values (layout of mcs_grid_read_fixed). */
MCS_API int mcs_grid_write_fixed(mcs_grid* g, int which, const int64_t* in);
/* cyl: density per cell (weight/dV, poisson.jl:79-81).  cart3d: charge per node in e. */
MCS_API int mcs_grid_read_density(mcs_grid* g, int which, double* out);
/* Device address and entry count of a charge array (int64), for collectives that sum the
 * deposits of several processes (e.g. an NCCL int64 all-reduce). */
MCS_API int mcs_grid_charge_ptr(mcs_grid* g, int which, void** dptr, int64_t* count);

/* ---- fields: the `efield` callable of advance! ---- */
/* FixedField (Swarm/src/Swarm.jl:28-32), generalised to any constant vector. */
MCS_API int mcs_field_uniform(mcs_ctx* ctx, double ex, double ey, double ez, mcs_field** out);
/* FieldInterp (MCStreamer/src/gridfields.jl:89-190) over a grid's stored field. */
MCS_API int mcs_field_from_grid(mcs_grid* g, mcs_field** out);
MCS_API int mcs_field_destroy(mcs_field* f);

/* ---- population: Population (JuMC/src/population.jl:4-36, 26-36) ---- */
/* `cells` = a cart3d grid stores positions as (cell index, in-cell offset) on that mesh;
 * NULL stores absolute positions. */
MCS_API int mcs_pop_create(mcs_ctx* ctx, int64_t capacity, int precision, mcs_grid* cells,
                           mcs_pop** out);
MCS_API int mcs_pop_destroy(mcs_pop* p);
/* Philox key and step counter (uniform #k of slot i at step t = Philox(seed; i, t, k/4, tag)). */
MCS_API int mcs_pop_set_seed(mcs_pop* p, uint64_t seed, uint32_t step);
MCS_API int mcs_pop_get_step(mcs_pop* p, uint32_t* step);
MCS_API int mcs_pop_upload(mcs_pop* p, const double* x, const double* v, const double* w,
                           const double* s, const uint8_t* active, int64_t n);
MCS_API int mcs_pop_download(mcs_pop* p, double* x, double* v, double* w, double* s,
                             uint8_t* active, int64_t cap, int64_t* n);
/* Device-to-device copy of a whole population (state, count, Philox key and step): a
 * snapshot / restore point.  Same context, precision and layout; dst capacity >= src's. */
/* Swarm initial condition drawn on the device: n electrons at the origin, weight 1,
 * isotropic Maxwellian velocities of mean energy mean_energy_ev, s = -log(u); every
 * electron's draws come from the population seed and its slot (Philox stream INIT).  The
 * reference starts its swarms on the host (Swarm/src/Swarm.jl:104-106). */
MCS_API int mcs_pop_init_maxwellian(mcs_pop* p, int64_t n, double mean_energy_ev);
/* Streamer initial condition drawn on the device (no counterpart in the reference, which
 * reads it from files: MCStreamer/src/initdens.jl): n electrons in a Gaussian cloud of
 * standard deviation sigma (m) per axis around (cx, cy, cz), speed sqrt(2 E/m) for
 * E = energy_ev in isotropic directions, weights log-uniform on [wmin, wmax], s = -log(u);
 * stored in the population's layout (cell + offset on a mesh; not sorted). */
MCS_API int mcs_pop_init_cloud(mcs_pop* p, int64_t n, double cx, double cy, double cz, double sigma,
                               double energy_ev, double wmin, double wmax);
/* Node field of a Gaussian charge e*rho_peak*exp(-r^2/2 sigma^2) centred at (cx, cy, cz)
 * plus the uniform background (ebx, eby, ebz), from Gauss's law, computed on the device
 * (cart3d grids). */
/* The stored field: cart3d 3 doubles per node (x fastest); cyl the er then the ez faces. */
MCS_API int mcs_grid_read_efield(mcs_grid* g, double* e);
/* Nodes [node0, node0 + count) of a cart3d grid's field (3 doubles each), and of a charge
 * array (int64 at 2^-32 e): a window of a large mesh without copying all of it. */
MCS_API int mcs_grid_read_efield_range(mcs_grid* g, int64_t node0, int64_t count, double* e);
MCS_API int mcs_grid_read_fixed_range(mcs_grid* g, int which, int64_t node0, int64_t count, int64_t* out);
/* The z-planes [z0, z1) of a cart3d grid's charge array that hold a nonzero value (z0 = z1
 * = 0 when all are zero); with mcs_grid_read_fixed_range a caller that keeps the charge on
 * the host moves only that slab (no counterpart in the reference). */
MCS_API int mcs_grid_fixed_plane_range(mcs_grid* g, int which, int64_t* z0, int64_t* z1);
MCS_API int mcs_grid_set_efield_gaussian(mcs_grid* g, double cx, double cy, double cz, double sigma,
                                         double rho_peak, double ebx, double eby, double ebz);
MCS_API int mcs_pop_copy(mcs_pop* dst, const mcs_pop* src);
/* nparticles (population.jl:106): particles in use, active or not. */
MCS_API int mcs_pop_nparticles(mcs_pop* p, int64_t* n);

/* ---- the electron step ---- */
/* advance!(mpopl, efield, dt, tracker) (JuMC/src/mixed_population.jl:24-54) with
 * do_one_collision! (collisions.jl:159-192), collide (electron.jl:108-139), apply!
 * (collisions.jl:96-123) and, when tracker != NULL, CollisionTracker (gridfields.jl:
 * 198-224) depositing +w per ionization and -w per attachment into MCS_Q_FIXED. */
MCS_API int mcs_advance(mcs_pop* p, const mcs_table* t, const mcs_field* f, double dt,
                        mcs_grid* tracker);
/* advance! followed by density!(deposit, val) of the post-step particles, fused in one
 * kernel (the streamer step: push + collide + track + deposit).  Needs a cell-layout
 * population whose mesh is the field, tracker (or NULL) and deposit grid.  Accumulates
 * into MCS_Q_PART. */
MCS_API int mcs_advance_deposit(mcs_pop* p, const mcs_table* t, const mcs_field* f, double dt,
                                mcs_grid* tracker, mcs_grid* deposit, double val);
/* advance!(popl, efield, dt, tracker) + density!(deposit, val) for a population that lives
 * in HOST memory in the Julia layout (x, v as interleaved triples; capacity slots each): the
 * particles [0, *n) are stepped and written back in place, the secondaries appended after
 * them in parent order, *n updated.  The population is cut into `chunks` pieces whose
 * uploads, fused mesh steps and downloads are pipelined over three streams; the result is
 * the same as mcs_pop_upload + mcs_advance_deposit + mcs_pop_download (random streams keyed
 * by global slot, int64 deposits), except that no per-step sums are logged.  p is device
 * workspace for one chunk and its secondaries (capacity >= ceil(n / chunks) plus room); it
 * keeps its staging buffers between calls.  The caller zeroes the deposit grid.  Pinned host
 * memory lets the transfers overlap. */
MCS_API int mcs_advance_deposit_host(mcs_pop* p, const mcs_table* t, const mcs_field* f, double dt,
                                     mcs_grid* tracker, mcs_grid* deposit, double val, double* x, double* v,
                                     double* w, double* s, uint8_t* active, int64_t* n, int64_t capacity,
                                     int chunks);
/* Bytes that the last mcs_advance_deposit_host call on p copied host -> device and device ->
 * host (0 before the first call).  A particle's weight, which the step leaves unchanged, goes
 * back to the host only when some weight of its chunk changed on upload (an FP64 weight that
 * an FP32 population rounds), so the download moves 57 instead of 65 bytes per stepped
 * particle when none did.  No reference counterpart: a transfer figure of the host-resident
 * path. */
MCS_API int mcs_pop_host_step_bytes(const mcs_pop* p, int64_t* h2d, int64_t* d2h);
/* Uniform source of advance! and collisions!.  The reference draws Julia's rand()
 * (JuMC/src/util.jl:5,8,17, collisions.jl:166, mixed_population.jl:48; rand() in a
 * single-threaded run is one serial stream); the library draws counter-based Philox streams
 * (MCS_UNIFORMS_PHILOX, the default).  MCS_UNIFORMS_INJECTED makes the following steps take
 * each particle's draws from caller-given values instead, so that a recorded run of the
 * reference can be replayed particle by particle: slot i < nslots consumes u[offsets[i]],
 * u[offsets[i] + 1], ... (offsets has nslots + 1 entries, u has offsets[nslots] values in
 * (0, 1]) in the order the reference draws them for that particle -- per collision: xi;
 * then elastic and excitation phi, u (randsphere); ionization phi, u, phi, u and the
 * secondary's nextcoll() (MCS_IONIZATION_UNIFORM: its sharing fraction first); attachment
 * and null nothing; then the particle's new nextcoll().  A slot's position carries over to
 * the next step; a particle that needs a value beyond its range (or a slot >= nslots that
 * draws) fails the step with MCS_ERR_UNIFORMS.  The values are copied to the device.
 * Photo-emission keeps its Philox streams; mesh-layout populations and
 * mcs_advance_deposit[_host] reject the mode (MCS_ERR_UNSUPPORTED).  MCS_UNIFORMS_PHILOX
 * (u and offsets ignored) switches back.  Replaces no reference function: it feeds the
 * reference's rand() calls. */
enum { MCS_UNIFORMS_PHILOX = 0, MCS_UNIFORMS_INJECTED = 1 };
MCS_API int mcs_set_uniform_source(mcs_pop* p, int mode, const double* u, const int64_t* offsets,
                                   int64_t nslots);
/* collisions!(mpopl, dt, tracker) (JuMC/src/mixed_population.jl:61-77). */
MCS_API int mcs_collisions(mcs_pop* p, const mcs_table* t, double dt, mcs_grid* tracker);
/* density!(grid, arr, mpopl, Electron, fields, val) (MCStreamer/src/poisson.jl:65-84)
 * into MCS_Q_PART (accumulates; zero it with mcs_grid_zero). */
MCS_API int mcs_deposit(mcs_pop* p, mcs_grid* g, double val);
/* repack! (JuMC/src/population.jl:191-215), same permutation. */
MCS_API int mcs_repack(mcs_pop* p);
/* Swarm.resample!(popl, n0, tol) (Swarm/src/Swarm.jl:193-223). */
MCS_API int mcs_swarm_resample(mcs_pop* p, int64_t n0, double tol);
/* Stable sort of the population by cell key of grid g (out-of-grid particles last). */
MCS_API int mcs_sort_cells(mcs_pop* p, mcs_grid* g);
/* resample!(popl, fields, ntarget, nmax) (MCStreamer/src/resample.jl:7-77). */
MCS_API int mcs_resample_cells(mcs_pop* p, mcs_grid* g, int ntarget, int nmax);
/* Allocates now, for the population's capacity, the device scratch that mcs_sort_cells and
 * mcs_resample_cells otherwise allocate on their first call (several GB for 1e8 slots), so
 * that a time-stepping loop does not pay it inside a step.  No counterpart in the reference. */
MCS_API int mcs_resample_reserve(mcs_pop* p);
/* Moments over the population (layout MCS_M_*), table may be NULL (no rate sums). */
MCS_API int mcs_moments(mcs_pop* p, const mcs_table* t, double* out, int nout);

/* Allocation-free moments.  No counterpart in the reference: an addition for callers that
 * must not allocate device memory when they ask for diagnostics -- e.g. a simulation loop
 * held to a memory budget fixed at start-up, or a host application whose own allocator
 * owns every device byte -- and that keep the particles in their own device arrays.
 * arrays[0..6] = x, y, z, vx, vy, vz, w (device, float or double per `precision`), active =
 * device bytes, n particles with absolute positions; writes the MCS_MOMENTS_BASE sums of
 * layout MCS_M_* to moments_out (device) on `stream` (a cudaStream_t, NULL = default) of
 * `device`.  It calls no allocator: its partial sums live in a fixed array inside the
 * library (about 1.2 MB per device that loads it, kept until exit), so n is limited to
 * MCS_NOALLOC_MAX_PARTICLES and larger n returns MCS_ERR_ARG.  The first call on a device
 * looks up that array's device address; make it before capturing a stream.  All calls
 * share the array: calls that overlap on the GPU race and must be serialised. */
#define MCS_NOALLOC_MAX_PARTICLES 67108864LL
MCS_API int mcs_moments_noalloc(int device, void* stream, int precision, const void* const* arrays,
                                const uint8_t* active, int64_t n, double* moments_out);

/* Per-step moments of the fused swarm loop (MCS_STEP_MOMENTS doubles per step). */
enum {
    MCS_S_COUNT = 0, MCS_S_W = 1, MCS_S_X = 2 /* 2..4 */, MCS_S_X2 = 5 /* 5..7 */,
    MCS_S_V = 8 /* 8..10 */, MCS_S_E = 11, MCS_STEP_MOMENTS = 12
};
/* The time loop of Swarm.swarm (Swarm/src/Swarm.jl:124-142) on the device: per step
 * advance! with the per-step sums of Swarm.jl:126-127 fused into the step kernel, then
 * (n0 > 0) Swarm.resample!(popl, n0, tol), then (repack_every > 0, every repack_every
 * steps) repack!.  The reference never repacks a swarm -- its roulette leaves holes and
 * the run stops at 0.9 maxp (Swarm.jl:139-141) -- so repack_every = 0 is its behaviour;
 * repacking keeps long runs inside a small capacity.  moments_out (host, may be NULL)
 * receives nsteps*MCS_STEP_MOMENTS doubles; they stay on the device until the loop ends. */
MCS_API int mcs_swarm_run(mcs_pop* p, const mcs_table* t, const mcs_field* f, double dt, int nsteps,
                          int64_t n0, double tol, int repack_every, double* moments_out);
/* Per-step diagnostics log (the sums MCStreamer reports every step, main.jl:269-279):
 * with capacity > 0 every following advance! writes the MCS_STEP_MOMENTS sums of its
 * post-step population into slot (steps since enabling) % capacity on the device;
 * capacity 0 disables it.  read copies slots [0, nsteps) to the host. */
MCS_API int mcs_pop_step_log(mcs_pop* p, int capacity);
MCS_API int mcs_pop_read_step_log(mcs_pop* p, double* out, int nsteps);

/* ---- Batched swarms: many independent Swarm.swarm solves on one GPU -----------------
 * Replaces the per-solve driver loop of Swarm/src/Swarm.jl:114-150 (one population, one
 * E/N point, one gas per call) for a caller that runs many of them (E/N sweeps, gas
 * mixtures, replicas).  Every instance is an FP32 swarm in a uniform field E with its own
 * collision table, seed and resampling target; a step advances all of them with the
 * sequence advance! -> Swarm.resample!(n0, tol) -> repack! that mcs_swarm_run(...,
 * repack_every = 1) applies to one population, and each instance's particles evolve
 * bit-identically to that single run with the same table, field and seed.
 * Instances join (add) and leave (remove) between steps.  Per-step sums of every instance
 * (MCS_BATCH_MOMENTS doubles: the MCS_STEP_MOMENTS sums, then the sum over actives of the
 * rate of the table's first ionization row and of its square) stay on the device in a
 * ring of MCS_BATCH_LOG steps. */
enum { MCS_BATCH_MOMENTS = 14, MCS_BATCH_LOG = 64, MCS_BATCH_VARIANTS = 22 };
MCS_API int mcs_batch_create(mcs_ctx* ctx, int max_instances, int64_t total_capacity, mcs_batch** out);
MCS_API int mcs_batch_destroy(mcs_batch* b);
/* Join: n particles in Julia layout (x, v as n x 3 row-major), region of `capacity` slots. */
MCS_API int mcs_batch_add(mcs_batch* b, const mcs_table* t, double ex, double ey, double ez, uint64_t seed,
                          int64_t n0, double tol, int64_t capacity, const double* x, const double* v,
                          const double* w, const double* s, const uint8_t* active, int64_t n, int* slot);
/* Join with electrons drawn on the device (no host data, no host wait): n electrons at the
 * origin with weight 1 and isotropic Maxwellian velocities of mean energy mean_energy_ev,
 * the same electrons mcs_pop_init_maxwellian draws for a population with this seed. */
MCS_API int mcs_batch_add_maxwellian(mcs_batch* b, const mcs_table* t, double ex, double ey, double ez,
                                     uint64_t seed, int64_t n0, double tol, int64_t capacity, int64_t n,
                                     double mean_energy_ev, int* slot);
/* Leave (stream-ordered: steps already enqueued still advance the instance). */
MCS_API int mcs_batch_remove(mcs_batch* b, int slot);
/* Double-buffered diagnostics without stalling the stream: enqueue copies of every slot's
 * ring, logged-step counts and the status word into pinned buffer buf (0 or 1), then wait
 * for them later; the pointers stay valid until the next enqueue into the same buffer. */
MCS_API int mcs_batch_logs_enqueue(mcs_batch* b, int buf);
MCS_API int mcs_batch_logs_wait(mcs_batch* b, int buf, const double** ring, const uint32_t** logpos);
/* nsteps batched steps of length dt on the context's stream; use_graph replays one captured
 * CUDA graph per step (re-captured when dt, the context flags or the variant change). */
MCS_API int mcs_batch_step(mcs_batch* b, double dt, int nsteps, int use_graph);
MCS_API int mcs_batch_sync(mcs_batch* b);
/* Per-instance particle counts and completed steps (arrays of max_instances; NULL skips). */
MCS_API int mcs_batch_state(mcs_batch* b, int64_t* n, uint32_t* steps);
/* The sums of every slot's most recent step (max_instances x MCS_BATCH_MOMENTS), one copy. */
MCS_API int mcs_batch_read_current(mcs_batch* b, double* out);
/* Every slot's ring of per-step sums (max_instances x MCS_BATCH_LOG x MCS_BATCH_MOMENTS;
 * step t of a slot sits at t % MCS_BATCH_LOG) and its count of logged steps. */
MCS_API int mcs_batch_read_logs(mcs_batch* b, double* ring, uint32_t* logpos);
/* The last `count` (<= MCS_BATCH_LOG) per-step sums of an instance, oldest first. */
MCS_API int mcs_batch_read_log(mcs_batch* b, int slot, double* out, int count);
MCS_API int mcs_batch_download(mcs_batch* b, int slot, double* x, double* v, double* w, double* s,
                               uint8_t* active, int64_t capacity, int64_t* n_out);
/* Time each (threads per block, particles per thread) variant of the batched step over
 * trial_steps steps of the current state (restored afterwards) and keep the fastest. */
MCS_API int mcs_batch_autotune(mcs_batch* b, double dt, int trial_steps, int* chosen, float* times_ms);
/* nsteps steps without the graph, timing (CUDA events on the context's stream) the
 * persistent advance! kernel and the whole step; per-step averages in ms. */
MCS_API int mcs_batch_profile(mcs_batch* b, double dt, int nsteps, float* kernel_ms, float* step_ms);
MCS_API int mcs_batch_set_variant(mcs_batch* b, int variant);
MCS_API int mcs_batch_variant_shape(int variant, int* block, int* ppt);
/* Resident CTAs per SM the variant's register budget is set for (1 = compiler's choice). */
MCS_API int mcs_batch_variant_min_blocks(int variant, int* min_blocks);
/* Idle lanes (of 32) at which the variant's particle queue writes back and refills. */
MCS_API int mcs_batch_variant_refill(int variant, int* idle_lanes);

/* ---- photons: PhotonState (JuMC/src/photon.jl:11-18) and photo-emission ----
 * PhotoEmission rows of a table (kind MCS_PHOTOEMISSION; electron.jl:88-105, lxcat.jl:86-93):
 * log(nu_min), log(nu_max) per row (1/s; other rows ignored), photon_multiplier and
 * photon_weight.  Required before a table with such rows is used. */
MCS_API int mcs_table_set_photoemission(mcs_table* t, const double* log_numin, const double* log_numax,
                                        double photon_multiplier, double photon_weight);
/* A photon population of `capacity` photons in FP64 whose collisions run at maxrate numax
 * (ZhelezniakCollisions(numax), photon.jl:27-37; MCStreamer/src/main.jl:115-121). */
MCS_API int mcs_photons_create(mcs_ctx* ctx, int64_t capacity, double numax, uint64_t seed, mcs_photons** out);
MCS_API int mcs_photons_destroy(mcs_photons* ph);
/* Julia layout: x, v interleaved triples, nu, w, s one double each, active one byte. */
MCS_API int mcs_photons_upload(mcs_photons* ph, const double* x, const double* v, const double* nu,
                               const double* w, const double* s, const uint8_t* active, int64_t n);
MCS_API int mcs_photons_download(mcs_photons* ph, double* x, double* v, double* nu, double* w, double* s,
                                 uint8_t* active, int64_t capacity, int64_t* n_out);
MCS_API int mcs_photons_count(mcs_photons* ph, int64_t* n);
/* dst <- src on the device (a snapshot of a photon population). */
MCS_API int mcs_photons_copy(mcs_photons* dst, const mcs_photons* src);
/* out[0] = actives(photons), out[1] = weight(photons) (JuMC/src/population.jl:114-131, as
 * MCStreamer's per-step diagnostics read them, main.jl:272-273): FP64 sums over the active
 * photons in a fixed order. */
MCS_API int mcs_photons_moments(mcs_photons* ph, double* out);
/* repack!(photons) (JuMC/src/population.jl:191-215): the inactive photons removed with the
 * reference's permutation (the k-th hole filled from the k-th active counted from the end). */
MCS_API int mcs_photons_repack(mcs_photons* ph);
/* Device times (ms) of the last mixed advance's photon kernels and the photons they handled:
 * the emission of the new photons and the photon step. */
MCS_API int mcs_photons_last_timing(mcs_photons* ph, float* emit_ms, int64_t* emitted, float* step_ms,
                                    int64_t* stepped);
/* advance!(mpopl, efield, dt, tracker) over electrons and photons (mixed_population.jl:24-54):
 * the electrons (absolute positions), whose photo-emission adds photons in serial parent
 * order, then every photon (the new ones too): straight flight, photo-ionization adding +w
 * to the tracker and an electron at rest, appended in serial photon order. */
MCS_API int mcs_advance_mixed(mcs_pop* electrons, mcs_photons* photons, const mcs_table* t, const mcs_field* f,
                              double dt, mcs_grid* tracker);
/* The photon half of mcs_advance_mixed alone. */
MCS_API int mcs_photon_advance(mcs_photons* photons, mcs_pop* electrons, double dt, mcs_grid* tracker);

/* ---- Poisson solve: poisson! (MCStreamer/src/poisson.jl:6-58) on a cylindrical grid ----
 * The multigrid is Multigrid.solve (Multigrid/src/Multigrid.jl:449-467) with MCStreamer's
 * MGConfig (MCStreamer/src/main.jl:131-144): bc Left/Right/Top Dirichlet, Bottom (axis)
 * Neumann, CylindricalConnector{1}, g = 1.  Potential u and right-hand side b are
 * (M+2)x(N+2) doubles indexed i + j*(M+2) (calloc_centers). */
enum { MCS_PSN_U = 0,         /* potential fields.u */
       MCS_PSN_B = 1,         /* right-hand side fields.q (charge density, C/m^3) */
       MCS_PSN_BCOND = 2,     /* free-boundary values at r = R of the last solve, N+2 doubles */
       MCS_PSN_FREEBC_F = 3   /* f_n of solve_freebc!, N doubles (download only) */
};
/* MGConfig(levels, smooth1, smooth2, maxiter, tolerance, s); s <= 0 takes dz^2 / eps0
 * (main.jl:138).  M and N must be multiples of 2^levels, the coarsest level at most 4096
 * cells. */
MCS_API int mcs_poisson_create(mcs_grid* g, int levels, int smooth1, int smooth2, int maxiter,
                               double tolerance, double s, mcs_poisson** out);
MCS_API int mcs_poisson_destroy(mcs_poisson* p);
MCS_API int mcs_poisson_upload(mcs_poisson* p, int which, const double* host);
MCS_API int mcs_poisson_download(mcs_poisson* p, int which, double* host);
/* Kernels this workspace has launched so far. */
MCS_API int mcs_poisson_launches(mcs_poisson* p, int64_t* count);
/* Zero u (MCS_PSN_U) or b (MCS_PSN_B) on the device. */
MCS_API int mcs_poisson_zero(mcs_poisson* p, int which);
/* Mean device time (ms) of one finest-level red-black pass, of one finest-level residual
 * and of one fused finest-level post-smoothing (interpolation + smooth2 sweeps; 0 when the
 * fused kernels are not in use), each launched `reps` times between CUDA events on the
 * context's stream, on scratch levels (u and b untouched). */
MCS_API int mcs_poisson_profile(mcs_poisson* p, int reps, float* gs_ms, float* residual_ms, float* tile_ms);
/* Multigrid.solve(mg, u, b, ws) on the device-resident u, b: fmg! calls in *iters, the
 * last residual RMS in *eps_last (either may be NULL). */
MCS_API int mcs_poisson_mg_solve(mcs_poisson* p, int* iters, double* eps_last);
/* solve_freebc!(u, b, grid, mg, ws) (MCStreamer/src/freebc.jl:4-36); iters[2] = fmg! calls
 * of the two solves.  b gets the inhomogeneous term, as in the reference. */
MCS_API int mcs_poisson_solve_freebc(mcs_poisson* p, int* iters);
/* b = Float32((qfixed + qpart - ne) / dV * e) from the grid's int64 cell charges
 * (poisson.jl:12-34 with the NullDenoiser); with a fluid on the grid, qfixed adds its FP64
 * density part and ne is the fluid density, else both are zero. */
MCS_API int mcs_poisson_assemble(mcs_poisson* p);
/* The grid's face fields from u (poisson.jl:47-57): er = -du/dr, ez = eb - du/dz. */
MCS_API int mcs_poisson_fields(mcs_poisson* p, double eb);
/* poisson! after density!: assemble, solve_freebc!, fields; returns after the fields are
 * written. */
MCS_API int mcs_poisson_run(mcs_poisson* p, double eb, int* iters);
/* f_n = L k (I1/I0 + K1/K0)(k R) / 2, k = pi n / L, n = 1..N (freebc.jl:17-20).  Host only. */
MCS_API int mcs_freebc_coefficients(double L, double R, int N, double* f);

/* ---- Electron fluid: MCStreamer/src/fluid.jl on a cylindrical grid ----
 * The fluid density ne and its derivative dne are (M+4)x(N+4) doubles with two ghost layers
 * (calloc_centers(T, grid, 2)): the reference's (i, j), i in -1..M+2, j in -1..N+2, at
 * (i+1) + (j+1)(M+4).  qfd is the FP64 density part of the grid's qfixed, (M+2)x(N+2) at
 * i + j(M+2).  The fluxes use the grid's face fields er, ez (the last mcs_poisson_fields or
 * mcs_grid_set_efield).  One fluid per grid; mcs_poisson_assemble subtracts its ne. */
#define MCS_FLUID_MOBILITY (1e24 / 2.6867811e+25) /* setdne!'s default mobility: 1e24 / co.nair */
MCS_API int mcs_fluid_create(mcs_grid* g, mcs_fluid** out);
MCS_API int mcs_fluid_destroy(mcs_fluid* f);
/* Copy ne (ghosts included) and/or qfd in from the host; either may be NULL. */
MCS_API int mcs_fluid_upload(mcs_fluid* f, const double* ne, const double* qfd);
/* Copy ne, dne and/or qfd out to the host; any may be NULL. */
MCS_API int mcs_fluid_download(mcs_fluid* f, double* ne, double* dne, double* qfd);
/* setneedle!(fields, sigma_z, sigma_r, position_z, position_r, ne0) (fluid.jl:3-13):
 * ne += ne0 exp(-rc^2/sigma_r^2 - max(0, zc - position_z)^2/sigma_z^2) on the interior and
 * qfixed += ne.  position_r is unused, as in the reference. */
MCS_API int mcs_fluid_set_needle(mcs_fluid* f, double sigma_z, double sigma_r, double position_z, double position_r,
                                 double ne0);
/* setdne!(fields, mobility) (fluid.jl:44-98), setnebc! included: Neumann ghosts of ne, then
 * dne from the Koren-limited upwind fluxes through every z and r face. */
MCS_API int mcs_fluid_derivatives(mcs_fluid* f, double mobility);
/* euler!(fields, dt) (fluid.jl:100-111): ne += dt dne on the interior. */
MCS_API int mcs_fluid_euler(mcs_fluid* f, double dt);
/* setdne!(fields, mobility) then euler!(fields, dt) (main.jl:308-311) in one kernel; ne, dne
 * and the ghosts end as the two calls leave them. */
MCS_API int mcs_fluid_step(mcs_fluid* f, double mobility, double dt);
/* Kernels this fluid has launched so far. */
MCS_API int mcs_fluid_launches(mcs_fluid* f, int64_t* count);

/* ---- Initial electrons from density files: initfromfiles! (MCStreamer/src/initdens.jl:64-159) ----
 * ne and q (electron density m^-3, charge density C/m^3) are M x N doubles with r fastest,
 * as loadinit returns them.  Per cell, in the reference's order: above fluid_threshold the
 * cell goes to the fluid (ne) and qfixed = q/e + ne; else nsample(method, ne, q, dV) draws
 * the electron count and weight and sets qfixed's density part, and the electrons are
 * placed uniformly in (r, z) and in angle, at rest, with s = nextcoll(), appended to p in
 * cell order.  method: NoiselessInitSampling(ppc) or PoissonInitSampling(ppc).  A finite
 * fluid_threshold needs a fluid on the grid (mcs_fluid_create); pass +inf otherwise.  More
 * electrons than p's free capacity is MCS_ERR_CAPACITY and changes nothing.  *added gets
 * the electrons appended. */
enum { MCS_INIT_NOISELESS = 0, MCS_INIT_POISSON = 1 };
MCS_API int mcs_init_from_density(mcs_pop* p, mcs_grid* g, const double* ne, const double* q, int method,
                                  int64_t ppc, double fluid_threshold, uint64_t seed, int64_t* added);
/* qfixed's FP64 density part on a cylindrical grid ((M+2)x(N+2), index i + j(M+2)): the
 * densities setneedle! and initfromfiles! put into qfixed, which poisson! adds to the int64
 * deposit's densities.  Reads zeros where nothing has been set. */
MCS_API int mcs_grid_read_qfixed_density(mcs_grid* g, double* out);
MCS_API int mcs_grid_write_qfixed_density(mcs_grid* g, const double* in);
/* The same with ne and q already in device memory of the context's device. */
MCS_API int mcs_init_from_density_device(mcs_pop* p, mcs_grid* g, const double* ne, const double* q, int method,
                                         int64_t ppc, double fluid_threshold, uint64_t seed, int64_t* added);

#ifdef __cplusplus
}
#endif
#endif /* MCS_H */
