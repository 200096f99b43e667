/*
 * oracle.h -- CPU FP64 restatement of JuMC's electron step (TEST INFRASTRUCTURE).
 *
 * This library is the checker, never the product: only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / reference arm load it.  The product path is the CUDA
 * library in mcstreamer_b200/ and fails loudly when that library is missing.
 *
 * Parity status: UNPINNED against the Julia reference.  The reference (aluque/mcstreamer,
 * pure Julia) ships no tests, golden vectors or fixtures (JuMC/test/runtests.jl:4-6 is an
 * empty testset) and no Julia toolchain exists to run it.  What is pinned: the
 * Philox4x32-10 known-answer vectors of Salmon et al. (SC'11, Random123 kat_vectors),
 * the Yoshida constants, exactness properties (uniform-field Yoshida == closed form,
 * elastic energy balance) and analytic swarm limits (constant collision frequency).
 *
 * Layouts mirror the Julia memory layouts so a ccall could pass the same pointers:
 *   x, v : 3 doubles per particle, interleaved   (Vector{SVector{3,Float64}})
 *   w, s : 1 double per particle                 (Vector{Float64})
 *   active: 1 byte per particle                  (Vector{Bool})
 *   rate : neps columns of nrows doubles, process index fastest (Julia Matrix rate[j,k])
 */
#ifndef MCS_ORACLE_H
#define MCS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Process kinds (closed set of JuMC CollisionProcess subtypes used on the hot path). */
enum { ORC_NULL = 0, ORC_ELASTIC = 1, ORC_EXCITATION = 2, ORC_IONIZATION = 3,
       ORC_ATTACHMENT = 4, ORC_IONIZATION_UNIFORM = 5, ORC_PHOTOEMISSION = 6 };

/* Philox stream tags (4th counter word). */
enum { ORC_TAG_ADVANCE = 0, ORC_TAG_SWARM_RESAMPLE = 1, ORC_TAG_CELL_RESAMPLE = 2,
       ORC_TAG_INIT = 3, ORC_TAG_COLLISIONS = 4, ORC_TAG_PHOTON = 5, ORC_TAG_DENSITY = 6 };
/* initfromfiles!: cell c's count draws from {c, 0, k/4, ORC_TAG_DENSITY}; its electron k from
 * the four words of {c, k, 0, ORC_TAG_DENSITY | ORC_TAG_DENSITY_PARTICLE} (r, z, phi, s). */
#define ORC_TAG_DENSITY_PARTICLE 0x40000000u
enum { ORC_INIT_NOISELESS = 0, ORC_INIT_POISSON = 1 };
/* Photo-emission streams of collision event j of an electron: the photon count draws
 * from {slot, step, k/4, ORC_TAG_PHOTON_COUNT | j}, photon p from words 4p..4p+3 of
 * {slot, step, p, ORC_TAG_PHOTON_DRAW | j} (direction phi, u; log-nu fraction; s). */
#define ORC_TAG_PHOTON_COUNT 0x20000000u
#define ORC_TAG_PHOTON_DRAW 0x40000000u

typedef struct {
    int nrows;            /* processes incl. the null row */
    int neps;             /* energy grid points */
    double e0, de;        /* energy grid: e_k = e0 + k*de (J), LinRange semantics */
    double emax;          /* last grid point (J) */
    const double* rate;   /* [neps][nrows] */
    const int* kind;      /* [nrows] */
    const double* param;  /* [nrows]: threshold (J) or mass ratio */
    double maxrate;       /* s^-1 */
    /* PhotoEmission rows (electron.jl:88-105): log(nu_min), log(nu_max) per row (NULL when
     * the table has none), photon_multiplier and photon_weight. */
    const double* pe_lmin;
    const double* pe_lmax;
    double pe_mult, pe_pw;
} orc_table;

/* Photon population (JuMC/src/photon.jl:11-18): PhotonState x, v, nu, w, s, active. */
typedef struct {
    double* x; double* v; double* nu; double* w; double* s; uint8_t* active;
    int64_t n, cap;
    uint64_t seed;        /* Philox key of the photon advance */
    uint32_t step;
    double numax;         /* ZhelezniakCollisions(numax): the photons' maxrate */
} orc_photons;

typedef struct {
    double* x; double* v; double* w; double* s; uint8_t* active;
    int64_t n;            /* particles in use (active or not) */
    int64_t cap;          /* capacity */
    uint64_t seed;        /* Philox key */
    uint32_t step;        /* Philox counter word 1 */
} orc_pop;

enum { ORC_FIELD_UNIFORM = 0, ORC_FIELD_CART3D = 1, ORC_FIELD_CYL = 2 };
typedef struct {
    int type;
    double e[3];                          /* uniform */
    int nx, ny, nz; double h, x0, y0, z0; /* cart3d: cells; nodes are (nx+1)(ny+1)(nz+1) */
    const double* enodes;                 /* cart3d: 3 per node, x fastest */
    double R, L; int M, N;                /* cyl: MCStreamer Grid(R, L, M, N) */
    const double* er; const double* ez;   /* cyl: (M+3) x (N+3), index i + j*(M+3), i,j from 0 */
} orc_field;

enum { ORC_TRACK_NONE = 0, ORC_TRACK_CART3D = 1, ORC_TRACK_CYL = 2 };
typedef struct {
    int type;
    int nx, ny, nz; double h, x0, y0, z0; int64_t* qnodes; /* cart3d CIC, 2^-32 fixed point */
    double R, L; int M, N; double* qcyl;                    /* cyl NGP, (M+2)x(N+2) i + j*(M+2) */
} orc_tracker;

/* ---- RNG ---- */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double orc_uniform(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t tag, uint32_t k);

/* ---- step (R1-R8, R15) ---- */
/* Returns 0, or a status: 3 capacity, 4 energy out of table, 5 field too high. */
int orc_advance(orc_pop* pop, const orc_table* tab, const orc_field* fld, double dt,
                orc_tracker* trk, int nthreads, int clamp_energy);
int orc_collisions(orc_pop* pop, const orc_table* tab, double dt, orc_tracker* trk,
                   int nthreads, int clamp_energy);
/* advance! with injected uniforms: slot i < nslots reads u[pos[i]] .. u[end[i] - 1] in the
 * reference's serial draw order (pos[i] is advanced); running out returns 11. */
int orc_advance_injected(orc_pop* pop, const orc_table* tab, const orc_field* fld, double dt,
                         orc_tracker* trk, int nthreads, int clamp_energy, const double* u, int64_t* pos,
                         const int64_t* end, int64_t nslots);

/* ---- helpers exposed for unit known-answer tests ---- */
void orc_efield(const orc_field* fld, const double x[3], double e[3]);
int orc_indweight(const orc_table* tab, double eng, int64_t* k, double* w);
void orc_yoshida(const orc_field* fld, double x[3], double v[3], double dt);

/* ---- population ops ---- */
int orc_repack(orc_pop* pop);                                      /* R12 */
int orc_swarm_resample(orc_pop* pop, int64_t n0, double tol);      /* R14 */
void orc_moments(const orc_pop* pop, const orc_table* tab, double* out); /* R13 */

/* ---- cells, deposit, resample ---- */
/* cell key of a position: cart3d (ix + nx*(iy + ny*iz)) / cyl (i + (M+2)*j); -1 if out. */
int64_t orc_cell_key(const orc_field* grid, const double x[3]);
/* stable sort of the population by cell key (inactive and out-of-grid last), R11 ordering. */
int orc_sort_cells(orc_pop* pop, const orc_field* grid);
int orc_resample_cells(orc_pop* pop, const orc_field* grid, int ntarget, int nmax,
                       uint32_t call);                             /* R11 */
/* R10: cart3d CIC int64 from f32 in-cell offsets (device quantisation) or cyl NGP. */
void orc_deposit(const orc_pop* pop, orc_tracker* trk, double val, int quantize_f32);

/* advance!(mpopl, efield, dt, tracker) over the electrons and the photons
 * (mixed_population.jl:24-54): electrons first, photo-emission appending photons; then every
 * photon (the new ones included), photo-ionization appending electrons. */
int orc_advance_mixed(orc_pop* electrons, orc_photons* photons, const orc_table* tab, const orc_field* fld,
                      double dt, orc_tracker* trk, int nthreads, int clamp_energy);
/* The photon half alone. */
int orc_photon_advance(orc_photons* photons, orc_pop* electrons, double dt, orc_tracker* trk, int nthreads);

/* Cylindrical multigrid (poisson.cpp): Multigrid.solve with MCStreamer's configuration.
 * Arrays (M+2)x(N+2), index i + j*(M+2).  Returns the number of fmg! calls. */
int orc_mg_solve(int M, int N, double s, int levels, double tol, int smooth1, int smooth2, int maxiter,
                 double* u, const double* b, double* eps_last);
double orc_mg_residual_rms(int M, int N, double s, const double* u, const double* b);
void orc_mg_apply_bc(double* a, int M, int N);
void orc_mg_gauss_seidel(double* u, const double* b, int M, int N);
void orc_mg_residual(double* r, const double* u, const double* b, double s, int M, int N);
void orc_mg_restrict(double* rh, const double* r, int M, int N);
void orc_mg_interpolate(double* f, const double* h, int M, int N, int add);

/* initfromfiles!(method, fields, loader; fluid_threshold, maxp) (MCStreamer/src/initdens.jl:
 * 64-102) over densities ne, q (M x N doubles, r fastest): electrons (x 3 per electron, w, s;
 * at rest, active) in cell order, qfixed's density part qfd ((M+2)x(N+2)) set per cell and
 * the fluid density ne_fluid ((M+4)x(N+4)) above the threshold.  Returns the electrons
 * written, or -1 when more than cap would be. */
/* repack!(photons) (JuMC/src/population.jl:191-215). */
int orc_photons_repack(orc_photons* ph);
int64_t orc_init_from_density(int M, int N, double R, double L, const double* ne, const double* q, int method,
                              int64_t p, double fluid_threshold, uint64_t seed, int64_t cap, double* x, double* w,
                              double* s, double* qfd, double* ne_fluid);

#ifdef __cplusplus
}
#endif
#endif
