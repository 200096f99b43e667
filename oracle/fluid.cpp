/* fluid.cpp -- CPU restatement of MCStreamer's electron fluid (MCStreamer/src/fluid.jl) and
 * of the fluid term of poisson!'s charge (poisson.jl:17-26).  Test infrastructure only: the
 * device kernels are checked against these loops, which follow the reference statement by
 * statement, every cell of dne accumulating its face terms in the reference's order.
 *
 * Layouts (column-major, r fastest):
 *   ne, dne : calloc_centers(T, grid, 2), (M+4) x (N+4), element (i, j) for i in -1..M+2,
 *             j in -1..N+2 at (i + 1) + (j + 1) * (M + 4);
 *   er, ez  : calloc_faces, (M+3) x (N+3), element (i, j) for i in 0..M+2, j in 0..N+2 at
 *             i + j * (M + 3);
 *   qfd     : the FP64 density part of qfixed (slice 1), (M+2) x (N+2) at i + j * (M + 2).
 * Cell centres rc = (i - 1/2) dr, zc = (j - 1/2) dz with dr = R / M, dz = L / N. */
#include <cmath>

namespace {

inline long cix(int i, int j, int M) { return (long)(i + 1) + (long)(j + 1) * (M + 4); }
inline long fix(int i, int j, int M) { return (long)i + (long)j * (M + 3); }

/* koren_limiter: fluid.jl:107-112 */
inline double koren(double theta) {
    if (theta >= 4.0) return 1.0;
    if (theta > 0.4) return 1.0 / 3.0 + theta / 6.0;
    if (theta > 0.0) return theta;
    return 0.0;
}

/* setnebc!: fluid.jl:19-38, whole rows and columns (ghosts included), in its order. */
void setnebc(int M, int N, double* ne) {
    for (int j = -1; j <= N + 2; ++j) ne[cix(0, j, M)] = ne[cix(1, j, M)];
    for (int j = -1; j <= N + 2; ++j) ne[cix(-1, j, M)] = ne[cix(1, j, M)];
    for (int i = -1; i <= M + 2; ++i) ne[cix(i, 0, M)] = ne[cix(i, 1, M)];
    for (int i = -1; i <= M + 2; ++i) ne[cix(i, -1, M)] = ne[cix(i, 1, M)];
    for (int j = -1; j <= N + 2; ++j) ne[cix(M + 1, j, M)] = ne[cix(M, j, M)];
    for (int j = -1; j <= N + 2; ++j) ne[cix(M + 2, j, M)] = ne[cix(M, j, M)];
    for (int i = -1; i <= M + 2; ++i) ne[cix(i, N + 1, M)] = ne[cix(i, N, M)];
    for (int i = -1; i <= M + 2; ++i) ne[cix(i, N + 2, M)] = ne[cix(i, N, M)];
}

}  // namespace

extern "C" {

/* setneedle!: fluid.jl:3-13.  position_r is taken and unused, as in the reference. */
void orc_fluid_needle(int M, int N, double R, double L, double sigma_z, double sigma_r, double position_z,
                      double position_r, double ne0, double* ne, double* qfd) {
    (void)position_r;
    const double dr = R / M, dz = L / N;
    for (int j = 1; j <= N; ++j)
        for (int i = 1; i <= M; ++i) {
            const double rc = ((double)(i - 1) + 0.5) * dr;
            const double zc = ((double)(j - 1) + 0.5) * dz;
            const double d = zc - position_z;
            const double z1 = d > 0.0 ? d : 0.0;
            const double a = -(rc * rc) / (sigma_r * sigma_r) - (z1 * z1) / (sigma_z * sigma_z);
            ne[cix(i, j, M)] += ne0 * std::exp(a);
            qfd[(long)i + (long)j * (M + 2)] += ne[cix(i, j, M)];
        }
}

void orc_fluid_setnebc(int M, int N, double* ne) { setnebc(M, N, ne); }

/* setdne!: fluid.jl:44-98 (setnebc! first, dne zeroed, the z fluxes face by face, then the
 * r fluxes). */
void orc_fluid_setdne(int M, int N, double R, double L, double mobility, double* ne, double* dne,
                      const double* er, const double* ez) {
    const double dr = R / M, dz = L / N;
    setnebc(M, N, ne);
    for (long k = 0; k < (long)(M + 4) * (N + 4); ++k) dne[k] = 0.0;
    /* The reference runs each face loop's inner index in parallel (@batch); here blocks of
     * the inner index go to OpenMP threads and every cell still receives its terms in the
     * serial order (its lower face, then its upper face). */
#pragma omp parallel for schedule(static)
    for (int i0 = 1; i0 <= M; i0 += 64)
    for (int j = 1; j <= N + 1; ++j)
        for (int i = i0; i <= M && i < i0 + 64; ++i) {
            const double v = -ez[fix(i, j, M)] * mobility;
            const int sv = std::signbit(v) ? -1 : 1;
            const int jd = j + (sv - 1) / 2, ju = j + (-sv - 1) / 2, ju2 = j + (-3 * sv - 1) / 2;
            const double theta = (ne[cix(i, ju, M)] - ne[cix(i, ju2, M)]) / (ne[cix(i, jd, M)] - ne[cix(i, ju, M)]);
            const double F = v * (ne[cix(i, ju, M)] + koren(theta) * (ne[cix(i, jd, M)] - ne[cix(i, ju, M)]));
            dne[cix(i, j, M)] += F / dz;
            dne[cix(i, j - 1, M)] -= F / dz;
        }
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= N; ++j)
        for (int i = 1; i <= M + 1; ++i) {
            const double v = -er[fix(i, j, M)] * mobility;
            const int sv = std::signbit(v) ? -1 : 1;
            const int id = i + (sv - 1) / 2, iu = i + (-sv - 1) / 2, iu2 = i + (-3 * sv - 1) / 2;
            const double theta = (ne[cix(iu, j, M)] - ne[cix(iu2, j, M)]) / (ne[cix(id, j, M)] - ne[cix(iu, j, M)]);
            const double F = v * (ne[cix(iu, j, M)] + koren(theta) * (ne[cix(id, j, M)] - ne[cix(iu, j, M)]));
            dne[cix(i, j, M)] += F / dr;
            dne[cix(i - 1, j, M)] -= F / dr;
        }
}

/* euler!: fluid.jl:100-111 */
void orc_fluid_euler(int M, int N, double dt, double* ne, const double* dne) {
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= N; ++j)
        for (int i = 1; i <= M; ++i) ne[cix(i, j, M)] += dt * dne[cix(i, j, M)];
}

double orc_fluid_koren(double theta) { return koren(theta); }

}  /* extern "C" */
