/*
 * poisson.cpp -- CPU FP64 restatement of the cylindrical multigrid Poisson solver that
 * MCStreamer's poisson! drives.  TEST INFRASTRUCTURE ONLY: loaded by tests/ and bench.py's
 * CPU arm as the checker, never by the product.
 *
 * Restates Multigrid/src/Multigrid.jl (laplacian 152-158, gauss_seidel! 168-178,
 * residual! 186-193, restrict! 213-226, interpolate! 232-258, buildmat 261-295, mgv!
 * 334-377, fmg! 380-434, solve 449-467), Multigrid/src/redblack.jl:38-46 and
 * Multigrid/src/boundaries.jl:110-133 with the configuration of MCStreamer/src/main.jl:
 * 131-144 (bc = Left/Right/Top Dirichlet, Bottom (axis) Neumann, CylindricalConnector{1},
 * g = 1).  Arrays are (M+2)x(N+2) doubles, r fastest: element (i, j) at i + j*(M+2), i the
 * r index and j the z index, ghosts at i = 0, M+1 and j = 0, N+1 (the parent arrays of
 * the reference's OffsetArrays; storage index = 1-based parent index - 1).
 *
 * Every operation is evaluated in the reference's order and unfused (built with
 * -ffp-contract=off).  Loops whose iterations are independent (one colour of a sweep, the
 * residual, restriction, interpolation) run on OpenMP threads, which changes no result.
 * Only the coarsest direct solve (a dense LU with partial pivoting here, a sparse
 * factorization in the reference) and the residual norm differ in their rounding.
 */
#include "oracle.h"

#include <cmath>
#include <cstring>
#include <vector>

namespace {

struct Level {
    int M = 0, N = 0;
    std::vector<double> a;
    long ld() const { return M + 2; }
    double* p() { return a.data(); }
};

// CylindricalConnector{1} (Multigrid.jl:37-39): x * (1 + d / (2 (c - g) - 1)), c the
// 1-based parent index, i.e. 2i - 1 for storage row i.
struct Conn {
    std::vector<double> fp, fm;   // d = +1, d = -1, per storage row 0..M+1
    explicit Conn(int M) : fp(M + 2), fm(M + 2) {
        for (int i = 1; i <= M + 1; ++i) {
            fp[i] = 1.0 + 1.0 / (double)(2 * i - 1);
            fm[i] = 1.0 + (-1.0) / (double)(2 * i - 1);
        }
    }
};

// setbc! of each (boundary, condition) in tuple order (boundaries.jl:110-133):
// Left, Right, Top Dirichlet (ghost = -1 * valid + 0), Bottom Neumann (ghost = valid + 0).
// Every ghost row/column covers the full extent, so the corners end as the later
// conditions leave them.
void apply_bc(double* a, int M, int N) {
    const long ld = M + 2;
    for (int i = 0; i <= M + 1; ++i) a[i] = -a[i + ld] + 0.0;
    for (int i = 0; i <= M + 1; ++i) a[i + (N + 1) * ld] = -a[i + N * ld] + 0.0;
    for (int j = 0; j <= N + 1; ++j) a[M + 1 + j * ld] = -a[M + j * ld] + 0.0;
    for (int j = 0; j <= N + 1; ++j) a[j * ld] = a[1 + j * ld] + 0.0;
}

// laplacian (Multigrid.jl:152-158) with the stencil order of lplstencil: +r, +z, -r, -z.
// Neighbours are addressed linearly, as the reference's column-major arrays are.
inline double lap(const double* u, long k, long ld, double fp, double fm) {
    double s = -4.0 * u[k];
    s += u[k + 1] * fp;
    s += u[k + ld] * 1.0;
    s += u[k - 1] * fm;
    s += u[k - ld] * 1.0;
    return s;
}

// gauss_seidel! with redblack2: pass `parity` visits, in every column j (storage 1..N),
// the rows 1, 3, ... <= M shifted by p = parity xor (j even).  With an odd M the shift
// reaches the ghost row M+1, whose +r neighbour is then the first element of the next
// column; the reference updates it there and so does this restatement.
void gauss_seidel(double* u, const double* b, int M, int N, const Conn& cn) {
    const long ld = M + 2;
    for (int parity = 0; parity < 2; ++parity)
#pragma omp parallel for schedule(static) if ((long)M * N > 65536)
        for (int j = 1; j <= N; ++j) {
            const int p = parity ^ ((j % 2) == 0 ? 1 : 0);
            for (int r = 1; r <= M; r += 2) {
                const int i = r + p;
                const long k = i + j * ld;
                const double l = lap(u, k, ld, cn.fp[i], cn.fm[i]);
                u[k] += 1.0 * (l + b[k]) / 4.0;
            }
        }
}

void residual(double* r, const double* u, const double* b, double s, int M, int N, const Conn& cn) {
    const long ld = M + 2;
#pragma omp parallel for schedule(static) if ((long)M * N > 65536)
    for (int j = 1; j <= N; ++j)
        for (int i = 1; i <= M; ++i) {
            const long k = i + j * ld;
            r[k] = s * b[k] + lap(u, k, ld, cn.fp[i], cn.fm[i]);
        }
}

// restrict!: coarse cell (I, J) <- 4 * (sum of its four fine children) / 4, children in
// cubestencil order (0,0), (0,1), (1,0), (1,1) (r offset first).
void restrict_(Level& h, Level& f) {
    const long ldh = h.ld(), ldf = f.ld();
#pragma omp parallel for schedule(static) if ((long)h.M * h.N > 16384)
    for (int J = 1; J <= h.N; ++J)
        for (int I = 1; I <= h.M; ++I) {
            const long k = (2 * I - 1) + (2 * J - 1) * ldf;
            double s = 0.0;
            s += f.a[k];
            s += f.a[k + ldf];
            s += f.a[k + 1];
            s += f.a[k + 1 + ldf];
            h.a[I + J * ldh] = 4.0 * s / 4.0;
        }
}

// interpolate!: fine child s of coarse cell (I, J) = sum over sh in cubestencil order of
// w(sh) * coarse[(I, J) + (2s - 1) .* sh], w = 9/16, 3/16, 3/16, 1/16; added or stored.
void interpolate(Level& f, Level& h, bool add) {
    const long ldh = h.ld(), ldf = f.ld();
    const double w[4] = {9.0 / 16.0, 3.0 / 16.0, 3.0 / 16.0, 1.0 / 16.0};
#pragma omp parallel for schedule(static) if ((long)h.M * h.N > 16384)
    for (int J = 1; J <= h.N; ++J)
        for (int I = 1; I <= h.M; ++I)
            for (int si = 0; si < 2; ++si)
                for (int sj = 0; sj < 2; ++sj) {
                    const int di = 2 * si - 1, dj = 2 * sj - 1;
                    double s = 0.0;
                    s += w[0] * h.a[I + J * ldh];
                    s += w[1] * h.a[I + (J + dj) * ldh];
                    s += w[2] * h.a[(I + di) + J * ldh];
                    s += w[3] * h.a[(I + di) + (J + dj) * ldh];
                    double& t = f.a[(2 * I - 1 + si) + (2 * J - 1 + sj) * ldf];
                    t = add ? t + s : s;
                }
}

void fill0(Level& a) {
    double* p = a.p();
    const long n = (long)a.a.size();
#pragma omp parallel for schedule(static) if (n > 65536)
    for (long k = 0; k < n; ++k) p[k] = 0.0;
}

struct MG {
    int M, N, levels, smooth1, smooth2, maxiter;
    double s, tol;
    std::vector<Level> res, res1, sol;
    std::vector<Conn> conn;
    // coarsest level: the Cartesian matrix of buildmat, LU-factorized with partial pivoting
    int nc = 0;
    std::vector<double> lu;
    std::vector<int> piv;

    MG(int M_, int N_, double s_, int levels_, double tol_, int s1, int s2, int maxiter_)
        : M(M_), N(N_), levels(levels_), smooth1(s1), smooth2(s2), maxiter(maxiter_), s(s_), tol(tol_) {
        for (int l = 0; l <= levels; ++l) {
            Level L;
            L.M = M >> l;
            L.N = N >> l;
            L.a.assign((size_t)(L.M + 2) * (L.N + 2), 0.0);
            res.push_back(L);
            res1.push_back(L);
            sol.push_back(L);
            conn.emplace_back(L.M);
        }
        build_coarse();
    }

    // buildmat (Multigrid.jl:261-295): -4 on the diagonal, +1 to inner neighbours, and a
    // neighbour across a boundary folded onto the cell itself with the condition's
    // coefficient (Dirichlet -1, Neumann +1).  No connector: the matrix is Cartesian.
    void build_coarse() {
        const int Mc = M >> levels, Nc = N >> levels;
        nc = Mc * Nc;
        lu.assign((size_t)nc * nc, 0.0);
        auto A = [&](int r, int c) -> double& { return lu[(size_t)r * nc + c]; };
        const int di[4] = {1, 0, -1, 0}, dj[4] = {0, 1, 0, -1};
        for (int j = 1; j <= Nc; ++j)
            for (int i = 1; i <= Mc; ++i) {
                const int p = (i - 1) + (j - 1) * Mc;
                A(p, p) -= 4.0;
                for (int d = 0; d < 4; ++d) {
                    int ni = i + di[d], nj = j + dj[d];
                    double m = 1.0;
                    if (nj == 0) { nj = 1; m = -1.0; }             // LeftBnd, Dirichlet
                    else if (nj == Nc + 1) { nj = Nc; m = -1.0; }  // RightBnd, Dirichlet
                    else if (ni == Mc + 1) { ni = Mc; m = -1.0; }  // TopBnd, Dirichlet
                    else if (ni == 0) { ni = 1; m = 1.0; }         // BottomBnd, Neumann
                    A(p, (ni - 1) + (nj - 1) * Mc) += m;
                }
            }
        piv.resize(nc);
        for (int k = 0; k < nc; ++k) {
            int best = k;
            for (int r = k + 1; r < nc; ++r)
                if (std::fabs(A(r, k)) > std::fabs(A(best, k))) best = r;
            piv[k] = best;
            if (best != k)
                for (int c = 0; c < nc; ++c) std::swap(A(k, c), A(best, c));
            for (int r = k + 1; r < nc; ++r) {
                A(r, k) /= A(k, k);
                for (int c = k + 1; c < nc; ++c) A(r, c) -= A(r, k) * A(k, c);
            }
        }
    }

    // ws.mat \ btop: solves mat * z = btop (btop = the restricted residual, column-major).
    void coarse_solve(Level& z, const Level& bt) {
        const int Mc = bt.M;
        std::vector<double> y(nc);
        for (int j = 1; j <= bt.N; ++j)
            for (int i = 1; i <= Mc; ++i) y[(i - 1) + (j - 1) * Mc] = bt.a[i + j * (Mc + 2)];
        auto A = [&](int r, int c) { return lu[(size_t)r * nc + c]; };
        for (int k = 0; k < nc; ++k) std::swap(y[k], y[piv[k]]);
        for (int r = 0; r < nc; ++r)
            for (int c = 0; c < r; ++c) y[r] -= A(r, c) * y[c];
        for (int r = nc - 1; r >= 0; --r) {
            for (int c = r + 1; c < nc; ++c) y[r] -= A(r, c) * y[c];
            y[r] /= A(r, r);
        }
        for (int j = 1; j <= bt.N; ++j)
            for (int i = 1; i <= Mc; ++i) z.a[i + j * (Mc + 2)] = y[(i - 1) + (j - 1) * Mc];
    }

    void smooth(Level& x, const Level& b, int l, int n) {
        for (int it = 0; it < n; ++it) {
            apply_bc(x.p(), x.M, x.N);
            gauss_seidel(x.p(), b.a.data(), x.M, x.N, conn[l]);
        }
    }

    // mgv! (Multigrid.jl:334-377); level l uses res1[l], res[l+1], sol[l+1].  The
    // apply!(r) before restrict! touches only ghosts, which restrict! never reads.
    void mgv(Level& x, const Level& b, int l) {
        if (l == levels) {
            smooth(x, b, l, 50);
            return;
        }
        smooth(x, b, l, smooth1);
        Level& r = res1[l];
        apply_bc(x.p(), x.M, x.N);
        residual(r.p(), x.p(), b.a.data(), 1.0, x.M, x.N, conn[l]);
        Level& rh = res[l + 1];
        restrict_(rh, r);
        Level& xh = sol[l + 1];
        fill0(xh);
        mgv(xh, rh, l + 1);
        interpolate(x, xh, true);
        smooth(x, b, l, smooth2);
    }

    double residual_rms(double* x, const double* b) {
        Level& r0 = res[0];
        fill0(r0);
        residual(r0.p(), x, b, s, M, N, conn[0]);
        double ss = 0.0;
        for (double v : r0.a) ss += v * v;
        return std::sqrt(ss) / std::sqrt((double)((long long)M * N));
    }

    // fmg! (Multigrid.jl:380-434): one full-multigrid correction of x; false once the
    // residual RMS is below s * tolerance.
    bool fmg(double* x, const double* b, double* eps_out) {
        apply_bc(x, M, N);
        const double eps = residual_rms(x, b);
        if (eps_out) *eps_out = eps;
        if (s * tol > eps) return false;
        for (int k = 0; k < levels; ++k) restrict_(res[k + 1], res[k]);
        coarse_solve(sol[levels], res[levels]);
        Level* z = &sol[levels];
        for (int k = 1; k <= levels; ++k) {
            Level& z1 = sol[levels - k];
            fill0(z1);
            apply_bc(z->p(), z->M, z->N);
            interpolate(z1, *z, false);
            mgv(z1, res[levels - k], levels - k);
            z = &z1;
        }
        const long n = (long)(M + 2) * (N + 2);
        const double* zz = z->a.data();
#pragma omp parallel for schedule(static) if (n > 65536)
        for (long k = 0; k < n; ++k) x[k] += zz[k];
        apply_bc(x, M, N);
        return true;
    }
};

}  // namespace

extern "C" {

// Multigrid.solve (Multigrid.jl:449-467): fmg! until converged or maxiter+1 calls.  Returns
// the number of fmg! calls (the reference's `iter`), or -1 on bad sizes.
int orc_mg_solve(int M, int N, double s, int levels, double tol, int smooth1, int smooth2, int maxiter,
                 double* u, const double* b, double* eps_last) {
    if (levels < 0 || M < 1 || N < 1 || (M >> levels) < 1 || (N >> levels) < 1 ||
        ((M >> levels) << levels) != M || ((N >> levels) << levels) != N)
        return -1;
    MG mg(M, N, s, levels, tol, smooth1, smooth2, maxiter);
    bool cont = true;
    int iter = 0;
    while (cont && iter <= maxiter) {
        cont = mg.fmg(u, b, eps_last);
        ++iter;
    }
    return iter;
}

// The residual RMS that fmg! tests: |s b + L u| / sqrt(M N) over the inner cells, after
// the boundary conditions are applied to (a copy of) u.
double orc_mg_residual_rms(int M, int N, double s, const double* u, const double* b) {
    std::vector<double> x(u, u + (size_t)(M + 2) * (N + 2));
    apply_bc(x.data(), M, N);
    Conn cn(M);
    std::vector<double> r((size_t)(M + 2) * (N + 2), 0.0);
    residual(r.data(), x.data(), b, s, M, N, cn);
    double ss = 0.0;
    for (double v : r) ss += v * v;
    return std::sqrt(ss) / std::sqrt((double)((long long)M * N));
}

// Single operations, for the device parity tests of the individual kernels.
void orc_mg_apply_bc(double* a, int M, int N) { apply_bc(a, M, N); }
void orc_mg_gauss_seidel(double* u, const double* b, int M, int N) {
    Conn cn(M);
    gauss_seidel(u, b, M, N, cn);
}
void orc_mg_residual(double* r, const double* u, const double* b, double s, int M, int N) {
    Conn cn(M);
    residual(r, u, b, s, M, N, cn);
}
void orc_mg_restrict(double* rh, const double* r, int M, int N) {   // M, N: coarse sizes
    Level h, f;
    h.M = M; h.N = N; h.a.assign((size_t)(M + 2) * (N + 2), 0.0);
    std::memcpy(h.a.data(), rh, h.a.size() * sizeof(double));
    f.M = 2 * M; f.N = 2 * N; f.a.assign(r, r + (size_t)(2 * M + 2) * (2 * N + 2));
    restrict_(h, f);
    std::memcpy(rh, h.a.data(), h.a.size() * sizeof(double));
}
void orc_mg_interpolate(double* f_, const double* h_, int M, int N, int add) {   // M, N: coarse
    Level h, f;
    h.M = M; h.N = N; h.a.assign(h_, h_ + (size_t)(M + 2) * (N + 2));
    f.M = 2 * M; f.N = 2 * N; f.a.assign(f_, f_ + (size_t)(2 * M + 2) * (2 * N + 2));
    interpolate(f, h, add != 0);
    std::memcpy(f_, f.a.data(), f.a.size() * sizeof(double));
}

}  // extern "C"
