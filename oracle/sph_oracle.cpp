// sph_oracle.cpp -- CPU restatement of SPH-2D's weakly-compressible time step.
//
// TEST INFRASTRUCTURE ONLY.  This file is the oracle that libsph_b200 is
// compared against; it is never linked into, loaded by or called from the
// product path.  Only tests/, __graft_entry__.smoke() and the cpu_baseline /
// --impl reference legs of bench.py may load it.
//
// It follows the reference's own loop structure (Fortran 90, mini-walker/SPH-2D):
// a pair list built i = 1..n-1 over the 3x3 background cells in the reference's
// stencil order, then one scatter loop per physical term in pair order.  The
// scatter is evaluated as "per pair terms first, then a per-particle sum over
// that particle's pairs in increasing pair index", which adds exactly the same
// numbers in exactly the same order as the Fortran scatter, so OpenMP threads
// do not change a single bit of the result.
//
// Pins (see tests/test_oracle.py):
//   * the Taylor-Green initialiser reproduces the reference's own t = 0 output
//     Taylor_Green_Vortex/Initial_particle_information.dat (10 decimals);
//   * the kinetic-energy decay of the reference configuration follows the
//     reference run's Taylor_Green_Vortex/Kinetic_energy.dat statistically.
// Bit-level agreement with ifort's libm cannot be pinned (no Fortran compiler
// here); the oracle uses glibc.
//
// Deliberate deviation (documented): the reference reuses last step's rates as
// K1 indexed by the previous step's subdomain order (time_iteration.f90:940-965
// after Devide_block_and_send_tasks.f90:670-701 rebuilt that order); here each
// particle carries its own rates.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/sph_b200.h"

namespace {

// ---------------------------------------------------------------------------
// Constants derived from the configuration.  With reference_literals the
// default-real (single precision) literals of the Fortran source are rounded
// to float first, as ifort does.
// ---------------------------------------------------------------------------
struct Consts {
    double pi_k;      // PI=3.14159265358 in compute_kernel.f90:32 (real(8) parameter from a default-real literal)
    double pi;        // information_module PI (exact double)
    double gauss_e9;  // exp(-9.0)               compute_kernel.f90:129
    double gauss_den; // (1-10*exp(-9.0))        compute_kernel.f90:123
    double cut_min;   // 1.0E-7                  find_particle_pair.f90:87
    double fs_thr;    // 0.65                    Define_freesurface...f90:123
    double c1414;     // 1.414                   Define_freesurface...f90:356,363
    double sps_dl;    // sqrt(2.0)/2.0           Solver_..._SPS.f90:266
    double sps_c012;  // 0.12                    :274
    double sps_23;    // 2.0/3.0                 :278
    double sps_blin;  // 2.0/3.0*0.0066          :286
    double sqrt_c0;   // sqrt(square_c_0)
    double eos_b;     // square_c_0*water_rho_0/7.0
    double support_volume; // PI*(kernel_scale*smooth_length)**dim
    double w_dx;      // kernel value at distance dx (Shift_particle_position.f90:56-68)
    double kernel_q_zero; // 1.0E-8 (Compute_Kernel.f90:258)
};

Consts g_K;
sph_config g_cfg;
// Test hook (oracle_set_muscl_gradient_scale): factor on the MUSCL reconstruction
// gradients grad p, grad u, grad v; 1 everywhere except in the pin tests, where 0
// turns the MUSCL solver's Riemann states into the unreconstructed ones.
double g_muscl_grad_scale = 1.0;

inline double pw3(double x) { return x * x * x; }
inline double pw4(double x) { double x2 = x * x; return x2 * x2; }
inline double pw7(double x) { double x2 = x * x; double x4 = x2 * x2; return x4 * x2 * x; }

// compute_kernel: Taylor_Green_Vortex/compute_kernel.f90:120-142 (model 4),
// Moving_Square_Or_Cylinder_Inside_a_Rectangular_Box/Compute_Kernel.f90:149-198,257-260.
void kernel(double d, const double pd[2], double h, double& w, double dw[2]) {
    const Consts& K = g_K;
    double q = d / h;
    w = 0.0; dw[0] = dw[1] = 0.0;
    if (g_cfg.kernel_model == SPH_KERNEL_GAUSSIAN) {
        double factor = 1.0 / (K.pi_k * (h * h) * K.gauss_den);
        if (d <= 3.0 * h) {
            double e = std::exp(-(q * q));
            w = (e - K.gauss_e9) * factor;
            for (int c = 0; c < 2; ++c) dw[c] = (e * (-2 * q)) * pd[c] / (d * h) * factor;
        }
    } else {
        double factor = 7.0 / (4 * K.pi_k * (h * h));
        if (d <= 2.0 * h) {
            double t = 1 - q / 2.0;
            w = factor * (1 + 2 * q) * pw4(t);
            for (int c = 0; c < 2; ++c) dw[c] = factor * (-5 * q * pw3(t)) * pd[c] / (d * h);
        }
    }
    if (q <= K.kernel_q_zero) { dw[0] = dw[1] = 0.0; }
}

// status_equation: Taylor_Green_Vortex/status_equation.f90:60-63,
// Moving_Square.../Status_Equation.f90:56-76.
inline void eos(double rho, double& p, double& c) {
    double r = rho / g_cfg.rho0;
    if (g_cfg.eos == SPH_EOS_TAIT) p = g_K.eos_b * (pw7(r) - 1.0) + g_cfg.background_p;
    else p = g_cfg.c0sq * (rho - g_cfg.rho0) + g_cfg.background_p;
    c = g_K.sqrt_c0 * pw3(r);
}

// matrix_inversion_less_three, n = 2: Taylor_Green_Vortex/function_module.f90:157-249.
// Returns 0 when the determinant is zero (check_error = 0).
int inv2(const double A[2][2], double R[2][2]) {
    double a1 = A[0][0], b1 = A[0][1], a2 = A[1][0], b2 = A[1][1];
    double det = (a1 * b2 - b1 * a2);
    if (det != 0) {
        R[0][0] = b2 / det; R[0][1] = -b1 / det;
        R[1][0] = -a2 / det; R[1][1] = a1 / det;
        return 1;
    }
    return 0;
}

// MUSCL_Limiter: Taylor_Green_Vortex/function_module.f90:34-80.
void muscl_limiter(double di, double dj, double dij, double& li, double& lj) {
    const double beta_lim = 1.3;
    const double diff = 0.5;
    double fi, fj, lim;
    if (dj > 0.0) {
        lim = std::max(0.0, std::max(std::min(beta_lim * di, dj), std::min(di, beta_lim * dj)));
        if (lim > 0.5 * dij && std::fabs(lim) > 0.0) {
            if (di > dj) { fi = diff; fj = 0.0; } else { fi = 0.0; fj = diff; }
            li = dij * fi; lj = dij * fj;
        } else { li = lim; lj = lim; }
    } else {
        lim = std::min(0.0, std::min(std::max(beta_lim * di, dj), std::max(di, beta_lim * dj)));
        if (lim < 0.5 * dij && std::fabs(lim) > 0.0) {
            if (di < dj) { fi = diff; fj = 0.0; } else { fi = 0.0; fj = diff; }
            li = dij * fi; lj = dij * fj;
        } else { li = lim; lj = lim; }
    }
}

void derive_consts(const sph_config& cfg) {
    Consts& K = g_K;
    bool q = cfg.reference_literals != 0;
    K.pi = 3.14159265358979324;
    K.pi_k = q ? (double)3.14159265358f : K.pi;
    if (q) {
        float e9 = std::exp(-9.0f);
        K.gauss_e9 = (double)e9;
        K.gauss_den = (double)(1.0f - 10.0f * e9);
        K.cut_min = (double)1.0e-7f;
        K.fs_thr = (double)(float)cfg.fs_threshold;
        K.c1414 = (double)1.414f;
        K.sps_dl = (double)(std::sqrt(2.0f) / 2.0f);
        K.sps_c012 = (double)0.12f;
        K.sps_23 = (double)(2.0f / 3.0f);
        K.sps_blin = (double)((2.0f / 3.0f) * 0.0066f);
        K.kernel_q_zero = (double)1.0e-8f;
    } else {
        K.gauss_e9 = std::exp(-9.0);
        K.gauss_den = 1.0 - 10.0 * K.gauss_e9;
        K.cut_min = 1.0e-7;
        K.fs_thr = cfg.fs_threshold;
        K.c1414 = 1.414;
        K.sps_dl = std::sqrt(2.0) / 2.0;
        K.sps_c012 = 0.12;
        K.sps_23 = 2.0 / 3.0;
        K.sps_blin = 2.0 / 3.0 * 0.0066;
        K.kernel_q_zero = 1.0e-8;
    }
    K.sqrt_c0 = std::sqrt(cfg.c0sq);
    K.eos_b = cfg.c0sq * cfg.rho0 / 7.0;
    double sr = cfg.kernel_scale * cfg.h;
    K.support_volume = K.pi * (sr * sr);
    double pd[2] = {0.0, 0.0}, dw[2];
    kernel(cfg.dx, pd, cfg.h, K.w_dx, dw);
}

// ---------------------------------------------------------------------------
// Particle arrays (the subdomain arrays of Public_variable_module).
// ---------------------------------------------------------------------------
struct Particles {
    int n = 0;
    std::vector<double> x, y, u, v, rho, mass, smass;
    std::vector<int> type;
    std::vector<int> itype;    // subdomain_particle_initial_type (body force)
    std::vector<int> src;      // image source (host index) or -1
    void resize(int m) {
        n = m;
        x.resize(m); y.resize(m); u.resize(m); v.resize(m); rho.resize(m); mass.resize(m);
        smass.resize(m); type.resize(m); itype.resize(m); src.resize(m);
    }
};

struct PairList {
    std::vector<int> pi, pj;
    std::vector<double> w, dw0, dw1, dx0, dx1;   // w, dwdx, position_difference_ij
    size_t size() const { return pi.size(); }
};

// Background grid of Taylor_Green_Vortex/Assign_boundary_particles.f90:80-114:
// cells of (kernel_scale+1)*h, particles inserted in increasing index order.
struct Grid {
    double ox, oy, cs;
    int nx, ny;
    std::vector<int> start, items; // CSR: cell -> particle indices (ascending)
    std::vector<int> cell;         // particle -> cell (or -1 when not binned)
};

void build_grid(const Particles& P, Grid& G) {
    const double cs = (g_cfg.kernel_scale + 1) * g_cfg.h;
    double lox = 1e300, loy = 1e300, hix = -1e300, hiy = -1e300;
    for (int i = 0; i < P.n; ++i) {
        if (P.type[i] == SPH_TYPE_ILL || P.type[i] == 0) continue;
        lox = std::min(lox, P.x[i]); hix = std::max(hix, P.x[i]);
        loy = std::min(loy, P.y[i]); hiy = std::max(hiy, P.y[i]);
    }
    if (lox > hix) { lox = loy = 0; hix = hiy = 1; }
    G.cs = cs;
    G.ox = lox - 2 * cs; G.oy = loy - 2 * cs;
    G.nx = (int)std::floor((hix - G.ox) / cs) + 3;
    G.ny = (int)std::floor((hiy - G.oy) / cs) + 3;
    const int nc = G.nx * G.ny;
    G.cell.assign(P.n, -1);
    std::vector<int> cnt(nc + 1, 0);
    for (int i = 0; i < P.n; ++i) {
        if (P.type[i] == SPH_TYPE_ILL || P.type[i] == 0) continue;
        int cx = (int)std::floor((P.x[i] - G.ox) / cs);
        int cy = (int)std::floor((P.y[i] - G.oy) / cs);
        int k = cy * G.nx + cx;
        G.cell[i] = k;
        cnt[k + 1]++;
    }
    for (int k = 0; k < nc; ++k) cnt[k + 1] += cnt[k];
    G.start = cnt;
    G.items.assign(cnt[nc], 0);
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    for (int i = 0; i < P.n; ++i) if (G.cell[i] >= 0) G.items[fill[G.cell[i]]++] = i;
}

// Stencil order of Taylor_Green_Vortex/Distribute_Backgroud_Grid.f90:104-112:
// self, left, right, up-left, up, up-right, down-left, down, down-right.
const int kStencil[9][2] = {{0, 0}, {-1, 0}, {1, 0}, {-1, 1}, {0, 1}, {1, 1}, {-1, -1}, {0, -1}, {1, -1}};

inline bool ms_solver() { return g_cfg.solver == SPH_SOLVER_MS_MODLR_DELTA || g_cfg.solver == SPH_SOLVER_MS_HLLC_DELTA; }

// Particles whose rates are assembled and integrated: water; the moving-square
// driver also integrates inlet/outlet particles (Single_step_compute.f90:273,
// SPH_Time_Iteration.f90:316).
inline bool integrated(int t) { return t == SPH_TYPE_WATER || (ms_solver() && t <= SPH_TYPE_INLET); }

inline bool pair_allowed(int ti, int tj) {
    if (g_cfg.pair_rule == SPH_PAIRS_ONE_FLUID) return !(ti != SPH_TYPE_WATER && tj != SPH_TYPE_WATER);
    if (ti == -2 && tj == -2) return false;
    if (ti == -3 && tj == -3) return false;
    if (ti == -201 && tj == -201) return false;
    return true;
}

// find_particle_pair: Taylor_Green_Vortex/find_particle_pair.f90:64-123.
void find_pairs(const Particles& P, const Grid& G, PairList& L) {
    const int n = P.n;
    std::vector<std::vector<int>> per_i(n);
    #pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n - 1; ++i) {
        int ci = G.cell[i];
        if (ci < 0) continue;
        int cx = ci % G.nx, cy = ci / G.nx;
        std::vector<int>& out = per_i[i];
        for (int s = 0; s < 9; ++s) {
            int nx = cx + kStencil[s][0], ny = cy + kStencil[s][1];
            if (nx < 0 || ny < 0 || nx >= G.nx || ny >= G.ny) continue;
            int c = ny * G.nx + nx;
            for (int t = G.start[c]; t < G.start[c + 1]; ++t) {
                int j = G.items[t];
                if (j <= i) continue;
                if (!pair_allowed(P.type[i], P.type[j])) continue;
                double pd0 = P.x[i] - P.x[j], pd1 = P.y[i] - P.y[j];
                double d = std::sqrt(pd0 * pd0 + pd1 * pd1);
                double hb = (g_cfg.h + g_cfg.h) / 2.0;
                if (d <= (g_cfg.kernel_scale * hb) && d >= g_K.cut_min) out.push_back(j);
            }
        }
    }
    size_t total = 0;
    std::vector<size_t> off(n + 1, 0);
    for (int i = 0; i < n; ++i) { off[i] = total; total += per_i[i].size(); }
    off[n] = total;
    L.pi.resize(total); L.pj.resize(total); L.w.resize(total);
    L.dw0.resize(total); L.dw1.resize(total); L.dx0.resize(total); L.dx1.resize(total);
    #pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; ++i) {
        size_t k = off[i];
        for (int j : per_i[i]) {
            double pd[2] = {P.x[i] - P.x[j], P.y[i] - P.y[j]};
            double d = std::sqrt(pd[0] * pd[0] + pd[1] * pd[1]);
            double hb = (g_cfg.h + g_cfg.h) / 2.0;
            double w, dw[2];
            kernel(d, pd, hb, w, dw);
            L.pi[k] = i; L.pj[k] = j; L.w[k] = w; L.dw0[k] = dw[0]; L.dw1[k] = dw[1];
            L.dx0[k] = pd[0]; L.dx1[k] = pd[1];
            ++k;
        }
    }
}

// Per-particle list of the pairs it appears in, in increasing pair index,
// with the side (0: particle is pair_i, 1: particle is pair_j).
struct Incidence {
    std::vector<size_t> start;
    std::vector<uint32_t> kk;   // pair index
    std::vector<uint8_t> side;
};

void build_incidence(int n, const PairList& L, Incidence& I) {
    std::vector<size_t> cnt(n + 1, 0);
    for (size_t k = 0; k < L.size(); ++k) { cnt[L.pi[k] + 1]++; cnt[L.pj[k] + 1]++; }
    for (int i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
    I.start = cnt;
    I.kk.resize(cnt[n]); I.side.resize(cnt[n]);
    std::vector<size_t> fill(cnt.begin(), cnt.end() - 1);
    for (size_t k = 0; k < L.size(); ++k) {
        size_t a = fill[L.pi[k]]++; I.kk[a] = (uint32_t)k; I.side[a] = 0;
        size_t b = fill[L.pj[k]]++; I.kk[b] = (uint32_t)k; I.side[b] = 1;
    }
}

// Scatter "acc(pair_i) += Ti(k); acc(pair_j) += Tj(k)" in pair order, written
// as a per-particle sum over its incident pairs (same additions, same order).
template <int NC>
void scatter(int n, const Incidence& I, const std::vector<double>* Ti, const std::vector<double>* Tj,
             std::vector<double>* acc) {
    #pragma omp parallel for schedule(static)
    for (int p = 0; p < n; ++p) {
        double s[NC];
        for (int c = 0; c < NC; ++c) s[c] = acc[c][p];
        for (size_t a = I.start[p]; a < I.start[p + 1]; ++a) {
            uint32_t k = I.kk[a];
            if (I.side[a] == 0) for (int c = 0; c < NC; ++c) s[c] = s[c] + Ti[c][k];
            else for (int c = 0; c < NC; ++c) s[c] = s[c] + Tj[c][k];
        }
        for (int c = 0; c < NC; ++c) acc[c][p] = s[c];
    }
}

// Everything single_step_compute produces (plus the intermediates tests look at).
struct Rhs {
    std::vector<double> p, c, vol;
    std::vector<double> fra_v, B[4], binv[4], sdw[2];
    std::vector<int> fs, near;
    std::vector<double> ndwi0, ndwi1, ndwj0, ndwj1;   // Normalized_dwdx_i/j
    std::vector<double> S[3], tau[3];                 // strain xx,xy,yy and tau xx,xy,yy
    std::vector<double> grho[2], gp[2], gu[2], gv[2];
    std::vector<double> drho, acc[2], avg[2];
    std::vector<double> shift[2];
    PairList L;
    Incidence I;
    Grid G;
    long long n_singular = 0;
};

inline void resize_zero(std::vector<double>& a, int n) { a.assign(n, 0.0); }

// Define_freesurface_and_Normailized_derivates:
// Taylor_Green_Vortex/Define_freesurface_and_Normailized_derivates.f90:65-440.
void define_free_surface(const Particles& P, Rhs& R) {
    const int n = P.n;
    const PairList& L = R.L;
    const size_t np = L.size();
    const double sv = g_K.support_volume;
    resize_zero(R.fra_v, n);
    {   // :79-93
        std::vector<double> ti(np), tj(np);
        #pragma omp parallel for
        for (size_t k = 0; k < np; ++k) { ti[k] = R.vol[L.pj[k]] / sv; tj[k] = R.vol[L.pi[k]] / sv; }
        scatter<1>(n, R.I, &ti, &tj, &R.fra_v);
    }
    R.fs.assign(n, 0);
    if (g_cfg.free_surface)           // :119-131 (MS: only with Has_FreeSurface_Or_Not)
        for (int i = 0; i < n; ++i)
            if (P.type[i] == SPH_TYPE_WATER && R.fra_v[i] <= g_K.fs_thr) R.fs[i] = 1;
    {   // :137-159  B(L,o) += (x_j-x_i)_L dwdx_o V ; sum_dwdx
        std::vector<double> ti[6], tj[6];
        for (int c = 0; c < 6; ++c) { ti[c].resize(np); tj[c].resize(np); }
        #pragma omp parallel for
        for (size_t k = 0; k < np; ++k) {
            int i = L.pi[k], j = L.pj[k];
            double pd[2] = {-L.dx0[k], -L.dx1[k]};
            double dw[2] = {L.dw0[k], L.dw1[k]};
            for (int a = 0; a < 2; ++a)
                for (int o = 0; o < 2; ++o) {
                    ti[a * 2 + o][k] = pd[a] * dw[o] * R.vol[j];
                    tj[a * 2 + o][k] = pd[a] * dw[o] * R.vol[i];
                }
            ti[4][k] = dw[0] * R.vol[j]; tj[4][k] = -(dw[0] * R.vol[i]);
            ti[5][k] = dw[1] * R.vol[j]; tj[5][k] = -(dw[1] * R.vol[i]);
        }
        std::vector<double> acc[6];
        for (int c = 0; c < 6; ++c) resize_zero(acc[c], n);
        scatter<6>(n, R.I, ti, tj, acc);
        for (int c = 0; c < 4; ++c) R.B[c] = acc[c];
        R.sdw[0] = acc[4]; R.sdw[1] = acc[5];
    }
    // :168-188 inverse; the reference assigns the identity after a successful
    // inversion (A.1); renormalize=1 keeps the inverse.
    for (int c = 0; c < 4; ++c) R.binv[c].assign(n, (c == 0 || c == 3) ? 1.0 : 0.0);
    R.n_singular = 0;
    for (int i = 0; i < n; ++i) {
        // MS also inverts for outlet particles (MS Define_freesurface...f90:131)
        if (!(P.type[i] == SPH_TYPE_WATER || (ms_solver() && P.type[i] == -202))) continue;
        double A[2][2] = {{R.B[0][i], R.B[1][i]}, {R.B[2][i], R.B[3][i]}}, Rm[2][2];
        int ok = inv2(A, Rm);
        if (!ok) { R.n_singular++; continue; }
        if (g_cfg.renormalize) {
            R.binv[0][i] = Rm[0][0]; R.binv[1][i] = Rm[0][1]; R.binv[2][i] = Rm[1][0]; R.binv[3][i] = Rm[1][1];
        }
    }
    // :295-376 normal vector and geometric test for the candidates
    const double h = g_cfg.h;
    const Grid& G = R.G;
    #pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
        if (!R.fs[i]) continue;
        double nv0 = R.binv[0][i] * R.sdw[0][i] + R.binv[1][i] * R.sdw[1][i];
        double nv1 = R.binv[2][i] * R.sdw[0][i] + R.binv[3][i] * R.sdw[1][i];
        double len = 0.0;
        len = len + nv0 * nv0;
        len = len + nv1 * nv1;
        len = std::sqrt(len);
        if (std::isnan(len)) { R.fs[i] = 0; continue; }
        if (len != 0.0) { nv0 = -nv0 / len; nv1 = -nv1 / len; }
        else { R.fs[i] = 0; continue; }
        double vx = P.x[i] + h * nv0, vy = P.y[i] + h * nv1;
        int ci = G.cell[i];
        int cx = ci % G.nx, cy = ci / G.nx;
        bool keep = true;
        for (int s = 0; s < 9; ++s) {
            int gx = cx + kStencil[s][0], gy = cy + kStencil[s][1];
            if (gx < 0 || gy < 0 || gx >= G.nx || gy >= G.ny) continue;
            int c = gy * G.nx + gx;
            for (int t = G.start[c]; t < G.start[c + 1]; ++t) {
                int j = G.items[t];
                if (P.type[j] != SPH_TYPE_WATER) continue;
                double pd0 = P.x[j] - P.x[i], pd1 = P.y[j] - P.y[i];
                double ji = std::sqrt(pd0 * pd0 + pd1 * pd1);
                double nd = nv0 * pd0 + nv1 * pd1;
                double q0 = P.x[j] - vx, q1 = P.y[j] - vy;
                double jt = std::sqrt(q0 * q0 + q1 * q1);
                if (ji >= g_K.c1414 * h && jt < h) keep = false;
                else if (ji < g_K.c1414 * h && std::acos(nd / ji) <= (g_K.pi / 4.0)) keep = false;
            }
        }
        if (!keep) R.fs[i] = 0;
    }
    // :418-440 near-surface flags
    R.near.assign(n, 0);
    for (size_t k = 0; k < np; ++k) {
        if (R.fs[L.pi[k]] == 1) R.near[L.pj[k]] = 1;
        if (R.fs[L.pj[k]] == 1) R.near[L.pi[k]] = 1;
    }
}

// Normalized_dwdx_i/j = B_i^-1 dwdx, B_j^-1 dwdx (Solver_..._SPS.f90:126-139).
void normalized_gradients(Rhs& R) {
    const PairList& L = R.L;
    const size_t np = L.size();
    R.ndwi0.resize(np); R.ndwi1.resize(np); R.ndwj0.resize(np); R.ndwj1.resize(np);
    #pragma omp parallel for
    for (size_t k = 0; k < np; ++k) {
        int i = L.pi[k], j = L.pj[k];
        R.ndwi0[k] = R.binv[0][i] * L.dw0[k] + R.binv[1][i] * L.dw1[k];
        R.ndwi1[k] = R.binv[2][i] * L.dw0[k] + R.binv[3][i] * L.dw1[k];
        R.ndwj0[k] = R.binv[0][j] * L.dw0[k] + R.binv[1][j] * L.dw1[k];
        R.ndwj1[k] = R.binv[2][j] * L.dw0[k] + R.binv[3][j] * L.dw1[k];
    }
}

// SPS strain tensor and stress: Solver_Normalized_Modified_Linear_Riemann_Delta_SPS.f90:144-182,256-296.
void sps_stress(const Particles& P, Rhs& R) {
    const int n = P.n;
    const PairList& L = R.L;
    const size_t np = L.size();
    std::vector<double> ti[3], tj[3];
    for (int c = 0; c < 3; ++c) { ti[c].resize(np); tj[c].resize(np); }
    #pragma omp parallel for
    for (size_t k = 0; k < np; ++k) {
        int i = L.pi[k], j = L.pj[k];
        double vd0 = -(P.u[i] - P.u[j]), vd1 = -(P.v[i] - P.v[j]);
        ti[0][k] = vd0 * R.ndwi0[k] * R.vol[j];
        ti[1][k] = (vd0 * R.ndwi1[k] + vd1 * R.ndwi0[k]) * R.vol[j];
        ti[2][k] = vd1 * R.ndwi1[k] * R.vol[j];
        tj[0][k] = vd0 * R.ndwj0[k] * R.vol[i];
        tj[1][k] = (vd0 * R.ndwj1[k] + vd1 * R.ndwj0[k]) * R.vol[i];
        tj[2][k] = vd1 * R.ndwj1[k] * R.vol[i];
    }
    for (int c = 0; c < 3; ++c) resize_zero(R.S[c], n);
    scatter<3>(n, R.I, ti, tj, R.S);
    for (int c = 0; c < 3; ++c) resize_zero(R.tau[c], n);
    const double dl = g_K.sps_dl * g_cfg.dx;
    for (int i = 0; i < n; ++i) {
        if (P.type[i] != SPH_TYPE_WATER) continue;
        double sxx = R.S[0][i], sxy = R.S[1][i], syy = R.S[2][i];
        double mes = sxx * sxx + syy * syy + 0.0 * 0.0;
        double les = sxy * sxy + 0.0 * 0.0 + 0.0 * 0.0;
        double abs2 = 2 * mes + les;
        double t = g_K.sps_c012 * dl;
        double nut = (t * t) * std::sqrt(abs2);
        double kk = g_K.sps_23 * nut * (sxx + syy);
        double blin = g_K.sps_blin * (dl * dl) * abs2;
        R.tau[0][i] = (2 * nut * sxx - kk - blin) * P.rho[i];
        R.tau[1][i] = (nut * sxy) * P.rho[i];
        R.tau[2][i] = (2 * nut * syy - kk - blin) * P.rho[i];
    }
}

// grad(phi) = sum (phi_j - phi_i) V B^-1 dwdx for the listed fields
// (Solver_Normalized_MUSCL_Linear_Riemann_Delta_SPS.f90:151-185; the rho part
// also Solver_Normalized_Modified_Linear_Riemann_Delta_SPS.f90:508-526).
void gradients(const Particles& P, Rhs& R, bool muscl) {
    const int n = P.n;
    const PairList& L = R.L;
    const size_t np = L.size();
    const int nf = muscl ? 4 : 1;
    std::vector<double> ti[8], tj[8];
    for (int c = 0; c < 2 * nf; ++c) { ti[c].resize(np); tj[c].resize(np); }
    #pragma omp parallel for
    for (size_t k = 0; k < np; ++k) {
        int i = L.pi[k], j = L.pj[k];
        double d[4];
        d[0] = -(P.rho[i] - P.rho[j]);
        if (muscl) {
            d[1] = R.p[j] - R.p[i];
            d[2] = -(P.u[i] - P.u[j]);
            d[3] = -(P.v[i] - P.v[j]);
        }
        double mi0 = R.binv[0][i] * L.dw0[k] + R.binv[1][i] * L.dw1[k];
        double mi1 = R.binv[2][i] * L.dw0[k] + R.binv[3][i] * L.dw1[k];
        double mj0 = R.binv[0][j] * L.dw0[k] + R.binv[1][j] * L.dw1[k];
        double mj1 = R.binv[2][j] * L.dw0[k] + R.binv[3][j] * L.dw1[k];
        for (int f = 0; f < nf; ++f) {
            ti[2 * f][k] = d[f] * R.vol[j] * mi0; ti[2 * f + 1][k] = d[f] * R.vol[j] * mi1;
            tj[2 * f][k] = d[f] * R.vol[i] * mj0; tj[2 * f + 1][k] = d[f] * R.vol[i] * mj1;
        }
    }
    std::vector<double> acc[8];
    for (int c = 0; c < 2 * nf; ++c) resize_zero(acc[c], n);
    if (muscl) scatter<8>(n, R.I, ti, tj, acc); else scatter<2>(n, R.I, ti, tj, acc);
    R.grho[0] = acc[0]; R.grho[1] = acc[1];
    if (muscl) { R.gp[0] = acc[2]; R.gp[1] = acc[3]; R.gu[0] = acc[4]; R.gu[1] = acc[5]; R.gv[0] = acc[6]; R.gv[1] = acc[7]; }
}

// Main pair loop of the two linear-Riemann solvers
// (Solver_Normalized_Modified_Linear_Riemann_Delta_SPS.f90:300-502,
//  Solver_Normalized_MUSCL_Linear_Riemann_Delta_SPS.f90:458-682)
// and the delta-SPH density diffusion (:552-583 / :690-721).  dsph: the plain
// method Solver_Normalized_Delta_SPH_SPS.f90, whose pair loop (:324-512) has no
// Riemann state (continuity with v_i - v_j, pressure p_i + p_j), no XSPH
// (:286-322 commented out, average_velocity zeroed by single_step_compute.f90:122)
// and the Antuono density diffusion (:610-636); its energy equation (dedt,
// :379-380, 435-468) feeds nothing else under the Tait EOS and is not formed.
void riemann_solver(const Particles& P, Rhs& R, bool muscl, bool dsph) {
    const int n = P.n;
    const PairList& L = R.L;
    const size_t np = L.size();
    const sph_config& C = g_cfg;
    const double hbar = (C.h + C.h) / 2.0;
    // term channels: 0 cont, 1-2 internal, 3-4 AV, 5-6 laplacian, 7-8 art_int, 9-10 SPS, 11-12 XSPH, 13 delta
    const int NT = 14;
    std::vector<double> ti[NT], tj[NT];
    for (int c = 0; c < NT; ++c) { ti[c].assign(np, 0.0); tj[c].assign(np, 0.0); }
    #pragma omp parallel for schedule(static)
    for (size_t k = 0; k < np; ++k) {
        const int i = L.pi[k], j = L.pj[k];
        const double Vi = R.vol[i], Vj = R.vol[j];
        const double ri = P.rho[i], rj = P.rho[j];
        const double ndi[2] = {R.ndwi0[k], R.ndwi1[k]}, ndj[2] = {R.ndwj0[k], R.ndwj1[k]};
        const double dwk[2] = {L.dw0[k], L.dw1[k]};
        const double cbar = (R.c[i] + R.c[j]) / 2.0;
        const double rbar = (ri + rj) / 2.0;
        double PL, PR, Pbar, vI[2], vJ[2], vbar[2], e[2], d;
        if (!muscl) {
            PL = R.p[i]; PR = R.p[j]; Pbar = (PL + PR) / 2.0;
            vI[0] = P.u[i]; vI[1] = P.v[i]; vJ[0] = P.u[j]; vJ[1] = P.v[j];
            vbar[0] = (vI[0] + vJ[0]) / 2.0; vbar[1] = (vI[1] + vJ[1]) / 2.0;
            double xij[2] = {L.dx0[k], L.dx1[k]};
            d = std::sqrt(xij[0] * xij[0] + xij[1] * xij[1]);
            e[0] = -xij[0] / d; e[1] = -xij[1] / d;
        } else {
            double xij[2] = {-L.dx0[k], -L.dx1[k]};   // j - i
            d = std::sqrt(xij[0] * xij[0] + xij[1] * xij[1]);
            e[0] = xij[0] / d; e[1] = xij[1] / d;
            double li, lj;
            double Di = 0.5 * (R.gp[0][i] * xij[0] + R.gp[1][i] * xij[1]);
            double Dj = -0.5 * (R.gp[0][j] * xij[0] + R.gp[1][j] * xij[1]);
            muscl_limiter(Di, Dj, R.p[j] - R.p[i], li, lj);
            PL = R.p[i] + li; PR = R.p[j] - lj; Pbar = (R.p[i] + R.p[j]) / 2.0;
            double vd0 = -(P.u[i] - P.u[j]), vd1 = -(P.v[i] - P.v[j]);
            Di = 0.5 * (R.gu[0][i] * xij[0] + R.gu[1][i] * xij[1]);
            Dj = -0.5 * (R.gu[0][j] * xij[0] + R.gu[1][j] * xij[1]);
            muscl_limiter(Di, Dj, vd0, li, lj);
            vI[0] = P.u[i] + li; vJ[0] = P.u[j] - lj;
            Di = 0.5 * (R.gv[0][i] * xij[0] + R.gv[1][i] * xij[1]);
            Dj = -0.5 * (R.gv[0][j] * xij[0] + R.gv[1][j] * xij[1]);
            muscl_limiter(Di, Dj, vd1, li, lj);
            vI[1] = P.v[i] + li; vJ[1] = P.v[j] - lj;
            vbar[0] = (P.u[i] + P.u[j]) / 2.0; vbar[1] = (P.v[i] + P.v[j]) / 2.0;
        }
        double UL = vI[0] * e[0] + vI[1] * e[1];
        double UR = vJ[0] * e[0] + vJ[1] * e[1];
        double Ubar = (UL + UR) / 2.0;
        double Us = Ubar + 0.5 * (PL - PR) / (rbar * g_K.sqrt_c0);
        double vs[2] = {(Us - Ubar) * e[0] + vbar[0], (Us - Ubar) * e[1] + vbar[1]};
        double bR = std::min(3.0 * (std::max((UL - UR), 0.0)), cbar);
        double Ps = Pbar + 0.5 * bR * rbar * (UL - UR);
        double vIs[2], vJs[2], IPs, JPs;
        if (R.near[i] == 1) { vIs[0] = vbar[0]; vIs[1] = vbar[1]; IPs = Pbar; }
        else { vIs[0] = vs[0]; vIs[1] = vs[1]; IPs = Ps; }
        if (R.near[j] == 1) { vJs[0] = vbar[0]; vJs[1] = vbar[1]; JPs = Pbar; }
        else { vJs[0] = vs[0]; vJs[1] = vs[1]; JPs = Ps; }
        double rho_ij = 1.0 / (ri * rj);
        if (dsph) {
            // Solver_Normalized_Delta_SPH_SPS.f90:335-374
            const double vd[2] = {P.u[i] - P.u[j], P.v[i] - P.v[j]};
            double tmi = vd[0] * ndi[0] + vd[1] * ndi[1];
            double tmj = vd[0] * ndj[0] + vd[1] * ndj[1];
            ti[0][k] = ri * Vj * tmi;
            tj[0][k] = rj * Vi * tmj;
            for (int a = 0; a < 2; ++a) {
                double tpi = -(R.p[i] + R.p[j]) * ndi[a] * rho_ij;
                double tpj = -(R.p[i] + R.p[j]) * ndj[a] * rho_ij;
                ti[1 + a][k] = P.mass[j] * tpi;
                tj[1 + a][k] = -(P.mass[i] * tpj);
            }
        } else {
            double tmi = (vI[0] - vIs[0]) * ndi[0] + (vI[1] - vIs[1]) * ndi[1];
            double tmj = -((vJ[0] - vJs[0]) * ndj[0] + (vJ[1] - vJs[1]) * ndj[1]);
            ti[0][k] = 2 * ri * Vj * tmi;
            tj[0][k] = 2 * rj * Vi * tmj;
            for (int a = 0; a < 2; ++a) {
                double tpi = -2 * IPs * ndi[a] * rho_ij;
                double tpj = -2 * JPs * ndj[a] * rho_ij;
                ti[1 + a][k] = P.mass[j] * tpi;
                tj[1 + a][k] = -(P.mass[i] * tpj);
            }
        }
        // artificial viscosity (:392-417)
        double vij[2] = {P.u[i] - P.u[j], P.v[i] - P.v[j]};
        double xij[2] = {L.dx0[k], L.dx1[k]};
        double r2 = xij[0] * xij[0] + xij[1] * xij[1];
        double vx = vij[0] * xij[0] + vij[1] * xij[1];
        if (vx < 0.0) {
            double fh = C.fai * hbar;
            double phi1 = hbar * vx / (r2 + fh * fh);
            double Pi = (-C.alpha * cbar * phi1 + C.beta * (phi1 * phi1)) / rbar;
            for (int a = 0; a < 2; ++a) {
                ti[3 + a][k] = P.mass[j] * (-Pi * ndi[a]);
                tj[3 + a][k] = -(P.mass[i] * (-Pi * ndj[a]));
            }
        }
        // Morris laplacian (:432-436)
        double rdi = xij[0] * ndi[0] + xij[1] * ndi[1];
        double rdj = xij[0] * ndj[0] + xij[1] * ndj[1];
        for (int a = 0; a < 2; ++a) {
            ti[5 + a][k] = Vj * 2 * C.nu * rdi / r2 * vij[a];
            tj[5 + a][k] = -(Vi * 2 * C.nu * rdj / r2 * vij[a]);
        }
        // delta-alpha artificial internal acceleration (:442-446)
        double tt = C.delta_alpha * hbar * cbar * vx / r2;
        for (int a = 0; a < 2; ++a) {
            ti[7 + a][k] = tt * ndi[a] * C.rho0 / ri * Vj;
            tj[7 + a][k] = -(tt * ndj[a] * C.rho0 / rj * Vi);
        }
        // SPS force with the unnormalised gradient (:450-492).  The Fortran
        // does not reset temp_p between the x and y component, so the y
        // component carries the scaled x term (reproduced with reference_literals).
        double tp = 0.0;
        tp = tp + (R.tau[0][i] + R.tau[0][j]) * dwk[0];
        tp = tp + (R.tau[1][i] + R.tau[1][j]) * dwk[1];
        tp = tp * rho_ij;
        ti[9][k] = P.smass[j] * tp; tj[9][k] = -(P.smass[i] * tp);
        if (!C.reference_literals) tp = 0.0;
        tp = tp + (R.tau[2][i] + R.tau[2][j]) * dwk[1] + (R.tau[1][i] + R.tau[1][j]) * dwk[0];
        tp = tp * rho_ij;
        ti[10][k] = P.smass[j] * tp; tj[10][k] = -(P.smass[i] * tp);
        // XSPH average velocity (:495-500, modified linear Riemann solver only)
        if (!muscl && !dsph) {
            for (int a = 0; a < 2; ++a) {
                ti[11 + a][k] = -(C.xsph_eps * 2 * P.mass[j] * vij[a] / (ri + rj) * L.w[k]);
                tj[11 + a][k] = C.xsph_eps * 2 * P.mass[i] * vij[a] / (ri + rj) * L.w[k];
            }
        }
    }
    std::vector<double> cont(n, 0.0), accs[12];
    for (int c = 0; c < 12; ++c) resize_zero(accs[c], n);
    scatter<1>(n, R.I, &ti[0], &tj[0], &cont);
    scatter<12>(n, R.I, &ti[1], &tj[1], accs);
    if (!muscl) gradients(P, R, false);   // modified solver computes grad rho after the main loop
    // delta-SPH (:552-583)
    #pragma omp parallel for schedule(static)
    for (size_t k = 0; k < np; ++k) {
        const int i = L.pi[k], j = L.pj[k];
        double pd[2] = {-L.dx0[k], -L.dx1[k]};
        double r2 = pd[0] * pd[0] + pd[1] * pd[1];
        double drho = -(P.rho[i] - P.rho[j]);
        double sg0 = R.grho[0][i] + R.grho[0][j], sg1 = R.grho[1][i] + R.grho[1][j];
        double cbar = (R.c[i] + R.c[j]) / 2.0;
        if (dsph) {
            // Solver_Normalized_Delta_SPH_SPS.f90:610-636
            double ps[2] = {2 * drho / r2 * pd[0] - sg0, 2 * drho / r2 * pd[1] - sg1};
            double tmi = ps[0] * R.ndwi0[k] + ps[1] * R.ndwi1[k];
            double tmj = ps[0] * R.ndwj0[k] + ps[1] * R.ndwj1[k];
            ti[13][k] = C.delta * hbar * cbar * tmi * R.vol[j];
            tj[13][k] = -(C.delta * hbar * cbar * tmj * R.vol[i]);
            continue;
        }
        double psi = drho - 0.5 * (sg0 * pd[0] + sg1 * pd[1]);
        double tmi = (pd[0] * R.ndwi0[k] + pd[1] * R.ndwi1[k]) / r2;
        double tmj = (pd[0] * R.ndwj0[k] + pd[1] * R.ndwj1[k]) / r2;
        ti[13][k] = 2 * C.delta * hbar * cbar * psi * tmi * R.vol[j];
        tj[13][k] = -(2 * C.delta * hbar * cbar * psi * tmj * R.vol[i]);
    }
    std::vector<double> corr(n, 0.0);
    scatter<1>(n, R.I, &ti[13], &tj[13], &corr);
    // assembly (single_step_compute.f90:152-171; drhodt += artifical_rho_correct, Solver :627-635)
    R.drho.assign(n, 0.0);
    for (int a = 0; a < 2; ++a) { R.acc[a].assign(n, 0.0); R.avg[a].assign(n, 0.0); }
    for (int i = 0; i < n; ++i) {
        R.drho[i] = cont[i];
        R.avg[0][i] = accs[10][i]; R.avg[1][i] = accs[11][i];
        if (P.type[i] != SPH_TYPE_WATER) continue;
        for (int a = 0; a < 2; ++a) {
            double internal = accs[0 + a][i], av = accs[2 + a][i], lap = accs[4 + a][i];
            double art = accs[6 + a][i], sps = accs[8 + a][i];
            R.acc[a][i] = internal + 0.0 + av + art + sps + lap;
        }
        R.drho[i] = R.drho[i] + corr[i];
    }
}

// The HLLC pair state of Moving_Square.../Solver_Normalized_HLLC_Riemann_Delta.f90:207-322:
// velocities rotated into the pair frame (normal e = (x_j - x_i)/|x_j - x_i|),
// acoustic star velocity and pressure (:225-228), rho* from the linear equation of
// state (:230), wave speeds with the shock factor guarded by rho_K > rho* (:239-278),
// the state sampled at x/t = the mean normal velocity (:281-317), then rotated back,
// P* = c0^2 (rho_HLLC - rho0) + p_b (:321-322).
void hllc_state(const double vI[2], const double vJ[2], const double vbar[2], const double e[2], double rL,
                double rR, double cL, double cR, double PL, double PR, double vs[2], double& Ps) {
    const sph_config& C = g_cfg;
    const double T[2][2] = {{e[0], e[1]}, {-e[1], e[0]}};
    const double VL[2] = {T[0][0] * vI[0] + T[0][1] * vI[1], T[1][0] * vI[0] + T[1][1] * vI[1]};
    const double VR[2] = {T[0][0] * vJ[0] + T[0][1] * vJ[1], T[1][0] * vJ[0] + T[1][1] * vJ[1]};
    const double V0 = T[0][0] * vbar[0] + T[0][1] * vbar[1];
    const double Us = (VR[0] * cL * rL + VL[0] * cR * rR + PL - PR) / (rL * cL + rR * cR);
    double Pst = (PR * cL * rL + PL * cR * rR - cL * rL * cR * rR * (VR[0] - VL[0])) / (rL * cL + rR * cR);
    const double rst = (Pst - C.background_p) / C.c0sq + C.rho0;
    double QL = 1.0, QR = 1.0;
    if (!(Pst <= PL) && rL > rst) QL = std::sqrt((rst / rL) * (Pst - PL) / (rL - rst)) / cL;
    const double SL = VL[0] - cL * QL;
    if (!(Pst <= PR) && rR > rst) QR = std::sqrt((rst / rR) * (Pst - PR) / (rR - rst)) / cR;
    const double SR = VR[0] + cR * QR;
    const double Sst = Us, xt = V0;
    double rH, VH[2];
    if (SL > xt) { rH = rL; VH[0] = VL[0]; VH[1] = VL[1]; }
    else if (Sst >= xt && xt >= SL) {
        double q = rL * ((SL - VL[0]) / (SL - Sst));
        rH = q; VH[0] = (Sst * q) / rH; VH[1] = (VL[1] * q) / rH;
    } else if (SR >= xt && xt >= Sst) {
        double q = rR * ((SR - VR[0]) / (SR - Sst));
        rH = q; VH[0] = (Sst * q) / rH; VH[1] = (VR[1] * q) / rH;
    } else { rH = rR; VH[0] = VR[0]; VH[1] = VR[1]; }
    vs[0] = T[0][0] * VH[0] + T[1][0] * VH[1];
    vs[1] = T[0][1] * VH[0] + T[1][1] * VH[1];
    Ps = C.c0sq * (rH - C.rho0) + C.background_p;
}

// The moving-square solvers: Moving_Square.../Solver_Normalized_Modified_Linear_Riemann_Delta.f90
// and Solver_Normalized_HLLC_Riemann_Delta.f90 (no SPS; XSPH average velocity
// computed first and added to the continuity flux; laplacianTerm switch), with
// the assembly of Moving_Square.../Single_step_compute.f90:253-283.
void ms_riemann_solver(const Particles& P, Rhs& R, bool hllc) {
    const int n = P.n;
    const PairList& L = R.L;
    const size_t np = L.size();
    const sph_config& C = g_cfg;
    const double hbar = (C.h + C.h) / 2.0;
    gradients(P, R, false);                        // grad rho with the normalised gradients (:100-112)
    {   // XSPH average velocity (:114-121)
        std::vector<double> ti[2], tj[2];
        for (int c = 0; c < 2; ++c) { ti[c].resize(np); tj[c].resize(np); resize_zero(R.avg[c], n); }
        #pragma omp parallel for
        for (size_t k = 0; k < np; ++k) {
            const int i = L.pi[k], j = L.pj[k];
            const double vd[2] = {P.u[i] - P.u[j], P.v[i] - P.v[j]};
            for (int a = 0; a < 2; ++a) {
                ti[a][k] = -(C.xsph_eps * P.mass[j] * vd[a] / (P.rho[i] + P.rho[j]) * L.w[k]);
                tj[a][k] = C.xsph_eps * P.mass[i] * vd[a] / (P.rho[i] + P.rho[j]) * L.w[k];
            }
        }
        scatter<2>(n, R.I, ti, tj, R.avg);
    }
    // channels: 0 cont, 1-2 internal, 3-4 AV, 5-6 laplacian, 7-8 art_int
    const int NT = 9;
    std::vector<double> ti[NT], tj[NT];
    for (int c = 0; c < NT; ++c) { ti[c].assign(np, 0.0); tj[c].assign(np, 0.0); }
    #pragma omp parallel for schedule(static)
    for (size_t k = 0; k < np; ++k) {
        const int i = L.pi[k], j = L.pj[k];
        const double Vi = R.vol[i], Vj = R.vol[j];
        const double ri = P.rho[i], rj = P.rho[j];
        const double ndi[2] = {R.ndwi0[k], R.ndwi1[k]}, ndj[2] = {R.ndwj0[k], R.ndwj1[k]};
        const double cbar = (R.c[i] + R.c[j]) / 2.0;
        const double rbar = (ri + rj) / 2.0;
        const double PL = R.p[i], PR = R.p[j], Pbar = (PL + PR) / 2.0;
        const double vI[2] = {P.u[i], P.v[i]}, vJ[2] = {P.u[j], P.v[j]};
        const double vbar[2] = {(vI[0] + vJ[0]) / 2.0, (vI[1] + vJ[1]) / 2.0};
        const double xij[2] = {L.dx0[k], L.dx1[k]};
        const double d = std::sqrt(xij[0] * xij[0] + xij[1] * xij[1]);
        const double e[2] = {-xij[0] / d, -xij[1] / d};
        double vs[2], Ps;
        if (!hllc) {
            double UL = vI[0] * e[0] + vI[1] * e[1];
            double UR = vJ[0] * e[0] + vJ[1] * e[1];
            double Ubar = (UL + UR) / 2.0;
            double Us = Ubar + 0.5 * (PL - PR) / (rbar * g_K.sqrt_c0);
            vs[0] = (Us - Ubar) * e[0] + vbar[0]; vs[1] = (Us - Ubar) * e[1] + vbar[1];
            double bR = std::min(3.0 * (std::max((UL - UR), 0.0)), cbar);
            Ps = Pbar + 0.5 * bR * rbar * (UL - UR);
        } else {
            hllc_state(vI, vJ, vbar, e, ri, rj, R.c[i], R.c[j], PL, PR, vs, Ps);
        }
        double vIs[2], vJs[2], IPs, JPs;
        if (R.near[i] == 1) { vIs[0] = vbar[0]; vIs[1] = vbar[1]; IPs = Pbar; }
        else { vIs[0] = vs[0]; vIs[1] = vs[1]; IPs = Ps; }
        if (R.near[j] == 1) { vJs[0] = vbar[0]; vJs[1] = vbar[1]; JPs = Pbar; }
        else { vJs[0] = vs[0]; vJs[1] = vs[1]; JPs = Ps; }
        double vdi[2] = {vI[0] - vIs[0] + R.avg[0][i] - R.avg[0][j], vI[1] - vIs[1] + R.avg[1][i] - R.avg[1][j]};
        double vdj[2] = {vJ[0] - vJs[0] + R.avg[0][j] - R.avg[0][i], vJ[1] - vJs[1] + R.avg[1][j] - R.avg[1][i]};
        double tmi = vdi[0] * ndi[0] + vdi[1] * ndi[1];
        double tmj = -(vdj[0] * ndj[0] + vdj[1] * ndj[1]);
        ti[0][k] = 2 * ri * Vj * tmi;
        tj[0][k] = 2 * rj * Vi * tmj;
        double rho_ij = 1.0 / (ri * rj);
        for (int a = 0; a < 2; ++a) {
            ti[1 + a][k] = P.mass[j] * (-2 * IPs * ndi[a] * rho_ij);
            tj[1 + a][k] = -(P.mass[i] * (-2 * JPs * ndj[a] * rho_ij));
        }
        double vij[2] = {P.u[i] - P.u[j], P.v[i] - P.v[j]};
        double r2 = xij[0] * xij[0] + xij[1] * xij[1];
        double vx = vij[0] * xij[0] + vij[1] * xij[1];
        if (vx < 0.0) {
            double fh = C.fai * hbar;
            double phi1 = hbar * vx / (r2 + fh * fh);
            double Pi = (-C.alpha * cbar * phi1 + C.beta * (phi1 * phi1)) / rbar;
            for (int a = 0; a < 2; ++a) {
                ti[3 + a][k] = P.mass[j] * (-Pi * ndi[a]);
                tj[3 + a][k] = -(P.mass[i] * (-Pi * ndj[a]));
            }
        }
        if (C.laplacian == 1) {
            double rdi = xij[0] * ndi[0] + xij[1] * ndi[1];
            double rdj = xij[0] * ndj[0] + xij[1] * ndj[1];
            for (int a = 0; a < 2; ++a) {
                ti[5 + a][k] = Vj * 2 * C.nu * rdi / r2 * vij[a];
                tj[5 + a][k] = -(Vi * 2 * C.nu * rdj / r2 * vij[a]);
            }
        } else {
            for (int a = 0; a < 2; ++a) {
                ti[5 + a][k] = Vj * 2 * (2 + 2) * C.nu * vx / r2 * ndi[a];
                tj[5 + a][k] = -(Vi * 2 * (2 + 2) * C.nu * vx / r2 * ndj[a]);
            }
        }
        double tt = C.delta_alpha * hbar * cbar * vx / r2;
        for (int a = 0; a < 2; ++a) {
            ti[7 + a][k] = tt * ndi[a] * C.rho0 / ri * Vj;
            tj[7 + a][k] = -(tt * ndj[a] * C.rho0 / rj * Vi);
        }
    }
    std::vector<double> cont(n, 0.0), accs[8];
    for (int c = 0; c < 8; ++c) resize_zero(accs[c], n);
    scatter<1>(n, R.I, &ti[0], &tj[0], &cont);
    scatter<8>(n, R.I, &ti[1], &tj[1], accs);
    // delta-SPH (:531-545)
    std::vector<double> dti(np), dtj(np), corr(n, 0.0);
    #pragma omp parallel for schedule(static)
    for (size_t k = 0; k < np; ++k) {
        const int i = L.pi[k], j = L.pj[k];
        double pd[2] = {-L.dx0[k], -L.dx1[k]};
        double r2 = pd[0] * pd[0] + pd[1] * pd[1];
        double drho = -(P.rho[i] - P.rho[j]);
        double sg0 = R.grho[0][i] + R.grho[0][j], sg1 = R.grho[1][i] + R.grho[1][j];
        double psi = drho - 0.5 * (sg0 * pd[0] + sg1 * pd[1]);
        double tmi = (pd[0] * R.ndwi0[k] + pd[1] * R.ndwi1[k]) / r2;
        double tmj = (pd[0] * R.ndwj0[k] + pd[1] * R.ndwj1[k]) / r2;
        double cbar = (R.c[i] + R.c[j]) / 2.0;
        dti[k] = 2 * C.delta * hbar * cbar * psi * tmi * R.vol[j];
        dtj[k] = -(2 * C.delta * hbar * cbar * psi * tmj * R.vol[i]);
    }
    scatter<1>(n, R.I, &dti, &dtj, &corr);
    R.drho.assign(n, 0.0);
    for (int a = 0; a < 2; ++a) R.acc[a].assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
        R.drho[i] = cont[i];
        if (!integrated(P.type[i])) continue;
        for (int a = 0; a < 2; ++a)
            R.acc[a][i] = accs[0 + a][i] + 0.0 + accs[2 + a][i] + accs[6 + a][i] + 0.0 + accs[4 + a][i];
        R.drho[i] = R.drho[i] + corr[i];
    }
}

// Calculate_Body_Force (Moving_Square.../Calculate_Body_Force.f90:53-142) and the
// sums of Moving_Square.../Single_step_compute.f90:228-243 (no gravity).
void body_force(const Particles& P, const Rhs& R, double out[6]) {
    const int n = P.n;
    const PairList& L = R.L;
    std::vector<double> bp[2], bv[2];
    for (int c = 0; c < 2; ++c) { bp[c].assign(n, 0.0); bv[c].assign(n, 0.0); }
    std::vector<int> nearb(n, 0);
    const double nu = g_cfg.nu;
    for (size_t k = 0; k < L.size(); ++k) {
        const int i = L.pi[k], j = L.pj[k];
        if (P.itype[i] != SPH_TYPE_BODY && P.itype[j] != SPH_TYPE_BODY) continue;
        double vij[2] = {P.u[i] - P.u[j], P.v[i] - P.v[j]};
        double xij[2] = {L.dx0[k], L.dx1[k]};
        double r2 = xij[0] * xij[0] + xij[1] * xij[1];
        double vx = vij[0] * xij[0] + vij[1] * xij[1];
        double ndi[2] = {R.ndwi0[k], R.ndwi1[k]}, ndj[2] = {R.ndwj0[k], R.ndwj1[k]};
        if (P.itype[j] == SPH_TYPE_BODY) {
            nearb[i] = 1;
            for (int a = 0; a < 2; ++a) bp[a][i] = bp[a][i] - R.vol[j] * (R.p[i] + R.p[j]) * ndi[a];
            if (g_cfg.laplacian == 1) {
                double rd = xij[0] * ndi[0] + xij[1] * ndi[1];
                for (int a = 0; a < 2; ++a) bv[a][i] = bv[a][i] + P.rho[i] * R.vol[j] * 2 * nu * rd / r2 * vij[a];
            } else {
                for (int a = 0; a < 2; ++a) bv[a][i] = bv[a][i] + P.rho[i] * R.vol[j] * 2 * (2 + 2) * nu * vx / r2 * ndi[a];
            }
        }
        if (P.itype[i] == SPH_TYPE_BODY) {
            nearb[j] = 1;
            for (int a = 0; a < 2; ++a) bp[a][j] = bp[a][j] + R.vol[i] * (R.p[i] + R.p[j]) * ndj[a];
            if (g_cfg.laplacian == 1) {
                double rd = xij[0] * ndj[0] + xij[1] * ndj[1];
                for (int a = 0; a < 2; ++a) bv[a][j] = bv[a][j] - P.rho[j] * R.vol[i] * 2 * nu * rd / r2 * vij[a];
            } else {
                for (int a = 0; a < 2; ++a) bv[a][j] = bv[a][j] - P.rho[j] * R.vol[i] * 2 * (2 + 2) * nu * vx / r2 * ndj[a];
            }
        }
    }
    for (int c = 0; c < 6; ++c) out[c] = 0.0;
    for (int i = 0; i < n; ++i) {
        if (!nearb[i]) continue;
        for (int a = 0; a < 2; ++a) {
            out[0 + a] = out[0 + a] + R.vol[i] * bp[a][i];
            out[2 + a] = out[2 + a] + R.vol[i] * bv[a][i];
            out[4 + a] = out[4 + a] + R.vol[i] * (bp[a][i] + bv[a][i] + 0.0);
        }
    }
}

// Ghost-assignment inputs of the moving-square driver: the wall labels
// (Boundary_particle_type, host index order), the body's Custom_velocity and
// Custom_accleration, and Real_physical_time.
std::vector<int> g_labels;
double g_bvel[2] = {0.0, 0.0}, g_bacc[2] = {0.0, 0.0};
double g_time = 0.0;
int g_n_host = 0;

// Assign_boundary_particles, fixed-ghost part (Moving_Square.../Assign_boundary_particles.f90:
// 611-941) with MLS_order_Boundary = 1: Fai_j = W_j V_j / sum W V over the
// non-ghost particles within kernel_scale * 1.2 h; pressure, velocity and mass
// interpolated (pressure with the gravity / body-acceleration term), body ghosts
// take the body velocity, wall ghosts the characteristic-variable branch during
// the shock release time (labels -6, -7; other labels keep the zero pressure
// they start from) and the mirrored velocity; then the density from the
// linear equation of state, or the rest state without neighbours.
void assign_ghosts(Particles& P, Rhs& R) {
    const sph_config& C = g_cfg;
    const bool q = C.reference_literals != 0;
    const double hg = (q ? (double)(float)C.ghost_h_factor : C.ghost_h_factor) * C.h;
    const double rg = C.kernel_scale * hg;
    const int n_host = std::min(g_n_host, P.n);
    // every ghost reads only non-ghost particles, so the order of assignment is free
    for (int i = 0; i < n_host; ++i) {
        if (P.type[i] != SPH_TYPE_FIX_GHOST) continue;
        const bool body = P.itype[i] == SPH_TYPE_BODY;
        const double ge[2] = {C.gravity[0] + (body ? g_bacc[0] : 0.0), C.gravity[1] + (body ? g_bacc[1] : 0.0)};
        std::vector<int> nb;
        std::vector<double> W;
        for (int j = 0; j < P.n; ++j) {
            if (P.type[j] == SPH_TYPE_FIX_GHOST || P.type[j] == SPH_TYPE_ILL || P.type[j] == 0) continue;
            double pd[2] = {P.x[i] - P.x[j], P.y[i] - P.y[j]};
            const double d = std::sqrt(pd[0] * pd[0] + pd[1] * pd[1]);
            if (!(d <= rg)) continue;
            double w, dw[2];
            kernel(d, pd, hg, w, dw);
            nb.push_back(j);
            W.push_back(w * P.mass[j] / P.rho[j]);
        }
        double pint = 0.0, uint = 0.0, vint = 0.0, m = 0.0;
        if (nb.size() >= 3) {
            double A = 0.0;
            for (double w : W) A += w;
            const double ainv = 1.0 / A;
            for (size_t k = 0; k < nb.size(); ++k) {
                const int j = nb[k];
                const double fai = ainv * W[k];
                const double pd0 = P.x[i] - P.x[j], pd1 = P.y[i] - P.y[j];
                pint = pint + R.p[j] * fai + P.rho[j] * fai * (ge[0] * pd0 + ge[1] * pd1);
                uint = uint + P.u[j] * fai;
                vint = vint + P.v[j] * fai;
                m = m + P.mass[j] * fai;
            }
        }
        double u, v, p = 0.0;
        const int lab = i < (int)g_labels.size() ? g_labels[i] : 0;
        if (body) {
            u = g_bvel[0]; v = g_bvel[1]; p = pint;
        } else {
            if (0.0 < g_time && g_time <= C.shock_release_time) {
                const double ri = (pint - C.background_p) / C.c0sq + C.rho0;
                const double c = g_K.sqrt_c0 * pw3(ri / C.rho0);
                u = uint; v = vint;
                if (lab == -6) {
                    const double J2 = ri * c * (vint - 0.0) + (pint - 0.0), J3 = -ri * c * (vint - 0.0) + (pint - 0.0);
                    v = 0.0 + (J2 - J3) / (2 * ri * c);
                    p = 0.0 + 0.5 * (J2 + J3);
                } else if (lab == -7) {
                    const double J2 = ri * c * (uint - 0.0) + (pint - 0.0), J3 = -ri * c * (uint - 0.0) + (pint - 0.0);
                    u = 0.0 + (J2 - J3) / (2 * ri * c);
                    p = 0.0 + 0.5 * (J2 + J3);
                }
            } else {
                u = uint; v = vint; p = pint;
            }
            if (lab == -6) { if (C.wall_bc == 1) v = -v; else { u = -u; v = -v; } }
            else if (lab == -7) { u = -u; v = -v; }
            else if (lab == -8) { if (C.wall_bc == 1) u = -u; else { u = -u; v = -v; } }
        }
        double rho, c;
        if (m != 0.0) {
            rho = (p - C.background_p) / C.c0sq + C.rho0;
            c = g_K.sqrt_c0 * pw3(rho / C.rho0);
        } else {
            u = 0.0; v = 0.0; p = 0.0; rho = C.rho0; m = 0.0; c = g_K.sqrt_c0;
        }
        P.u[i] = u; P.v[i] = v; P.rho[i] = rho; P.mass[i] = m; P.smass[i] = m;
        R.p[i] = p; R.c[i] = c; R.vol[i] = m / rho;
    }
}

// single_step_compute (Taylor_Green_Vortex/single_step_compute.f90:62-171).
void single_step_compute(Particles& P, Rhs& R) {
    const int n = P.n;
    R.p.assign(n, 0.0); R.c.assign(n, 0.0); R.vol.assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
        if (P.type[i] == SPH_TYPE_ILL) continue;
        eos(P.rho[i], R.p[i], R.c[i]);
    }
    for (int i = 0; i < n; ++i) R.vol[i] = P.mass[i] / P.rho[i];   // Assign_boundary_particles.f90:303-308
    if (g_cfg.ghost_assign) assign_ghosts(P, R);    // MS Single_step_compute.f90:73
    build_grid(P, R.G);
    R.L = PairList();
    find_pairs(P, R.G, R.L);
    build_incidence(n, R.L, R.I);
    define_free_surface(P, R);
    normalized_gradients(R);
    if (ms_solver()) {
        for (int c = 0; c < 3; ++c) { resize_zero(R.S[c], n); resize_zero(R.tau[c], n); }
        ms_riemann_solver(P, R, g_cfg.solver == SPH_SOLVER_MS_HLLC_DELTA);
        return;
    }
    const bool muscl = g_cfg.solver == SPH_SOLVER_MUSCL_DELTA_SPS;
    if (muscl) {
        gradients(P, R, true);
        if (g_muscl_grad_scale != 1.0)       // test hook: scale the reconstruction gradients
            for (int c = 0; c < 2; ++c)
                for (int i = 0; i < n; ++i) {
                    R.gp[c][i] *= g_muscl_grad_scale;
                    R.gu[c][i] *= g_muscl_grad_scale;
                    R.gv[c][i] *= g_muscl_grad_scale;
                }
    }
    sps_stress(P, R);
    riemann_solver(P, R, muscl, g_cfg.solver == SPH_SOLVER_DELTA_SPS);
}

// Shift_particle_position: Taylor_Green_Vortex/Shift_particle_position.f90:56-136,
// using the pair data of the last right-hand side.
void shift_particles(Particles& P, int n_host, const Rhs& R) {
    const PairList& L = R.L;
    const size_t np = L.size();
    const sph_config& C = g_cfg;
    std::vector<double> ti[2], tj[2], acc[2];
    for (int c = 0; c < 2; ++c) { ti[c].resize(np); tj[c].resize(np); resize_zero(acc[c], P.n); }
    const double h2 = C.h * C.h;
    #pragma omp parallel for
    for (size_t k = 0; k < np; ++k) {
        double r = L.w[k] / g_K.w_dx;
        double rn = 1.0;
        for (int s = 0; s < C.shift_n; ++s) rn *= r;
        if (C.shift_n == 4) rn = pw4(r);
        double f = C.shift_beta * h2 * (1 + C.shift_R * rn);
        ti[0][k] = -(f * R.ndwi0[k] * R.vol[L.pj[k]]);
        ti[1][k] = -(f * R.ndwi1[k] * R.vol[L.pj[k]]);
        tj[0][k] = f * R.ndwj0[k] * R.vol[L.pi[k]];
        tj[1][k] = f * R.ndwj1[k] * R.vol[L.pi[k]];
    }
    scatter<2>(P.n, R.I, ti, tj, acc);
    for (int i = 0; i < n_host; ++i) {
        if (P.type[i] != SPH_TYPE_WATER) continue;
        if (R.near[i] == 1) continue;
        double s0 = acc[0][i], s1 = acc[1][i];
        double amp = std::sqrt(s0 * s0 + s1 * s1);
        if (amp > C.shift_max) { s0 = s0 / amp * C.shift_max; s1 = s1 / amp * C.shift_max; }
        P.x[i] = P.x[i] + s0; P.y[i] = P.y[i] + s1;
        P.rho[i] = P.rho[i] + R.grho[0][i] * s0;
        P.rho[i] = P.rho[i] + R.grho[1][i] * s1;
    }
}

// Distribute_Period_Boundary_Particle: Taylor_Green_Vortex/Distribute_Period_Boundary_Particle.f90:56-206.
void periodic_images(const Particles& H, Particles& P) {
    const sph_config& C = g_cfg;
    const double band = C.kernel_scale * C.h;
    const double Lx = C.box_hi[0] - C.box_lo[0], Ly = C.box_hi[1] - C.box_lo[1];
    P = H;
    for (int i = 0; i < H.n; ++i) P.src[i] = -1;
    auto push = [&](int i, double nx, double ny) {
        int m = P.n;
        P.resize(m + 1);
        P.x[m] = nx; P.y[m] = ny; P.u[m] = P.u[i]; P.v[m] = P.v[i];
        P.rho[m] = P.rho[i]; P.mass[m] = P.mass[i]; P.smass[m] = P.smass[i];
        P.type[m] = SPH_TYPE_PERIODIC; P.itype[m] = SPH_TYPE_PERIODIC;
        P.src[m] = (i < H.n) ? i : P.src[i];
    };
    for (int i = 0; i < H.n; ++i) {
        if (H.type[i] == SPH_TYPE_ILL) continue;
        if (P.x[i] <= (C.box_lo[0] + band) && P.x[i] >= C.box_lo[0]) push(i, P.x[i] + Lx, P.y[i]);
        if (P.x[i] >= (C.box_hi[0] - band) && P.x[i] <= C.box_hi[0]) push(i, P.x[i] - Lx, P.y[i]);
    }
    const int nlr = P.n;
    for (int i = 0; i < nlr; ++i) {
        if (P.type[i] == SPH_TYPE_ILL) continue;
        if (P.y[i] <= (C.box_lo[1] + band) && P.y[i] >= C.box_lo[1]) push(i, P.x[i], P.y[i] + Ly);
        if (P.y[i] >= (C.box_hi[1] - band) && P.y[i] <= C.box_hi[1]) push(i, P.x[i], P.y[i] - Ly);
    }
}

void wrap_periodic(Particles& H) {
    const sph_config& C = g_cfg;
    const double Lx = C.box_hi[0] - C.box_lo[0], Ly = C.box_hi[1] - C.box_lo[1];
    for (int i = 0; i < H.n; ++i) {
        if (H.type[i] == SPH_TYPE_ILL) continue;
        if (H.x[i] > C.box_hi[0]) H.x[i] = H.x[i] - Lx;
        else if (H.x[i] < C.box_lo[0]) H.x[i] = H.x[i] + Lx;
        if (H.y[i] > C.box_hi[1]) H.y[i] = H.y[i] - Ly;
        else if (H.y[i] < C.box_lo[1]) H.y[i] = H.y[i] + Ly;
    }
}

// Matrix inverse by Gauss-Jordan elimination with full pivoting, in place,
// the method of BRINV (Taylor_Green_Vortex/function_module.f90:568-639).
// Returns false when the largest remaining pivot is negligible (d + 1 == 1).
bool gauss_jordan_inverse(std::vector<double>& A, int n) {
    std::vector<int> rowp(n), colp(n);
    auto at = [&](int i, int j) -> double& { return A[(size_t)i * n + j]; };
    for (int k = 0; k < n; ++k) {
        double d = 0.0;
        for (int i = k; i < n; ++i)
            for (int j = k; j < n; ++j)
                if (std::fabs(at(i, j)) > d) { d = std::fabs(at(i, j)); rowp[k] = i; colp[k] = j; }
        if (d + 1.0 == 1.0) return false;
        for (int j = 0; j < n; ++j) std::swap(at(k, j), at(rowp[k], j));
        for (int i = 0; i < n; ++i) std::swap(at(i, k), at(i, colp[k]));
        at(k, k) = 1.0 / at(k, k);
        for (int j = 0; j < n; ++j) if (j != k) at(k, j) = at(k, j) * at(k, k);
        for (int i = 0; i < n; ++i)
            if (i != k)
                for (int j = 0; j < n; ++j)
                    if (j != k) at(i, j) = at(i, j) - at(i, k) * at(k, j);
        for (int i = 0; i < n; ++i) if (i != k) at(i, k) = -at(i, k) * at(k, k);
    }
    for (int k = n - 1; k >= 0; --k) {
        for (int j = 0; j < n; ++j) std::swap(at(k, j), at(colp[k], j));
        for (int i = 0; i < n; ++i) std::swap(at(i, k), at(i, rowp[k]));
    }
    return true;
}

// matrix_inversion_less_three, n = 3 (Taylor_Green_Vortex/function_module.f90:157-249):
// the adjugate over the determinant; false when the determinant is zero.
bool inverse3(std::vector<double>& A) {
    auto a = [&](int i, int j) { return A[(size_t)i * 3 + j]; };
    const double det = a(0, 0) * (a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1)) - a(0, 1) * (a(1, 0) * a(2, 2) - a(1, 2) * a(2, 0)) +
                       a(0, 2) * (a(1, 0) * a(2, 1) - a(1, 1) * a(2, 0));
    if (det == 0.0) return false;
    std::vector<double> R(9);
    R[0] = (a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1)) / det;
    R[1] = -(a(0, 1) * a(2, 2) - a(0, 2) * a(2, 1)) / det;
    R[2] = (a(0, 1) * a(1, 2) - a(0, 2) * a(1, 1)) / det;
    R[3] = -(a(1, 0) * a(2, 2) - a(1, 2) * a(2, 0)) / det;
    R[4] = (a(0, 0) * a(2, 2) - a(0, 2) * a(2, 0)) / det;
    R[5] = -(a(0, 0) * a(1, 2) - a(0, 2) * a(1, 0)) / det;
    R[6] = (a(1, 0) * a(2, 1) - a(1, 1) * a(2, 0)) / det;
    R[7] = -(a(0, 0) * a(2, 1) - a(0, 1) * a(2, 0)) / det;
    R[8] = (a(0, 0) * a(1, 1) - a(0, 1) * a(1, 0)) / det;
    A = R;
    return true;
}

// Reinitialize_particle_density (Taylor_Green_Vortex/Reinitialize_particle_density.f90:98-181,
// MLS_Interpolation_In_Subdomain_Domain.f90:96-285; the moving-square variant
// Moving_Square.../Reinitialize_particle_density.f90:92-200 includes the particle
// itself, weights the kernel by the neighbour volume, has no order-6 fallback and
// keeps the old density on NaN).  Candidates: the 3x3 background cells in stencil
// order (the effect list of Assign_boundary_particles), on the current positions.
void mls_reinit(Particles& P, int n_host) {
    const int m = g_cfg.mls_order;
    const bool ms = ms_solver();
    const double hb = (g_cfg.h + g_cfg.h) / 2.0;
    const double alpha = g_cfg.mls_alpha;
    Grid G;
    build_grid(P, G);
    const std::vector<double> rho_old = P.rho;
    std::vector<double> rho_new(n_host);
    #pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n_host; ++i) {
        rho_new[i] = rho_old[i];
        if (P.type[i] != SPH_TYPE_WATER) continue;
        std::vector<int> nb;
        std::vector<double> W;
        const int ci = G.cell[i];
        const int cx = ci % G.nx, cy = ci / G.nx;
        for (int s = 0; s < 9; ++s) {
            const int gx = cx + kStencil[s][0], gy = cy + kStencil[s][1];
            if (gx < 0 || gy < 0 || gx >= G.nx || gy >= G.ny) continue;
            const int c = gy * G.nx + gx;
            for (int t = G.start[c]; t < G.start[c + 1]; ++t) {
                const int j = G.items[t];
                double pd[2] = {P.x[i] - P.x[j], P.y[i] - P.y[j]};
                const double d = std::sqrt(pd[0] * pd[0] + pd[1] * pd[1]);
                if (!(d <= g_cfg.kernel_scale * hb)) continue;
                if (!ms && !(d >= g_K.cut_min)) continue;
                double w, dw[2];
                kernel(d, pd, hb, w, dw);
                if (ms) w = w * (P.mass[j] / rho_old[j]);
                nb.push_back(j);
                W.push_back(w);
            }
        }
        const int k = (int)nb.size();
        std::vector<double> fai(k);
        double sw = 0.0;
        for (int q = 0; q < k; ++q) sw += W[q];
        bool shepard = false;
        // P (m x k), augmented by alpha I with weights alpha (:155-172)
        std::vector<double> Pm((size_t)m * (k + m), 0.0), Wd(k + m, 0.0);
        for (int q = 0; q < k; ++q) {
            const int j = nb[q];
            const double dx = (P.x[j] - P.x[i]) / g_cfg.h, dy = (P.y[j] - P.y[i]) / g_cfg.h;
            double pv[6] = {1.0, dx, dy, dx * dx, dx * dy, dy * dy};
            for (int r = 0; r < m; ++r) Pm[(size_t)r * (k + m) + q] = pv[r];
            Wd[q] = W[q];
        }
        for (int L = 0; L < m; ++L) { Pm[(size_t)L * (k + m) + k + L] = alpha; Wd[k + L] = alpha; }
        // B = P W, A = B P^T (:176-180)
        std::vector<double> B((size_t)m * (k + m)), A((size_t)m * m, 0.0);
        for (int r = 0; r < m; ++r)
            for (int q = 0; q < k + m; ++q) B[(size_t)r * (k + m) + q] = Pm[(size_t)r * (k + m) + q] * Wd[q];
        for (int r = 0; r < m; ++r)
            for (int c = 0; c < m; ++c) {
                double a = 0.0;
                for (int q = 0; q < k + m; ++q) a += B[(size_t)r * (k + m) + q] * Pm[(size_t)c * (k + m) + q];
                A[(size_t)r * m + c] = a;
            }
        const bool ok = m == 6 ? gauss_jordan_inverse(A, 6) : inverse3(A);
        if (!ok) shepard = true;
        if (!ms && m == 6 && k <= 8) shepard = true;
        double rho = 0.0;
        for (int q = 0; q < k; ++q) {
            double f;
            if (shepard) f = W[q] / sw;
            else {   // Fai = row 1 of A^-1 B  (P_i = e_1)
                f = 0.0;
                for (int r = 0; r < m; ++r) f += A[(size_t)0 * m + r] * B[(size_t)r * (k + m) + q];
            }
            rho += rho_old[nb[q]] * f;
        }
        if (ms && std::isnan(rho)) rho = rho_old[i];
        rho_new[i] = rho;
    }
    for (int i = 0; i < n_host; ++i) P.rho[i] = rho_new[i];
}

// RefreshDensity_MLS_Order = 1 (Taylor_Green_Vortex/Reinitialize_particle_density.f90:71-92,
// Moving_Square.../Reinitialize_particle_density.f90:66-88) on the pair list and
// volumes of the step's last RHS: for pairs of particles of the same type,
// rho_i += m_j w_ij / sum_w(i) for water particles, sum_w(i) = sum_j w_ij V_j over
// the same pairs (Define_freesurface_and_Normailized_derivates.f90:87-91).  Other
// particles keep their density.
void mls_order1(Particles& P, int n_host, const Rhs& R) {
    const PairList& L = R.L;
    std::vector<double> sw(P.n, 0.0), rho(P.n, 0.0);
    for (size_t k = 0; k < L.size(); ++k) {
        const int i = L.pi[k], j = L.pj[k];
        if (P.type[i] != P.type[j]) continue;
        sw[i] += L.w[k] * R.vol[j];
        sw[j] += L.w[k] * R.vol[i];
    }
    for (size_t k = 0; k < L.size(); ++k) {
        const int i = L.pi[k], j = L.pj[k];
        if (P.type[i] != P.type[j]) continue;
        if (P.type[i] == SPH_TYPE_WATER) rho[i] += P.mass[j] * L.w[k] / sw[i];
        if (P.type[j] == SPH_TYPE_WATER) rho[j] += P.mass[i] * L.w[k] / sw[j];
    }
    for (int i = 0; i < n_host; ++i)
        if (P.type[i] == SPH_TYPE_WATER) P.rho[i] = rho[i];
}

void reinit_density(Particles& P, int n_host, const Rhs& R) {
    if (g_cfg.mls_order == 1) mls_order1(P, n_host, R);
    else mls_reinit(P, n_host);
}

struct Sim {
    sph_config cfg;
    Particles H;                      // host particles
    std::vector<double> rdrho, racc0, racc1, ravg0, ravg1;  // last rates, carried per particle
    long long step = 0;               // completed steps
    Rhs last;
    int last_images = 0;
    double bf[6] = {0, 0, 0, 0, 0, 0};   // body force of the last RHS
};

// Euler predictor-corrector of Moving_Square.../SPH_Time_Iteration.f90:304-334
// (Iteration_Method 2): one RHS per step after the first, rates of the last RHS
// reused for the predictor.
// Real_time = Real_time + dt and Body_Motion_Solver at the start of a step
// (MS SPH_Time_Iteration.f90:71-114): the body moves with Custom_velocity.
void advance_time_and_body(Sim& S, double dt) {
    g_time += dt;
    g_n_host = S.H.n;
    if (!g_cfg.ghost_assign) return;
    for (int i = 0; i < S.H.n; ++i)
        if (S.H.itype[i] == SPH_TYPE_BODY) { S.H.x[i] += g_bvel[0] * dt; S.H.y[i] += g_bvel[1] * dt; }
}

void run_step_euler_pc(Sim& S, double dt) {
    const int n = S.H.n;
    advance_time_and_body(S, dt);
    if (g_cfg.periodic) wrap_periodic(S.H);
    Particles P;
    if (g_cfg.periodic) periodic_images(S.H, P);
    else { P = S.H; for (int i = 0; i < n; ++i) P.src[i] = -1; }
    S.last_images = P.n - n;
    const Particles B0 = P;
    Rhs R;
    if (S.step == 0) {
        single_step_compute(P, R);
    } else {
        R.drho.assign(P.n, 0.0);
        for (int a = 0; a < 2; ++a) { R.acc[a].assign(P.n, 0.0); R.avg[a].assign(P.n, 0.0); }
        for (int i = 0; i < n; ++i) {
            R.drho[i] = S.rdrho[i]; R.acc[0][i] = S.racc0[i]; R.acc[1][i] = S.racc1[i];
            R.avg[0][i] = S.ravg0[i]; R.avg[1][i] = S.ravg1[i];
        }
    }
    std::vector<double> td(n), ta0(n), ta1(n), tv0(n), tv1(n);
    for (int i = 0; i < n; ++i) { td[i] = R.drho[i]; ta0[i] = R.acc[0][i]; ta1[i] = R.acc[1][i]; tv0[i] = P.u[i]; tv1[i] = P.v[i]; }
    for (int i = 0; i < n; ++i) {
        if (!integrated(P.type[i])) continue;
        P.rho[i] = B0.rho[i] + R.drho[i] * dt;
        P.x[i] = B0.x[i] + dt * (P.u[i] + R.avg[0][i]) + 0.5 * R.acc[0][i] * (dt * dt);
        P.y[i] = B0.y[i] + dt * (P.v[i] + R.avg[1][i]) + 0.5 * R.acc[1][i] * (dt * dt);
        P.u[i] = B0.u[i] + dt * R.acc[0][i];
        P.v[i] = B0.v[i] + dt * R.acc[1][i];
    }
    single_step_compute(P, R);
    if (g_cfg.solver == SPH_SOLVER_MS_MODLR_DELTA || g_cfg.solver == SPH_SOLVER_MS_HLLC_DELTA) body_force(P, R, S.bf);
    for (int i = 0; i < n; ++i) {
        if (!integrated(P.type[i])) continue;
        P.rho[i] = B0.rho[i] + 0.5 * (R.drho[i] + td[i]) * dt;
        P.x[i] = B0.x[i] + 0.5 * dt * (P.u[i] + tv0[i]) + R.avg[0][i] * dt + 0.5 * R.acc[0][i] * (dt * dt);
        P.y[i] = B0.y[i] + 0.5 * dt * (P.v[i] + tv1[i]) + R.avg[1][i] * dt + 0.5 * R.acc[1][i] * (dt * dt);
        P.u[i] = B0.u[i] + 0.5 * dt * (R.acc[0][i] + ta0[i]);
        P.v[i] = B0.v[i] + 0.5 * dt * (R.acc[1][i] + ta1[i]);
    }
    S.rdrho.assign(R.drho.begin(), R.drho.begin() + n);
    S.racc0.assign(R.acc[0].begin(), R.acc[0].begin() + n);
    S.racc1.assign(R.acc[1].begin(), R.acc[1].begin() + n);
    S.ravg0.assign(R.avg[0].begin(), R.avg[0].begin() + n);
    S.ravg1.assign(R.avg[1].begin(), R.avg[1].begin() + n);
    if (g_cfg.mls_order && (S.step + 1) % g_cfg.mls_every == 0) reinit_density(P, n, R);
    if (g_cfg.shifting) shift_particles(P, n, R);
    for (int i = 0; i < n; ++i) {
        S.H.x[i] = P.x[i]; S.H.y[i] = P.y[i]; S.H.u[i] = P.u[i]; S.H.v[i] = P.v[i]; S.H.rho[i] = P.rho[i];
    }
    S.last = std::move(R);
    S.step++;
}

// One time step of time_iteration.f90:781-1073 (Runge-Kutta branch): stage
// updates :942-1047, then Shift_particle_position with the last RHS pair data.
void run_step(Sim& S, double dt) {
    const int n = S.H.n;
    advance_time_and_body(S, dt);
    if (g_cfg.periodic) wrap_periodic(S.H);
    Particles P;
    if (g_cfg.periodic) periodic_images(S.H, P);
    else { P = S.H; for (int i = 0; i < n; ++i) P.src[i] = -1; }
    S.last_images = P.n - n;
    const Particles B0 = P;
    Rhs R;
    std::vector<double> K1r(n), K1a0(n), K1a1(n), K1v0(n), K1v1(n);
    std::vector<double> K2r(n), K2a0(n), K2a1(n), K2v0(n), K2v1(n);
    std::vector<double> K3r(n), K3a0(n), K3a1(n), K3v0(n), K3v1(n);
    auto save = [&](std::vector<double>& kr, std::vector<double>& ka0, std::vector<double>& ka1,
                    std::vector<double>& kv0, std::vector<double>& kv1, const std::vector<double>& dr,
                    const std::vector<double>& a0, const std::vector<double>& a1) {
        for (int i = 0; i < n; ++i) { kr[i] = dr[i]; ka0[i] = a0[i]; ka1[i] = a1[i]; kv0[i] = P.u[i]; kv1[i] = P.v[i]; }
    };
    // stage 1: from a fresh RHS in the first step, from the carried rates afterwards
    if (S.step == 0) {
        single_step_compute(P, R);
    } else {
        R.drho.assign(P.n, 0.0);
        for (int a = 0; a < 2; ++a) { R.acc[a].assign(P.n, 0.0); R.avg[a].assign(P.n, 0.0); }
        for (int i = 0; i < n; ++i) {
            R.drho[i] = S.rdrho[i]; R.acc[0][i] = S.racc0[i]; R.acc[1][i] = S.racc1[i];
            R.avg[0][i] = S.ravg0[i]; R.avg[1][i] = S.ravg1[i];
        }
    }
    {
        // the half step uses drhodt*dt/2 and 0.5*dt*a (equal in value)
        for (int i = 0; i < n; ++i) {
            if (P.type[i] != SPH_TYPE_WATER) continue;
            P.rho[i] = B0.rho[i] + R.drho[i] * dt / 2;
            P.u[i] = B0.u[i] + 0.5 * dt * R.acc[0][i] + R.avg[0][i];
            P.x[i] = B0.x[i] + 0.5 * dt * P.u[i];
            P.v[i] = B0.v[i] + 0.5 * dt * R.acc[1][i] + R.avg[1][i];
            P.y[i] = B0.y[i] + 0.5 * dt * P.v[i];
        }
        save(K1r, K1a0, K1a1, K1v0, K1v1, R.drho, R.acc[0], R.acc[1]);
    }
    single_step_compute(P, R);
    for (int i = 0; i < n; ++i) {
        if (P.type[i] != SPH_TYPE_WATER) continue;
        P.rho[i] = B0.rho[i] + R.drho[i] * dt / 2;
        P.u[i] = B0.u[i] + 0.5 * dt * R.acc[0][i] + R.avg[0][i];
        P.x[i] = B0.x[i] + 0.5 * dt * P.u[i];
        P.v[i] = B0.v[i] + 0.5 * dt * R.acc[1][i] + R.avg[1][i];
        P.y[i] = B0.y[i] + 0.5 * dt * P.v[i];
    }
    save(K2r, K2a0, K2a1, K2v0, K2v1, R.drho, R.acc[0], R.acc[1]);
    single_step_compute(P, R);
    for (int i = 0; i < n; ++i) {
        if (P.type[i] != SPH_TYPE_WATER) continue;
        P.rho[i] = B0.rho[i] + R.drho[i] * dt;
        P.u[i] = B0.u[i] + dt * R.acc[0][i] + R.avg[0][i];
        P.x[i] = B0.x[i] + dt * P.u[i];
        P.v[i] = B0.v[i] + dt * R.acc[1][i] + R.avg[1][i];
        P.y[i] = B0.y[i] + dt * P.v[i];
    }
    save(K3r, K3a0, K3a1, K3v0, K3v1, R.drho, R.acc[0], R.acc[1]);
    single_step_compute(P, R);
    if (ms_solver()) body_force(P, R, S.bf);
    for (int i = 0; i < n; ++i) {
        if (P.type[i] != SPH_TYPE_WATER) continue;
        P.rho[i] = B0.rho[i] + (K1r[i] + 2 * K2r[i] + 2 * K3r[i] + R.drho[i]) * dt / 6.0;
        P.u[i] = B0.u[i] + (K1a0[i] + 2 * K2a0[i] + 2 * K3a0[i] + R.acc[0][i]) * dt / 6.0 + R.avg[0][i];
        P.x[i] = B0.x[i] + (K1v0[i] + 2 * K2v0[i] + 2 * K3v0[i] + P.u[i]) * dt / 6.0 + 0.5 * dt * dt * R.acc[0][i];
        P.v[i] = B0.v[i] + (K1a1[i] + 2 * K2a1[i] + 2 * K3a1[i] + R.acc[1][i]) * dt / 6.0 + R.avg[1][i];
        P.y[i] = B0.y[i] + (K1v1[i] + 2 * K2v1[i] + 2 * K3v1[i] + P.v[i]) * dt / 6.0 + 0.5 * dt * dt * R.acc[1][i];
    }
    // carry this step's last rates as next step's K1 (per particle)
    S.rdrho.assign(R.drho.begin(), R.drho.begin() + n);
    S.racc0.assign(R.acc[0].begin(), R.acc[0].begin() + n);
    S.racc1.assign(R.acc[1].begin(), R.acc[1].begin() + n);
    S.ravg0.assign(R.avg[0].begin(), R.avg[0].begin() + n);
    S.ravg1.assign(R.avg[1].begin(), R.avg[1].begin() + n);
    // Reinitialize_particle_density every MLS_time_step steps, before shifting (:673-682)
    if (g_cfg.mls_order && (S.step + 1) % g_cfg.mls_every == 0) reinit_density(P, n, R);
    if (g_cfg.shifting) shift_particles(P, n, R);
    // copy the host particles back (images are discarded)
    for (int i = 0; i < n; ++i) {
        S.H.x[i] = P.x[i]; S.H.y[i] = P.y[i]; S.H.u[i] = P.u[i]; S.H.v[i] = P.v[i]; S.H.rho[i] = P.rho[i];
    }
    S.last = std::move(R);
    S.step++;
}

Particles make_particles(int n, const double* pos, const double* vel, const double* rho, const double* mass,
                         const int* type, const double* smass) {
    Particles H;
    H.resize(n);
    for (int i = 0; i < n; ++i) {
        H.x[i] = pos[i]; H.y[i] = pos[n + i];
        H.u[i] = vel[i]; H.v[i] = vel[n + i];
        H.rho[i] = rho[i]; H.mass[i] = mass[i];
        H.smass[i] = smass ? smass[i] : mass[i];
        H.type[i] = type[i]; H.itype[i] = type[i]; H.src[i] = -1;
    }
    return H;
}

}  // namespace

// ===========================================================================
// C interface used by the tests (ctypes).  All arrays are column-major (n,2)
// like the Fortran module arrays.
// ===========================================================================
extern "C" {

// Reinitialize_particle_density alone on the given particles (no images):
// rho_out = the re-initialised densities of the n particles.
int oracle_mls_reinit(const sph_config* cfg, int n, const double* pos, const double* rho, const double* mass,
                      const int* type, double* rho_out) {
    if (!cfg || n <= 0 || !(cfg->mls_order == 3 || cfg->mls_order == 6)) return -1;
    g_cfg = *cfg;
    derive_consts(*cfg);
    std::vector<double> zero(2 * (size_t)n, 0.0);
    Particles P = make_particles(n, pos, zero.data(), rho, mass, type, nullptr);
    mls_reinit(P, n);
    for (int i = 0; i < n; ++i) rho_out[i] = P.rho[i];
    return 0;
}

// Inputs of the ghost assignment for the following oracle calls.
void oracle_set_ghost_state(int n, const int* labels, const double* bvel, const double* bacc, double t) {
    g_labels.assign(labels ? labels : nullptr, labels ? labels + n : nullptr);
    if (!labels) g_labels.assign(n, 0);
    for (int k = 0; k < 2; ++k) { g_bvel[k] = bvel ? bvel[k] : 0.0; g_bacc[k] = bacc ? bacc[k] : 0.0; }
    g_time = t;
    g_n_host = n;
}

// Test hooks for the pins of the MUSCL and HLLC paths (tests/test_oracle_pins.py).
void oracle_set_muscl_gradient_scale(double s) { g_muscl_grad_scale = s; }

void oracle_muscl_limiter(double di, double dj, double dij, double* li, double* lj) {
    muscl_limiter(di, dj, dij, *li, *lj);
}

// The HLLC pair state for one pair: in[0..1] v_i, in[2..3] v_j, in[4..5] the unit
// vector from i to j, in[6..11] rho_i, rho_j, c_i, c_j, p_i, p_j; out[0..1] v*, out[2] P*.
// The configuration supplies c0^2, rho0 and the background pressure.
int oracle_hllc_state(const sph_config* cfg, const double* in, double* out) {
    if (!cfg || !in || !out) return -1;
    g_cfg = *cfg;
    derive_consts(*cfg);
    const double vI[2] = {in[0], in[1]}, vJ[2] = {in[2], in[3]}, e[2] = {in[4], in[5]};
    const double vbar[2] = {(vI[0] + vJ[0]) / 2.0, (vI[1] + vJ[1]) / 2.0};
    double vs[2], Ps;
    hllc_state(vI, vJ, vbar, e, in[6], in[7], in[8], in[9], in[10], in[11], vs, Ps);
    out[0] = vs[0]; out[1] = vs[1]; out[2] = Ps;
    return 0;
}

int oracle_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
    return omp_get_max_threads();
#else
    (void)nthreads;
    return 1;
#endif
}

// Taylor-Green lattice, Taylor_Green_Vortex/Distribute_Initial_Particle.f90:206-231.
// sign = +1: the reference field (u = U sin cos, p = +rho0 U^2/4 (...));
// sign = -1: the quarter-period shifted field (u = -U cos sin, p = -rho0 U^2/4 (...)).
// exponent: the inverse-Tait exponent (0.142857142 as a default real in the reference).
int oracle_tgv_init(int nx, int ny, double lx, double ly, double U, double rho0, double c0sq, int sign,
                    int reference_literals, double* pos, double* vel, double* rho, double* mass, double* press) {
    const double PI = 3.14159265358979324;
    const double dx = lx / nx, dy = ly / ny;
    const int n = nx * ny;
    const double ex = reference_literals ? (double)0.142857142f : 1.0 / 7.0;
    int k = 0;
    for (int i = 1; i <= ny; ++i)
        for (int j = 1; j <= nx; ++j) {
            double x = (j - 1) * dx + dx / 2.0;
            double y = (i - 1) * dy + dy / 2.0;
            double u, v, p;
            if (sign > 0) {
                u = U * std::sin(2 * PI * x) * std::cos(2 * PI * y);
                v = -U * std::cos(2 * PI * x) * std::sin(2 * PI * y);
                p = 0.25 * rho0 * (U * U) * (std::cos(4 * PI * x) + std::cos(4 * PI * y));
            } else {
                u = -U * std::cos(2 * PI * x) * std::sin(2 * PI * y);
                v = U * std::sin(2 * PI * x) * std::cos(2 * PI * y);
                p = -0.25 * rho0 * (U * U) * (std::cos(4 * PI * x) + std::cos(4 * PI * y));
            }
            double r = rho0 * std::pow(1 + 7 * p / (c0sq * rho0), ex);
            pos[k] = x; pos[n + k] = y; vel[k] = u; vel[n + k] = v;
            rho[k] = r; mass[k] = dx * dy * r;
            if (press) press[k] = p;
            ++k;
        }
    return 0;
}

// Pair list of the current particles (no periodic images added here).
long long oracle_find_particle_pair(const sph_config* cfg, int n, const double* pos, const int* type,
                                    long long pair_cap, int* pair_i, int* pair_j, double* w, double* dwdx) {
    g_cfg = *cfg;
    derive_consts(*cfg);
    Particles P;
    P.resize(n);
    for (int i = 0; i < n; ++i) { P.x[i] = pos[i]; P.y[i] = pos[n + i]; P.type[i] = type[i]; }
    Grid G;
    build_grid(P, G);
    PairList L;
    find_pairs(P, G, L);
    long long np = (long long)L.size();
    for (long long k = 0; k < np && k < pair_cap; ++k) {
        pair_i[k] = L.pi[k] + 1; pair_j[k] = L.pj[k] + 1;
        if (w) w[k] = L.w[k];
        if (dwdx) { dwdx[k] = L.dw0[k]; dwdx[pair_cap + k] = L.dw1[k]; }
    }
    return np;
}

// Periodic images appended after the n host particles; returns the new count
// (or -1 if it would exceed cap).  Arrays are sized cap.
int oracle_periodic_images(const sph_config* cfg, int n, int cap, double* pos, double* vel, double* rho,
                           double* mass, int* type, int* src) {
    g_cfg = *cfg;
    derive_consts(*cfg);
    Particles H;
    H.resize(n);
    for (int i = 0; i < n; ++i) {
        H.x[i] = pos[i]; H.y[i] = pos[cap + i]; H.u[i] = vel[i]; H.v[i] = vel[cap + i];
        H.rho[i] = rho[i]; H.mass[i] = mass[i]; H.smass[i] = mass[i]; H.type[i] = type[i];
    }
    Particles P;
    periodic_images(H, P);
    if (P.n > cap) return -1;
    for (int i = 0; i < P.n; ++i) {
        pos[i] = P.x[i]; pos[cap + i] = P.y[i]; vel[i] = P.u[i]; vel[cap + i] = P.v[i];
        rho[i] = P.rho[i]; mass[i] = P.mass[i]; type[i] = P.type[i];
        if (src) src[i] = P.src[i];
    }
    return P.n;
}

// One single_step_compute on exactly the given particles.  Outputs are [n]
// or [2n] (column-major) and may be NULL; binv is [4n] (B11,B12,B21,B22 blocks),
// tau [3n] (xx,xy,yy), grads [8n] (rho x,y, p x,y, u x,y, v x,y).
long long oracle_rhs(const sph_config* cfg, int n, const double* pos, const double* vel, const double* rho,
                     const double* mass, const int* type, const double* smass, double* drhodt, double* acc,
                     double* avg, int* fs, int* near_fs, double* fra_v, double* binv, double* tau,
                     double* grads) {
    g_cfg = *cfg;
    derive_consts(*cfg);
    Particles P = make_particles(n, pos, vel, rho, mass, type, smass);
    Rhs R;
    single_step_compute(P, R);
    for (int i = 0; i < n; ++i) {
        if (drhodt) drhodt[i] = R.drho[i];
        if (acc) { acc[i] = R.acc[0][i]; acc[n + i] = R.acc[1][i]; }
        if (avg) { avg[i] = R.avg[0][i]; avg[n + i] = R.avg[1][i]; }
        if (fs) fs[i] = R.fs[i];
        if (near_fs) near_fs[i] = R.near[i];
        if (fra_v) fra_v[i] = R.fra_v[i];
        if (binv) for (int c = 0; c < 4; ++c) binv[c * n + i] = R.binv[c][i];
        if (tau) for (int c = 0; c < 3; ++c) tau[c * n + i] = R.tau[c][i];
        if (grads) {
            grads[i] = R.grho[0][i]; grads[n + i] = R.grho[1][i];
            bool m = !R.gp[0].empty();
            grads[2 * n + i] = m ? R.gp[0][i] : 0.0; grads[3 * n + i] = m ? R.gp[1][i] : 0.0;
            grads[4 * n + i] = m ? R.gu[0][i] : 0.0; grads[5 * n + i] = m ? R.gu[1][i] : 0.0;
            grads[6 * n + i] = m ? R.gv[0][i] : 0.0; grads[7 * n + i] = m ? R.gv[1][i] : 0.0;
        }
    }
    return (long long)R.L.size();
}

void* oracle_create(const sph_config* cfg, int n, const double* pos, const double* vel, const double* rho,
                    const double* mass, const int* type, const double* smass) {
    Sim* S = new Sim();
    S->cfg = *cfg;
    S->H = make_particles(n, pos, vel, rho, mass, type, smass);
    return S;
}

int oracle_run(void* h, int nsteps, double dt) {
    Sim* S = (Sim*)h;
    g_cfg = S->cfg;
    derive_consts(S->cfg);
    for (int s = 0; s < nsteps; ++s) {
        if (S->cfg.integrator == SPH_INTEGRATOR_EULER_PC) run_step_euler_pc(*S, dt);
        else run_step(*S, dt);
    }
    return 0;
}

int oracle_set_initial_type(void* h, int n, const int* itype) {
    Sim* S = (Sim*)h;
    if (n != S->H.n) return -1;
    for (int i = 0; i < n; ++i) S->H.itype[i] = itype[i];
    return 0;
}

void oracle_body_force(void* h, double* out) {
    Sim* S = (Sim*)h;
    for (int c = 0; c < 6; ++c) out[c] = S->bf[c];
}

// Body force of one RHS on exactly the given particles (itype: initial types).
int oracle_rhs_body_force(const sph_config* cfg, int n, const double* pos, const double* vel, const double* rho,
                          const double* mass, const int* type, const int* itype, double* out) {
    g_cfg = *cfg;
    derive_consts(*cfg);
    Particles P = make_particles(n, pos, vel, rho, mass, type, nullptr);
    for (int i = 0; i < n; ++i) P.itype[i] = itype[i];
    Rhs R;
    single_step_compute(P, R);
    body_force(P, R, out);
    return 0;
}

int oracle_get_state(void* h, int n, double* pos, double* vel, double* rho, double* press) {
    Sim* S = (Sim*)h;
    if (n != S->H.n) return -1;
    g_cfg = S->cfg;
    derive_consts(S->cfg);
    for (int i = 0; i < n; ++i) {
        if (pos) { pos[i] = S->H.x[i]; pos[n + i] = S->H.y[i]; }
        if (vel) { vel[i] = S->H.u[i]; vel[n + i] = S->H.v[i]; }
        if (rho) rho[i] = S->H.rho[i];
        if (press) { double p, c; eos(S->H.rho[i], p, c); press[i] = p; }
    }
    return 0;
}

double oracle_kinetic_energy(void* h) {
    Sim* S = (Sim*)h;
    double ke = 0.0;
    for (int i = 0; i < S->H.n; ++i) {
        if (S->H.type[i] != SPH_TYPE_WATER) continue;
        ke = ke + 0.5 * S->H.mass[i] * (S->H.u[i] * S->H.u[i] + S->H.v[i] * S->H.v[i]);
    }
    return ke;
}

long long oracle_last_pair_count(void* h) { return (long long)((Sim*)h)->last.L.size(); }
int oracle_last_images(void* h) { return ((Sim*)h)->last_images; }

void oracle_destroy(void* h) { delete (Sim*)h; }

}  // extern "C"
