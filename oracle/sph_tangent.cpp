// sph_tangent.cpp -- FP64 tangent-linear model of the Taylor-Green time step.
//
// TEST INFRASTRUCTURE ONLY: the CPU reference the GPU adjoint
// (sph_adjoint_forward / sph_adjoint_backward) is checked against.  Never
// linked into, loaded by or called from the product path.
//
// The step is written once, templated on the scalar type: with double it is a
// second restatement of the oracle's Taylor-Green step (the pair loops of
// Solver_Normalized_Modified_Linear_Riemann_Delta_SPS.f90:126-583 and the
// Runge-Kutta stages of time_iteration.f90:781-1073, with the particle shift
// of Shift_particle_position.f90:56-136 when on, in the oracle's pair
// orientation and term order), pinned against sph_oracle.cpp by the tests;
// with Dual (value + one directional derivative, forward-mode differentiation)
// it returns the loss and its derivative along a chosen direction of the
// initial position, velocity, density and viscosity: the tangent-linear model.
// Branches (support test, max/min of the Riemann dissipation, the artificial-
// viscosity switch, periodic wrap and images) are taken on the values, so the
// derivative is that of the taken branch with the pair set held fixed, which
// is what the adjoint differentiates too.
//
// Scope: (1) Taylor-Green: the modified linear Riemann and the MUSCL linear
// Riemann delta-SPH + SPS solvers, RK4 with the K1 reuse, periodic images
// (oracle_tangent); (2) moving square:
// the modified linear Riemann and the HLLC solvers with XSPH in the continuity flux, the
// fixed-ghost assignment, the body force and the Euler predictor-corrector with
// a per-step body motion (oracle_tangent_ms).  Either kernel, with or without
// renormalisation, with or without shifting (the capped shift on the last
// RHS's pairs, exponent 4 in (2)), density re-initialisation (orders 1, 3, 6),
// no free-surface particles.  Other inputs return SPH_E_CONFIG.
// The pair search is a plain double loop (small cases only).

#include <cmath>
#include <cstring>
#include <vector>

#include "../include/sph_b200.h"

namespace {

struct Dual {
    double v, d;
    Dual(double a = 0.0, double b = 0.0) : v(a), d(b) {}
};
inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
inline Dual operator-(Dual a) { return {-a.v, -a.d}; }
inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
inline Dual operator/(Dual a, Dual b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
inline Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
inline Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
inline Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
inline Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
inline Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
inline Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
inline Dual operator/(Dual a, double b) { return {a.v / b, a.d / b}; }
inline Dual operator/(double a, Dual b) { return {a / b.v, -a * b.d / (b.v * b.v)}; }
inline Dual& operator+=(Dual& a, Dual b) { a = a + b; return a; }
inline Dual& operator-=(Dual& a, Dual b) { a = a - b; return a; }
inline Dual sqrt(Dual a) { double s = std::sqrt(a.v); return {s, s > 0.0 ? a.d / (2.0 * s) : 0.0}; }
inline Dual exp(Dual a) { double e = std::exp(a.v); return {e, e * a.d}; }
inline double val(double a) { return a; }
inline double val(const Dual& a) { return a.v; }
using std::exp;
using std::sqrt;

// Constants of the configuration (the same derivation as the oracle's).
struct TConsts {
    double pi_k, pi, e9, den, cut_min, fs_thr, dl, c012, c23, cblin, sqrt_c0, eos_b, sv, q_zero;
    double w_dx;      // kernel value at distance dx (Shift_particle_position.f90:56-68)
};

TConsts derive(const sph_config& c) {
    TConsts K;
    const bool q = c.reference_literals != 0;
    K.pi = 3.14159265358979324;
    K.pi_k = q ? (double)3.14159265358f : K.pi;
    if (q) {
        float e9 = std::exp(-9.0f);
        K.e9 = (double)e9;
        K.den = (double)(1.0f - 10.0f * e9);
        K.cut_min = (double)1.0e-7f;
        K.fs_thr = (double)(float)c.fs_threshold;
        K.dl = (double)(std::sqrt(2.0f) / 2.0f);
        K.c012 = (double)0.12f;
        K.c23 = (double)(2.0f / 3.0f);
        K.cblin = (double)((2.0f / 3.0f) * 0.0066f);
        K.q_zero = (double)1.0e-8f;
    } else {
        K.e9 = std::exp(-9.0);
        K.den = 1.0 - 10.0 * K.e9;
        K.cut_min = 1.0e-7;
        K.fs_thr = c.fs_threshold;
        K.dl = std::sqrt(2.0) / 2.0;
        K.c012 = 0.12;
        K.c23 = 2.0 / 3.0;
        K.cblin = 2.0 / 3.0 * 0.0066;
        K.q_zero = 1.0e-8;
    }
    K.sqrt_c0 = std::sqrt(c.c0sq);
    K.eos_b = c.c0sq * c.rho0 / 7.0;
    const double sr = c.kernel_scale * c.h;
    K.sv = K.pi * (sr * sr);
    {
        const double h = c.h, q = c.dx / h;
        if (c.kernel_model == SPH_KERNEL_GAUSSIAN) {
            const double factor = 1.0 / (K.pi_k * (h * h) * K.den);
            K.w_dx = c.dx <= 3.0 * h ? (std::exp(-(q * q)) - K.e9) * factor : 0.0;
        } else {
            const double factor = 7.0 / (4 * K.pi_k * (h * h));
            const double t = 1.0 - q / 2.0, t2 = t * t;
            K.w_dx = c.dx <= 2.0 * h ? factor * (1.0 + 2.0 * q) * (t2 * t2) : 0.0;
        }
    }
    return K;
}

// MUSCL_Limiter (Taylor_Green_Vortex/function_module.f90:34-80), branches taken on
// the values, with std::min / std::max's choice of operand on ties.
template <class T>
inline T tmin(const T& a, const T& b) { return val(b) < val(a) ? b : a; }
template <class T>
inline T tmax(const T& a, const T& b) { return val(a) < val(b) ? b : a; }
template <class T>
void muscl_limiter_t(const T& di, const T& dj, const T& dij, T& li, T& lj) {
    const double beta_lim = 1.3, diff = 0.5;
    if (val(dj) > 0.0) {
        const T lim = tmax(T(0.0), tmax(tmin(beta_lim * di, dj), tmin(di, beta_lim * dj)));
        if (val(lim) > 0.5 * val(dij) && std::fabs(val(lim)) > 0.0) {
            const bool first = val(di) > val(dj);
            li = dij * (first ? diff : 0.0); lj = dij * (first ? 0.0 : diff);
        } else { li = lim; lj = lim; }
    } else {
        const T lim = tmin(T(0.0), tmin(tmax(beta_lim * di, dj), tmax(di, beta_lim * dj)));
        if (val(lim) < 0.5 * val(dij) && std::fabs(val(lim)) > 0.0) {
            const bool first = val(di) < val(dj);
            li = dij * (first ? diff : 0.0); lj = dij * (first ? 0.0 : diff);
        } else { li = lim; lj = lim; }
    }
}

// All particles of one step (hosts, then periodic images).
template <class T>
struct Parts {
    std::vector<T> x, y, u, v, rho;
    std::vector<double> mass, smass;
    std::vector<int> type;
    int n = 0;
    void push(const T& x_, const T& y_, const T& u_, const T& v_, const T& r_, double m, double sm, int t) {
        x.push_back(x_); y.push_back(y_); u.push_back(u_); v.push_back(v_); rho.push_back(r_);
        mass.push_back(m); smass.push_back(sm); type.push_back(t);
        ++n;
    }
};

template <class T>
struct Model {
    sph_config C;
    TConsts K;
    T nu;

    // compute_kernel (Taylor_Green_Vortex/compute_kernel.f90:120-142; Wendland C2 of
    // Moving_Square.../Compute_Kernel.f90:179-193)
    void kernel(const T& d, const T& p0, const T& p1, double h, T& w, T& g0, T& g1) const {
        const T q = d / h;
        w = T(0.0); g0 = T(0.0); g1 = T(0.0);
        if (C.kernel_model == SPH_KERNEL_GAUSSIAN) {
            const double factor = 1.0 / (K.pi_k * (h * h) * K.den);
            if (val(d) <= 3.0 * h) {
                const T e = exp(-(q * q));
                w = (e - K.e9) * factor;
                g0 = (e * (-2.0 * q)) * p0 / (d * h) * factor;
                g1 = (e * (-2.0 * q)) * p1 / (d * h) * factor;
            }
        } else {
            const double factor = 7.0 / (4 * K.pi_k * (h * h));
            if (val(d) <= 2.0 * h) {
                const T t = 1.0 - q / 2.0;
                const T t2 = t * t;
                w = factor * (1.0 + 2.0 * q) * (t2 * t2);
                g0 = factor * (-5.0 * q * (t2 * t)) * p0 / (d * h);
                g1 = factor * (-5.0 * q * (t2 * t)) * p1 / (d * h);
            }
        }
        if (val(q) <= K.q_zero) { g0 = T(0.0); g1 = T(0.0); }
    }

    // status_equation (Taylor_Green_Vortex/status_equation.f90:60-63)
    void eos(const T& rho, T& p, T& c) const {
        const T r = rho / C.rho0;
        const T r3 = r * r * r;
        if (C.eos == SPH_EOS_TAIT) p = K.eos_b * (r3 * r3 * r - 1.0) + C.background_p;
        else p = C.c0sq * (rho - C.rho0) + C.background_p;
        c = K.sqrt_c0 * r3;
    }

    // single_step_compute with the modified linear Riemann solver: drho and acc
    // of every particle (zero acceleration for non-water particles).  With sh
    // given, also the particle shift of Shift_particle_position.f90:56-100 on
    // this RHS's pairs, sh[0..1][i] = -beta h^2 sum_j (1 + R (w/w_dx)^4) V_j
    // B_i^-1 grad_i W, and the normalised density gradient gr[0..1].
    int rhs(const Parts<T>& P, std::vector<T>& drho, std::vector<T>& acc0, std::vector<T>& acc1,
            std::vector<T>* sh = nullptr, std::vector<T>* gr = nullptr, std::vector<T>* o1 = nullptr) const {
        const int n = P.n;
        std::vector<T> p(n), c(n), vol(n);
        for (int i = 0; i < n; ++i) { eos(P.rho[i], p[i], c[i]); vol[i] = P.mass[i] / P.rho[i]; }
        const double hb = (C.h + C.h) / 2.0;
        const double rcut = C.kernel_scale * hb;
        // find_particle_pair (find_particle_pair.f90:64-123): every i < j within the support
        std::vector<int> pi, pj;
        for (int i = 0; i < n - 1; ++i)
            for (int j = i + 1; j < n; ++j) {
                if (P.type[i] != SPH_TYPE_WATER && P.type[j] != SPH_TYPE_WATER) continue;
                const double a = val(P.x[i]) - val(P.x[j]), b = val(P.y[i]) - val(P.y[j]);
                if (std::fabs(a) > rcut || std::fabs(b) > rcut) continue;
                const double d = std::sqrt(a * a + b * b);
                if (d <= rcut && d >= K.cut_min) { pi.push_back(i); pj.push_back(j); }
            }
        const size_t np = pi.size();
        std::vector<T> dx0(np), dx1(np), w(np), dw0(np), dw1(np);
        for (size_t k = 0; k < np; ++k) {
            const int i = pi[k], j = pj[k];
            dx0[k] = P.x[i] - P.x[j]; dx1[k] = P.y[i] - P.y[j];
            const T d = sqrt(dx0[k] * dx0[k] + dx1[k] * dx1[k]);
            kernel(d, dx0[k], dx1[k], hb, w[k], dw0[k], dw1[k]);
        }
        if (o1) {
            // RefreshDensity_MLS_Order = 1 on this RHS's pairs (Reinitialize_particle_density.f90:71-92):
            // rho_i = sum m_j w_ij / sum_w(i), sum_w(i) = sum w_ij V_j, same-type pairs
            std::vector<T> sw(n, T(0.0)), acc(n, T(0.0));
            for (size_t k = 0; k < np; ++k) {
                const int i = pi[k], j = pj[k];
                if (P.type[i] != P.type[j]) continue;
                sw[i] += w[k] * vol[j]; sw[j] += w[k] * vol[i];
            }
            for (size_t k = 0; k < np; ++k) {
                const int i = pi[k], j = pj[k];
                if (P.type[i] != P.type[j]) continue;
                if (P.type[i] == SPH_TYPE_WATER) acc[i] += P.mass[j] * w[k] / sw[i];
                if (P.type[j] == SPH_TYPE_WATER) acc[j] += P.mass[i] * w[k] / sw[j];
            }
            *o1 = acc;
        }
        // volume fraction: free-surface candidates are outside this model's scope
        if (C.free_surface) {
            std::vector<double> fra(n, 0.0);
            for (size_t k = 0; k < np; ++k) {
                fra[pi[k]] += val(vol[pj[k]]) / K.sv;
                fra[pj[k]] += val(vol[pi[k]]) / K.sv;
            }
            for (int i = 0; i < n; ++i)
                if (P.type[i] == SPH_TYPE_WATER && fra[i] <= K.fs_thr) return SPH_E_CONFIG;
        }
        // B(L,o) += (x_j - x_i)_L dwdx_o V (Define_freesurface...f90:137-159) and its inverse
        std::vector<T> bi[4];
        for (int q = 0; q < 4; ++q) bi[q].assign(n, T(q == 0 || q == 3 ? 1.0 : 0.0));
        if (C.renormalize) {
            std::vector<T> B[4];
            for (int q = 0; q < 4; ++q) B[q].assign(n, T(0.0));
            for (size_t k = 0; k < np; ++k) {
                const int i = pi[k], j = pj[k];
                const T pd[2] = {-dx0[k], -dx1[k]}, dw[2] = {dw0[k], dw1[k]};
                for (int a = 0; a < 2; ++a)
                    for (int o = 0; o < 2; ++o) {
                        B[a * 2 + o][i] += pd[a] * dw[o] * vol[j];
                        B[a * 2 + o][j] += pd[a] * dw[o] * vol[i];
                    }
            }
            for (int i = 0; i < n; ++i) {
                if (P.type[i] != SPH_TYPE_WATER) continue;
                const T det = B[0][i] * B[3][i] - B[1][i] * B[2][i];
                if (val(det) == 0.0) continue;
                bi[0][i] = B[3][i] / det; bi[1][i] = -B[1][i] / det;
                bi[2][i] = -B[2][i] / det; bi[3][i] = B[0][i] / det;
            }
        }
        std::vector<T> ni0(np), ni1(np), nj0(np), nj1(np);
        for (size_t k = 0; k < np; ++k) {
            const int i = pi[k], j = pj[k];
            ni0[k] = bi[0][i] * dw0[k] + bi[1][i] * dw1[k];
            ni1[k] = bi[2][i] * dw0[k] + bi[3][i] * dw1[k];
            nj0[k] = bi[0][j] * dw0[k] + bi[1][j] * dw1[k];
            nj1[k] = bi[2][j] * dw0[k] + bi[3][j] * dw1[k];
        }
        // SPS strain and stress (Solver_..._SPS.f90:144-182, 256-296)
        std::vector<T> S[3], tau[3];
        for (int q = 0; q < 3; ++q) { S[q].assign(n, T(0.0)); tau[q].assign(n, T(0.0)); }
        for (size_t k = 0; k < np; ++k) {
            const int i = pi[k], j = pj[k];
            const T vd0 = -(P.u[i] - P.u[j]), vd1 = -(P.v[i] - P.v[j]);
            S[0][i] += vd0 * ni0[k] * vol[j];
            S[1][i] += (vd0 * ni1[k] + vd1 * ni0[k]) * vol[j];
            S[2][i] += vd1 * ni1[k] * vol[j];
            S[0][j] += vd0 * nj0[k] * vol[i];
            S[1][j] += (vd0 * nj1[k] + vd1 * nj0[k]) * vol[i];
            S[2][j] += vd1 * nj1[k] * vol[i];
        }
        const double dl = K.dl * C.dx;
        for (int i = 0; i < n; ++i) {
            if (P.type[i] != SPH_TYPE_WATER) continue;
            const T sxx = S[0][i], sxy = S[1][i], syy = S[2][i];
            const T abs2 = 2.0 * (sxx * sxx + syy * syy) + sxy * sxy;
            const double t = K.c012 * dl;
            const T nut = (t * t) * sqrt(abs2);
            const T kk = K.c23 * nut * (sxx + syy);
            const T blin = K.cblin * (dl * dl) * abs2;
            tau[0][i] = (2.0 * nut * sxx - kk - blin) * P.rho[i];
            tau[1][i] = (nut * sxy) * P.rho[i];
            tau[2][i] = (2.0 * nut * syy - kk - blin) * P.rho[i];
        }
        // MUSCL: normalised gradients of p, u, v (Solver_Normalized_MUSCL_Linear_Riemann_Delta_SPS.f90:151-185)
        const bool muscl = C.solver == SPH_SOLVER_MUSCL_DELTA_SPS;
        // the plain delta-SPH method (Solver_Normalized_Delta_SPH_SPS.f90:335-374,
        // 610-636): no Riemann state (v* = v-bar, P* = P-bar), Antuono's diffusion
        const bool dsph = C.solver == SPH_SOLVER_DELTA_SPS;
        std::vector<T> gp[2], gu[2], gv[2];
        if (muscl) {
            for (int q = 0; q < 2; ++q) { gp[q].assign(n, T(0.0)); gu[q].assign(n, T(0.0)); gv[q].assign(n, T(0.0)); }
            for (size_t k = 0; k < np; ++k) {
                const int i = pi[k], j = pj[k];
                const T dpp = p[j] - p[i], dpu = -(P.u[i] - P.u[j]), dpv = -(P.v[i] - P.v[j]);
                gp[0][i] += dpp * vol[j] * ni0[k]; gp[1][i] += dpp * vol[j] * ni1[k];
                gp[0][j] += dpp * vol[i] * nj0[k]; gp[1][j] += dpp * vol[i] * nj1[k];
                gu[0][i] += dpu * vol[j] * ni0[k]; gu[1][i] += dpu * vol[j] * ni1[k];
                gu[0][j] += dpu * vol[i] * nj0[k]; gu[1][j] += dpu * vol[i] * nj1[k];
                gv[0][i] += dpv * vol[j] * ni0[k]; gv[1][i] += dpv * vol[j] * ni1[k];
                gv[0][j] += dpv * vol[i] * nj0[k]; gv[1][j] += dpv * vol[i] * nj1[k];
            }
        }
        // main pair loop (Solver_..._SPS.f90:300-502)
        std::vector<T> cont(n, T(0.0)), a0(n, T(0.0)), a1(n, T(0.0));
        for (size_t k = 0; k < np; ++k) {
            const int i = pi[k], j = pj[k];
            const T Vi = vol[i], Vj = vol[j], ri = P.rho[i], rj = P.rho[j];
            const T cbar = (c[i] + c[j]) / 2.0, rbar = (ri + rj) / 2.0;
            const T Pbar = (p[i] + p[j]) / 2.0;
            const T vbar0 = (P.u[i] + P.u[j]) / 2.0, vbar1 = (P.v[i] + P.v[j]) / 2.0;
            const T r2 = dx0[k] * dx0[k] + dx1[k] * dx1[k];
            const T d = sqrt(r2);
            const T e0 = -dx0[k] / d, e1 = -dx1[k] / d;
            // left / right states: the particles' own, or the MUSCL reconstructions
            // (Solver_Normalized_MUSCL_Linear_Riemann_Delta_SPS.f90:470-502)
            T PL = p[i], PR = p[j], uI = P.u[i], vI = P.v[i], uJ = P.u[j], vJ = P.v[j];
            if (muscl) {
                const T x0 = -dx0[k], x1 = -dx1[k];     // j - i
                T li, lj;
                muscl_limiter_t(0.5 * (gp[0][i] * x0 + gp[1][i] * x1), -0.5 * (gp[0][j] * x0 + gp[1][j] * x1),
                                p[j] - p[i], li, lj);
                PL = p[i] + li; PR = p[j] - lj;
                muscl_limiter_t(0.5 * (gu[0][i] * x0 + gu[1][i] * x1), -0.5 * (gu[0][j] * x0 + gu[1][j] * x1),
                                -(P.u[i] - P.u[j]), li, lj);
                uI = P.u[i] + li; uJ = P.u[j] - lj;
                muscl_limiter_t(0.5 * (gv[0][i] * x0 + gv[1][i] * x1), -0.5 * (gv[0][j] * x0 + gv[1][j] * x1),
                                -(P.v[i] - P.v[j]), li, lj);
                vI = P.v[i] + li; vJ = P.v[j] - lj;
            }
            const T UL = uI * e0 + vI * e1, UR = uJ * e0 + vJ * e1;
            const T Ubar = (UL + UR) / 2.0;
            const T Us = Ubar + 0.5 * (PL - PR) / (rbar * K.sqrt_c0);
            const T vs0 = (Us - Ubar) * e0 + vbar0, vs1 = (Us - Ubar) * e1 + vbar1;
            const T dU = UL - UR;
            const T m3 = val(dU) > 0.0 ? 3.0 * dU : T(0.0);
            const T bR = val(m3) < val(cbar) ? m3 : cbar;
            const T Ps = dsph ? Pbar : Pbar + 0.5 * bR * rbar * dU;
            const T ws0 = dsph ? vbar0 : vs0, ws1 = dsph ? vbar1 : vs1;
            const T tmi = (uI - ws0) * ni0[k] + (vI - ws1) * ni1[k];
            const T tmj = -((uJ - ws0) * nj0[k] + (vJ - ws1) * nj1[k]);
            cont[i] += 2.0 * ri * Vj * tmi;
            cont[j] += 2.0 * rj * Vi * tmj;
            const T rij = 1.0 / (ri * rj);
            a0[i] += P.mass[j] * (-2.0 * Ps * ni0[k] * rij);
            a1[i] += P.mass[j] * (-2.0 * Ps * ni1[k] * rij);
            a0[j] -= P.mass[i] * (-2.0 * Ps * nj0[k] * rij);
            a1[j] -= P.mass[i] * (-2.0 * Ps * nj1[k] * rij);
            const T vij0 = P.u[i] - P.u[j], vij1 = P.v[i] - P.v[j];
            const T vx = vij0 * dx0[k] + vij1 * dx1[k];
            if (val(vx) < 0.0) {       // artificial viscosity (:392-417)
                const double fh = C.fai * hb;
                const T phi = hb * vx / (r2 + fh * fh);
                const T Pi = (-C.alpha * cbar * phi + C.beta * (phi * phi)) / rbar;
                a0[i] += P.mass[j] * (-Pi * ni0[k]); a1[i] += P.mass[j] * (-Pi * ni1[k]);
                a0[j] -= P.mass[i] * (-Pi * nj0[k]); a1[j] -= P.mass[i] * (-Pi * nj1[k]);
            }
            // Morris laplacian (:432-436)
            const T rdi = dx0[k] * ni0[k] + dx1[k] * ni1[k], rdj = dx0[k] * nj0[k] + dx1[k] * nj1[k];
            a0[i] += Vj * 2.0 * nu * rdi / r2 * vij0; a1[i] += Vj * 2.0 * nu * rdi / r2 * vij1;
            a0[j] -= Vi * 2.0 * nu * rdj / r2 * vij0; a1[j] -= Vi * 2.0 * nu * rdj / r2 * vij1;
            // delta-alpha artificial internal acceleration (:442-446)
            const T tt = C.delta_alpha * hb * cbar * vx / r2;
            a0[i] += tt * ni0[k] * C.rho0 / ri * Vj; a1[i] += tt * ni1[k] * C.rho0 / ri * Vj;
            a0[j] -= tt * nj0[k] * C.rho0 / rj * Vi; a1[j] -= tt * nj1[k] * C.rho0 / rj * Vi;
            // SPS force with the unnormalised gradient (:450-492), temp_p carried with the literals
            T tp = ((tau[0][i] + tau[0][j]) * dw0[k] + (tau[1][i] + tau[1][j]) * dw1[k]) * rij;
            a0[i] += P.smass[j] * tp; a0[j] -= P.smass[i] * tp;
            if (!C.reference_literals) tp = T(0.0);
            tp = (tp + (tau[2][i] + tau[2][j]) * dw1[k] + (tau[1][i] + tau[1][j]) * dw0[k]) * rij;
            a1[i] += P.smass[j] * tp; a1[j] -= P.smass[i] * tp;
        }
        // grad rho (:508-526) and delta-SPH (:552-583)
        std::vector<T> g0(n, T(0.0)), g1(n, T(0.0)), corr(n, T(0.0));
        for (size_t k = 0; k < np; ++k) {
            const int i = pi[k], j = pj[k];
            const T dr = -(P.rho[i] - P.rho[j]);
            g0[i] += dr * vol[j] * ni0[k]; g1[i] += dr * vol[j] * ni1[k];
            g0[j] += dr * vol[i] * nj0[k]; g1[j] += dr * vol[i] * nj1[k];
        }
        for (size_t k = 0; k < np; ++k) {
            const int i = pi[k], j = pj[k];
            const T pd0 = -dx0[k], pd1 = -dx1[k];
            const T r2 = pd0 * pd0 + pd1 * pd1;
            const T dr = -(P.rho[i] - P.rho[j]);
            const T cbar = (c[i] + c[j]) / 2.0;
            if (dsph) {
                const T ps0 = 2.0 * dr / r2 * pd0 - (g0[i] + g0[j]), ps1 = 2.0 * dr / r2 * pd1 - (g1[i] + g1[j]);
                corr[i] += C.delta * hb * cbar * (ps0 * ni0[k] + ps1 * ni1[k]) * vol[j];
                corr[j] -= C.delta * hb * cbar * (ps0 * nj0[k] + ps1 * nj1[k]) * vol[i];
                continue;
            }
            const T psi = dr - 0.5 * ((g0[i] + g0[j]) * pd0 + (g1[i] + g1[j]) * pd1);
            const T tmi = (pd0 * ni0[k] + pd1 * ni1[k]) / r2, tmj = (pd0 * nj0[k] + pd1 * nj1[k]) / r2;
            corr[i] += 2.0 * C.delta * hb * cbar * psi * tmi * vol[j];
            corr[j] -= 2.0 * C.delta * hb * cbar * psi * tmj * vol[i];
        }
        drho.assign(n, T(0.0)); acc0.assign(n, T(0.0)); acc1.assign(n, T(0.0));
        for (int i = 0; i < n; ++i) {
            drho[i] = cont[i];
            if (P.type[i] != SPH_TYPE_WATER) continue;
            drho[i] = drho[i] + corr[i];
            acc0[i] = a0[i]; acc1[i] = a1[i];
        }
        if (sh) {
            sh[0].assign(n, T(0.0)); sh[1].assign(n, T(0.0));
            const double h2 = C.h * C.h;
            for (size_t k = 0; k < np; ++k) {
                const int i = pi[k], j = pj[k];
                const T r = w[k] / K.w_dx;
                const T r2 = r * r;
                const T f = C.shift_beta * h2 * (1.0 + C.shift_R * (r2 * r2));
                sh[0][i] += -(f * ni0[k] * vol[j]); sh[1][i] += -(f * ni1[k] * vol[j]);
                sh[0][j] += f * nj0[k] * vol[i]; sh[1][j] += f * nj1[k] * vol[i];
            }
            gr[0] = g0; gr[1] = g1;
        }
        return SPH_OK;
    }

    // Reinitialize_particle_density, orders 3 and 6 (Reinitialize_particle_density.f90:
    // 98-181, MLS_Interpolation_In_Subdomain_Domain.f90:96-285) for the water
    // particles among the first n, from every particle within the support at the
    // current positions: rho_i = c.r with A c = e_1, A = sum W p p^T + alpha^3 I,
    // r = sum rho_j W p, p = (1, dx, dy[, dx^2, dx dy, dy^2]), (dx, dy) = (x_j - x_i)/h;
    // Shepard weights W / sum W when A is singular or, at order 6, with at most 8
    // neighbours.  A c = e_1 by Gaussian elimination (A is symmetric positive
    // definite; the oracle inverts it by Gauss-Jordan, the same c to rounding).
    void mls(Parts<T>& P, int n) const {
        const int m = C.mls_order;
        const double hb = (C.h + C.h) / 2.0, rcut = C.kernel_scale * hb;
        const double a3 = C.mls_alpha * C.mls_alpha * C.mls_alpha;
        std::vector<T> out(n);
        for (int i = 0; i < n; ++i) {
            out[i] = P.rho[i];
            if (P.type[i] != SPH_TYPE_WATER) continue;
            T A[6][7], r[6];
            for (int a = 0; a < 6; ++a) { r[a] = T(0.0); for (int b = 0; b < 7; ++b) A[a][b] = T(0.0); }
            T sw(0.0), srw(0.0);
            int k = 0;
            for (int j = 0; j < P.n; ++j) {
                const T px = P.x[i] - P.x[j], py = P.y[i] - P.y[j];
                const double d0 = std::sqrt(val(px) * val(px) + val(py) * val(py));
                if (!(d0 <= rcut) || !(d0 >= K.cut_min)) continue;
                T w, g0, g1;
                kernel(sqrt(px * px + py * py), px, py, hb, w, g0, g1);
                const T dx = -px / C.h, dy = -py / C.h;
                const T p[6] = {T(1.0), dx, dy, dx * dx, dx * dy, dy * dy};
                for (int a = 0; a < m; ++a) {
                    for (int b = 0; b < m; ++b) A[a][b] += w * p[a] * p[b];
                    r[a] += P.rho[j] * w * p[a];
                }
                sw += w; srw += P.rho[j] * w;
                ++k;
            }
            for (int a = 0; a < m; ++a) { A[a][a] += a3; A[a][m] = T(a == 0 ? 1.0 : 0.0); }
            bool ok = true;
            for (int c = 0; c < m && ok; ++c) {
                if (!(val(A[c][c]) > 0.0)) { ok = false; break; }
                for (int q = c + 1; q < m; ++q) {
                    const T f = A[q][c] / A[c][c];
                    for (int b = c; b <= m; ++b) A[q][b] -= f * A[c][b];
                }
            }
            if (!ok || (m == 6 && k <= 8)) { out[i] = srw / sw; continue; }
            T cs[6];
            for (int a = m - 1; a >= 0; --a) {
                T t = A[a][m];
                for (int b = a + 1; b < m; ++b) t -= A[a][b] * cs[b];
                cs[a] = t / A[a][a];
            }
            T rho(0.0);
            for (int a = 0; a < m; ++a) rho += cs[a] * r[a];
            out[i] = rho;
        }
        for (int i = 0; i < n; ++i) P.rho[i] = out[i];
    }

    // Distribute_Period_Boundary_Particle (:56-206): wrap, then left/right images
    // of the hosts and bottom/top images of hosts and left/right images.
    void images(std::vector<T>& hx, std::vector<T>& hy, const std::vector<T>& hu, const std::vector<T>& hv,
                const std::vector<T>& hr, const std::vector<double>& mass, const std::vector<double>& smass,
                const std::vector<int>& type, Parts<T>& P) const {
        const int n = (int)hx.size();
        const double Lx = C.box_hi[0] - C.box_lo[0], Ly = C.box_hi[1] - C.box_lo[1];
        for (int i = 0; i < n && C.periodic; ++i) {
            if (val(hx[i]) > C.box_hi[0]) hx[i] = hx[i] - Lx;
            else if (val(hx[i]) < C.box_lo[0]) hx[i] = hx[i] + Lx;
            if (val(hy[i]) > C.box_hi[1]) hy[i] = hy[i] - Ly;
            else if (val(hy[i]) < C.box_lo[1]) hy[i] = hy[i] + Ly;
        }
        P = Parts<T>();
        for (int i = 0; i < n; ++i) P.push(hx[i], hy[i], hu[i], hv[i], hr[i], mass[i], smass[i], type[i]);
        if (!C.periodic) return;
        const double band = C.kernel_scale * C.h;
        for (int i = 0; i < n; ++i) {
            const double x = val(P.x[i]);
            if (x <= C.box_lo[0] + band && x >= C.box_lo[0])
                P.push(P.x[i] + Lx, P.y[i], P.u[i], P.v[i], P.rho[i], P.mass[i], P.smass[i], SPH_TYPE_PERIODIC);
            if (x >= C.box_hi[0] - band && x <= C.box_hi[0])
                P.push(P.x[i] - Lx, P.y[i], P.u[i], P.v[i], P.rho[i], P.mass[i], P.smass[i], SPH_TYPE_PERIODIC);
        }
        const int nlr = P.n;
        for (int i = 0; i < nlr; ++i) {
            const double y = val(P.y[i]);
            if (y <= C.box_lo[1] + band && y >= C.box_lo[1])
                P.push(P.x[i], P.y[i] + Ly, P.u[i], P.v[i], P.rho[i], P.mass[i], P.smass[i], SPH_TYPE_PERIODIC);
            if (y >= C.box_hi[1] - band && y <= C.box_hi[1])
                P.push(P.x[i], P.y[i] - Ly, P.u[i], P.v[i], P.rho[i], P.mass[i], P.smass[i], SPH_TYPE_PERIODIC);
        }
    }
};

template <class T>
int run(const sph_config& cfg, int n, const T* x0, const T* y0, const T* u0, const T* v0, const T* r0,
        const double* mass, const int* type, const T& nu, int nsteps, double dt, std::vector<T>* out) {
    Model<T> M;
    M.C = cfg;
    M.K = derive(cfg);
    M.nu = nu;
    std::vector<T> hx(x0, x0 + n), hy(y0, y0 + n), hu(u0, u0 + n), hv(v0, v0 + n), hr(r0, r0 + n);
    std::vector<double> ms(mass, mass + n);
    std::vector<int> ty(type, type + n);
    std::vector<T> cr(n), ca0(n), ca1(n);
    for (int s = 0; s < nsteps; ++s) {
        Parts<T> P, B0;
        M.images(hx, hy, hu, hv, hr, ms, ms, ty, P);
        B0 = P;
        std::vector<T> dr, a0, a1;
        int rc;
        if (s == 0) {
            if ((rc = M.rhs(P, dr, a0, a1))) return rc;
        } else {
            dr.assign(P.n, T(0.0)); a0.assign(P.n, T(0.0)); a1.assign(P.n, T(0.0));
            for (int i = 0; i < n; ++i) { dr[i] = cr[i]; a0[i] = ca0[i]; a1[i] = ca1[i]; }
        }
        std::vector<T> Kr(n), Ka0(n), Ka1(n), Kv0(n), Kv1(n);
        std::vector<T> sh[2], gr[2], o1;
        // density re-initialisation after every mls_every-th step (1-based)
        const bool mls_step = cfg.mls_order != 0 && (s + 1) % cfg.mls_every == 0;
        // stages (time_iteration.f90:942-1047): water particles only
        for (int st = 0; st < 3; ++st) {
            const double f = st < 2 ? 0.5 * dt : dt;
            const double wgt = st == 0 ? 1.0 : 2.0;
            for (int i = 0; i < n; ++i) {
                if (P.type[i] != SPH_TYPE_WATER) continue;
                P.rho[i] = st < 2 ? B0.rho[i] + dr[i] * dt / 2 : B0.rho[i] + dr[i] * dt;
                P.u[i] = B0.u[i] + f * a0[i];
                P.x[i] = B0.x[i] + f * P.u[i];
                P.v[i] = B0.v[i] + f * a1[i];
                P.y[i] = B0.y[i] + f * P.v[i];
                Kr[i] += wgt * dr[i]; Ka0[i] += wgt * a0[i]; Ka1[i] += wgt * a1[i];
                Kv0[i] += wgt * P.u[i]; Kv1[i] += wgt * P.v[i];
            }
            if ((rc = M.rhs(P, dr, a0, a1, st == 2 && cfg.shifting ? sh : nullptr, gr,
                            st == 2 && mls_step && cfg.mls_order == 1 ? &o1 : nullptr)))
                return rc;
        }
        for (int i = 0; i < n; ++i) {
            if (P.type[i] != SPH_TYPE_WATER) continue;
            P.rho[i] = B0.rho[i] + (Kr[i] + dr[i]) * dt / 6.0;
            P.u[i] = B0.u[i] + (Ka0[i] + a0[i]) * dt / 6.0;
            P.x[i] = B0.x[i] + (Kv0[i] + P.u[i]) * dt / 6.0 + 0.5 * dt * dt * a0[i];
            P.v[i] = B0.v[i] + (Ka1[i] + a1[i]) * dt / 6.0;
            P.y[i] = B0.y[i] + (Kv1[i] + P.v[i]) * dt / 6.0 + 0.5 * dt * dt * a1[i];
        }
        if (mls_step) {
            if (cfg.mls_order == 1) {
                for (int i = 0; i < n; ++i)
                    if (P.type[i] == SPH_TYPE_WATER) P.rho[i] = o1[i];
            } else {
                M.mls(P, n);
            }
        }
        if (cfg.shifting) {
            // Shift_particle_position.f90:97-136 on the last RHS's pairs: capped
            // shift of the water particles (none is near a surface in this model's
            // scope) and the first-order density correction
            for (int i = 0; i < n; ++i) {
                if (P.type[i] != SPH_TYPE_WATER) continue;
                T s0 = sh[0][i], s1 = sh[1][i];
                const T amp = sqrt(s0 * s0 + s1 * s1);
                if (val(amp) > cfg.shift_max) { s0 = s0 / amp * cfg.shift_max; s1 = s1 / amp * cfg.shift_max; }
                P.x[i] = P.x[i] + s0; P.y[i] = P.y[i] + s1;
                P.rho[i] = P.rho[i] + gr[0][i] * s0;
                P.rho[i] = P.rho[i] + gr[1][i] * s1;
            }
        }
        for (int i = 0; i < n; ++i) {
            cr[i] = dr[i]; ca0[i] = a0[i]; ca1[i] = a1[i];
            hx[i] = P.x[i]; hy[i] = P.y[i]; hu[i] = P.u[i]; hv[i] = P.v[i]; hr[i] = P.rho[i];
        }
    }
    out[0] = hx; out[1] = hy; out[2] = hu; out[3] = hv; out[4] = hr;
    return SPH_OK;
}

// ---------------------------------------------------------------------------
// Moving-square step (Moving_Square_Cylinder_Flow/...): the modified linear
// Riemann solver, or the HLLC solver (Solver_Normalized_HLLC_Riemann_Delta.f90),
// with the XSPH velocity inside the continuity flux
// (Solver_Normalized_Modified_Linear_Riemann_Delta.f90:100-336), the fixed-ghost
// assignment (Assign_boundary_particles.f90:611-941, MLS order 1), the body force
// (Calculate_Body_Force.f90:53-142) and the Euler predictor-corrector with the
// carried rates (SPH_Time_Iteration.f90:313-394), the body moved at each step
// start by a per-step velocity (Body_Motion_Solver.f90:187-193).  The same
// steps, in the same pair orientation and order, as sph_oracle.cpp's
// ms_riemann_solver / assign_ghosts / body_force / run_step_euler_pc, with the
// masses as scalars of type T (the ghost masses are interpolated).
// ---------------------------------------------------------------------------
// The HLLC pair state of Moving_Square.../Solver_Normalized_HLLC_Riemann_Delta.f90:207-322
// (the same operations as sph_oracle.cpp's hllc_state), on scalars of type T:
// branches on the values, derivatives through the taken branch.
template <class T>
void hllc_state_t(const sph_config& C, const T vI[2], const T vJ[2], const T vbar[2], const T e[2], const T& rL,
                  const T& rR, const T& cL, const T& cR, const T& PL, const T& PR, T vs[2], T& Ps) {
    const T Tm[2][2] = {{e[0], e[1]}, {-e[1], e[0]}};
    const T VL[2] = {Tm[0][0] * vI[0] + Tm[0][1] * vI[1], Tm[1][0] * vI[0] + Tm[1][1] * vI[1]};
    const T VR[2] = {Tm[0][0] * vJ[0] + Tm[0][1] * vJ[1], Tm[1][0] * vJ[0] + Tm[1][1] * vJ[1]};
    const T V0 = Tm[0][0] * vbar[0] + Tm[0][1] * vbar[1];
    const T Us = (VR[0] * cL * rL + VL[0] * cR * rR + PL - PR) / (rL * cL + rR * cR);
    const T Pst = (PR * cL * rL + PL * cR * rR - cL * rL * cR * rR * (VR[0] - VL[0])) / (rL * cL + rR * cR);
    const T rst = (Pst - C.background_p) / C.c0sq + C.rho0;
    T QL(1.0), QR(1.0);
    if (!(val(Pst) <= val(PL)) && val(rL) > val(rst)) QL = sqrt((rst / rL) * (Pst - PL) / (rL - rst)) / cL;
    const T SL = VL[0] - cL * QL;
    if (!(val(Pst) <= val(PR)) && val(rR) > val(rst)) QR = sqrt((rst / rR) * (Pst - PR) / (rR - rst)) / cR;
    const T SR = VR[0] + cR * QR;
    T rH, VH[2];
    if (val(SL) > val(V0)) { rH = rL; VH[0] = VL[0]; VH[1] = VL[1]; }
    else if (val(Us) >= val(V0) && val(V0) >= val(SL)) {
        const T q = rL * ((SL - VL[0]) / (SL - Us));
        rH = q; VH[0] = (Us * q) / rH; VH[1] = (VL[1] * q) / rH;
    } else if (val(SR) >= val(V0) && val(V0) >= val(Us)) {
        const T q = rR * ((SR - VR[0]) / (SR - Us));
        rH = q; VH[0] = (Us * q) / rH; VH[1] = (VR[1] * q) / rH;
    } else { rH = rR; VH[0] = VR[0]; VH[1] = VR[1]; }
    vs[0] = Tm[0][0] * VH[0] + Tm[1][0] * VH[1];
    vs[1] = Tm[0][1] * VH[0] + Tm[1][1] * VH[1];
    Ps = C.c0sq * (rH - C.rho0) + C.background_p;
}

template <class T>
struct MSParts {
    std::vector<T> x, y, u, v, rho, mass;
    std::vector<int> type, itype, label;
    int n = 0;
};

template <class T>
struct MSModel {
    Model<T> M;
    double t = 0.0;          // Real_physical_time of the step
    T bvel[2], bacc[2];      // Custom_velocity, Custom_accleration of the step

    bool pair_allowed(int ti, int tj) const {
        if (M.C.pair_rule == SPH_PAIRS_ONE_FLUID) return !(ti != SPH_TYPE_WATER && tj != SPH_TYPE_WATER);
        if (ti == -2 && tj == -2) return false;
        if (ti == -3 && tj == -3) return false;
        if (ti == -201 && tj == -201) return false;
        return true;
    }

    void assign_ghosts(MSParts<T>& P, std::vector<T>& p, std::vector<T>& c, std::vector<T>& vol) const {
        const sph_config& C = M.C;
        const bool q = C.reference_literals != 0;
        const double hg = (q ? (double)(float)C.ghost_h_factor : C.ghost_h_factor) * C.h;
        const double rg = C.kernel_scale * hg;
        for (int i = 0; i < P.n; ++i) {
            if (P.type[i] != SPH_TYPE_FIX_GHOST) continue;
            const bool body = P.itype[i] == SPH_TYPE_BODY;
            const T ge0 = body ? C.gravity[0] + bacc[0] : T(C.gravity[0]);
            const T ge1 = body ? C.gravity[1] + bacc[1] : T(C.gravity[1]);
            std::vector<int> nb;
            std::vector<T> W;
            for (int j = 0; j < P.n; ++j) {
                if (P.type[j] == SPH_TYPE_FIX_GHOST || P.type[j] == SPH_TYPE_ILL || P.type[j] == 0) continue;
                const T pd0 = P.x[i] - P.x[j], pd1 = P.y[i] - P.y[j];
                const T d = sqrt(pd0 * pd0 + pd1 * pd1);
                if (!(val(d) <= rg)) continue;
                T w, g0, g1;
                M.kernel(d, pd0, pd1, hg, w, g0, g1);
                nb.push_back(j);
                W.push_back(w * P.mass[j] / P.rho[j]);
            }
            T pint(0.0), uint(0.0), vint(0.0), m(0.0);
            if (nb.size() >= 3) {
                T A(0.0);
                for (const T& w : W) A += w;
                const T ainv = 1.0 / A;
                for (size_t k = 0; k < nb.size(); ++k) {
                    const int j = nb[k];
                    const T fai = ainv * W[k];
                    const T pd0 = P.x[i] - P.x[j], pd1 = P.y[i] - P.y[j];
                    pint = pint + p[j] * fai + P.rho[j] * fai * (ge0 * pd0 + ge1 * pd1);
                    uint = uint + P.u[j] * fai;
                    vint = vint + P.v[j] * fai;
                    m = m + P.mass[j] * fai;
                }
            }
            T u, v, pr(0.0);
            const int lab = P.label[i];
            if (body) {
                u = bvel[0]; v = bvel[1]; pr = pint;
            } else {
                if (0.0 < t && t <= C.shock_release_time) {
                    const T ri = (pint - C.background_p) / C.c0sq + C.rho0;
                    const T r = ri / C.rho0;
                    const T cc = M.K.sqrt_c0 * (r * r * r);
                    u = uint; v = vint;
                    if (lab == -6 || lab == -7) {
                        const T vn = lab == -6 ? vint : uint;
                        const T J2 = ri * cc * vn + pint, J3 = -ri * cc * vn + pint;
                        const T vsn = (J2 - J3) / (2.0 * ri * cc);
                        if (lab == -6) v = vsn; else u = vsn;
                        pr = 0.5 * (J2 + J3);
                    }
                } else {
                    u = uint; v = vint; pr = pint;
                }
                if (lab == -6) { if (C.wall_bc == 1) v = -v; else { u = -u; v = -v; } }
                else if (lab == -7) { u = -u; v = -v; }
                else if (lab == -8) { if (C.wall_bc == 1) u = -u; else { u = -u; v = -v; } }
            }
            T rho, cc;
            if (val(m) != 0.0) {
                rho = (pr - C.background_p) / C.c0sq + C.rho0;
                const T r = rho / C.rho0;
                cc = M.K.sqrt_c0 * (r * r * r);
            } else {
                u = T(0.0); v = T(0.0); pr = T(0.0); rho = T(C.rho0); m = T(0.0); cc = T(M.K.sqrt_c0);
            }
            P.u[i] = u; P.v[i] = v; P.rho[i] = rho; P.mass[i] = m;
            p[i] = pr; c[i] = cc; vol[i] = m / rho;
        }
    }

    // Reinitialize_particle_density, orders 3 and 6, moving-square variant
    // (Moving_Square.../Reinitialize_particle_density.f90:92-200 with
    // SPH_Subroutine_Module.f90:2565-2792) on the state after the corrector, the
    // ghosts as the corrector RHS assigned them: for a water particle i every
    // particle j within the support, i itself included, weighted by W_ij V_j,
    // V_j = m_j / rho_j; rho_i = c.r with A c = e_1, A = sum W V p p^T + alpha^3 I,
    // r = sum rho_j W V p; Shepard weights when A is singular (no few-neighbour
    // fallback); the old density where the result is NaN.
    void mls(MSParts<T>& P) const {
        const sph_config& C = M.C;
        const int m = C.mls_order;
        const double hb = (C.h + C.h) / 2.0, rcut = C.kernel_scale * hb;
        const double a3 = C.mls_alpha * C.mls_alpha * C.mls_alpha;
        std::vector<T> out(P.n);
        for (int i = 0; i < P.n; ++i) {
            out[i] = P.rho[i];
            if (P.type[i] != SPH_TYPE_WATER) continue;
            T A[6][7], r[6];
            for (int a = 0; a < 6; ++a) { r[a] = T(0.0); for (int b = 0; b < 7; ++b) A[a][b] = T(0.0); }
            T sw(0.0), srw(0.0);
            for (int j = 0; j < P.n; ++j) {
                const T px = P.x[i] - P.x[j], py = P.y[i] - P.y[j];
                const double d0 = std::sqrt(val(px) * val(px) + val(py) * val(py));
                if (!(d0 <= rcut)) continue;
                T w, g0, g1;
                // the particle itself: distance 0 with no derivative
                M.kernel(j == i ? T(0.0) : sqrt(px * px + py * py), px, py, hb, w, g0, g1);
                w = w * (P.mass[j] / P.rho[j]);
                const T dx = -px / C.h, dy = -py / C.h;
                const T p[6] = {T(1.0), dx, dy, dx * dx, dx * dy, dy * dy};
                for (int a = 0; a < m; ++a) {
                    for (int b = 0; b < m; ++b) A[a][b] += w * p[a] * p[b];
                    r[a] += P.rho[j] * w * p[a];
                }
                sw += w; srw += P.rho[j] * w;
            }
            for (int a = 0; a < m; ++a) { A[a][a] += a3; A[a][m] = T(a == 0 ? 1.0 : 0.0); }
            bool ok = true;
            for (int c = 0; c < m && ok; ++c) {
                if (!(val(A[c][c]) > 0.0)) { ok = false; break; }
                for (int q = c + 1; q < m; ++q) {
                    const T f = A[q][c] / A[c][c];
                    for (int b = c; b <= m; ++b) A[q][b] -= f * A[c][b];
                }
            }
            T rho(0.0);
            if (!ok) {
                rho = srw / sw;
            } else {
                T cs[6];
                for (int a = m - 1; a >= 0; --a) {
                    T t = A[a][m];
                    for (int b = a + 1; b < m; ++b) t -= A[a][b] * cs[b];
                    cs[a] = t / A[a][a];
                }
                for (int a = 0; a < m; ++a) rho += cs[a] * r[a];
            }
            if (!std::isnan(val(rho))) out[i] = rho;
        }
        for (int i = 0; i < P.n; ++i) P.rho[i] = out[i];
    }

    // single_step_compute of the moving square: the rates of every particle and,
    // when fx is given, the x body force of this RHS.
    int rhs(MSParts<T>& P, std::vector<T>& drho, std::vector<T>* acc, std::vector<T>* avg, T* fx,
            std::vector<T>* sh = nullptr, std::vector<T>* gr = nullptr, std::vector<T>* o1 = nullptr) const {
        const sph_config& C = M.C;
        const TConsts& K = M.K;
        const T& nu = M.nu;
        const int n = P.n;
        std::vector<T> p(n), c(n), vol(n);
        for (int i = 0; i < n; ++i) {
            if (P.type[i] == SPH_TYPE_ILL) continue;
            M.eos(P.rho[i], p[i], c[i]);
        }
        for (int i = 0; i < n; ++i) vol[i] = P.mass[i] / P.rho[i];
        if (C.ghost_assign) assign_ghosts(P, p, c, vol);
        const double hb = (C.h + C.h) / 2.0;
        const double rcut = C.kernel_scale * hb;
        std::vector<int> pi, pj;
        for (int i = 0; i < n - 1; ++i)
            for (int j = i + 1; j < n; ++j) {
                if (!pair_allowed(P.type[i], P.type[j])) continue;
                const double a = val(P.x[i]) - val(P.x[j]), b = val(P.y[i]) - val(P.y[j]);
                if (std::fabs(a) > rcut || std::fabs(b) > rcut) continue;
                const double d = std::sqrt(a * a + b * b);
                if (d <= rcut && d >= K.cut_min) { pi.push_back(i); pj.push_back(j); }
            }
        const size_t np = pi.size();
        std::vector<T> dx0(np), dx1(np), w(np), dw0(np), dw1(np);
        for (size_t k = 0; k < np; ++k) {
            const int i = pi[k], j = pj[k];
            dx0[k] = P.x[i] - P.x[j]; dx1[k] = P.y[i] - P.y[j];
            const T d = sqrt(dx0[k] * dx0[k] + dx1[k] * dx1[k]);
            M.kernel(d, dx0[k], dx1[k], hb, w[k], dw0[k], dw1[k]);
        }
        if (o1) {
            // RefreshDensity_MLS_Order = 1 on this RHS's pairs (Moving_Square.../
            // Reinitialize_particle_density.f90:66-88): rho_i = sum m_j w_ij / sum_w(i),
            // sum_w(i) = sum w_ij V_j over the same-type pairs
            std::vector<T> sw(n, T(0.0)), a1(n, T(0.0));
            for (size_t k = 0; k < np; ++k) {
                const int i = pi[k], j = pj[k];
                if (P.type[i] != P.type[j]) continue;
                sw[i] += w[k] * vol[j]; sw[j] += w[k] * vol[i];
            }
            for (size_t k = 0; k < np; ++k) {
                const int i = pi[k], j = pj[k];
                if (P.type[i] != P.type[j]) continue;
                if (P.type[i] == SPH_TYPE_WATER) a1[i] += P.mass[j] * w[k] / sw[i];
                if (P.type[j] == SPH_TYPE_WATER) a1[j] += P.mass[i] * w[k] / sw[j];
            }
            *o1 = a1;
        }
        std::vector<T> bi[4];
        for (int q = 0; q < 4; ++q) bi[q].assign(n, T(q == 0 || q == 3 ? 1.0 : 0.0));
        if (C.renormalize) {
            std::vector<T> B[4];
            for (int q = 0; q < 4; ++q) B[q].assign(n, T(0.0));
            for (size_t k = 0; k < np; ++k) {
                const int i = pi[k], j = pj[k];
                const T pd[2] = {-dx0[k], -dx1[k]}, dw[2] = {dw0[k], dw1[k]};
                for (int a = 0; a < 2; ++a)
                    for (int o = 0; o < 2; ++o) {
                        B[a * 2 + o][i] += pd[a] * dw[o] * vol[j];
                        B[a * 2 + o][j] += pd[a] * dw[o] * vol[i];
                    }
            }
            for (int i = 0; i < n; ++i) {
                if (P.type[i] != SPH_TYPE_WATER) continue;
                const T det = B[0][i] * B[3][i] - B[1][i] * B[2][i];
                if (val(det) == 0.0) continue;
                bi[0][i] = B[3][i] / det; bi[1][i] = -B[1][i] / det;
                bi[2][i] = -B[2][i] / det; bi[3][i] = B[0][i] / det;
            }
        }
        std::vector<T> ni0(np), ni1(np), nj0(np), nj1(np);
        for (size_t k = 0; k < np; ++k) {
            const int i = pi[k], j = pj[k];
            ni0[k] = bi[0][i] * dw0[k] + bi[1][i] * dw1[k];
            ni1[k] = bi[2][i] * dw0[k] + bi[3][i] * dw1[k];
            nj0[k] = bi[0][j] * dw0[k] + bi[1][j] * dw1[k];
            nj1[k] = bi[2][j] * dw0[k] + bi[3][j] * dw1[k];
        }
        // grad rho (:100-112) and the XSPH average velocity (:114-121)
        std::vector<T> g0(n, T(0.0)), g1(n, T(0.0));
        for (int a = 0; a < 2; ++a) avg[a].assign(n, T(0.0));
        for (size_t k = 0; k < np; ++k) {
            const int i = pi[k], j = pj[k];
            const T dr = -(P.rho[i] - P.rho[j]);
            g0[i] += dr * vol[j] * ni0[k]; g1[i] += dr * vol[j] * ni1[k];
            g0[j] += dr * vol[i] * nj0[k]; g1[j] += dr * vol[i] * nj1[k];
            const T vd[2] = {P.u[i] - P.u[j], P.v[i] - P.v[j]};
            for (int a = 0; a < 2; ++a) {
                avg[a][i] += -(C.xsph_eps * P.mass[j] * vd[a] / (P.rho[i] + P.rho[j]) * w[k]);
                avg[a][j] += C.xsph_eps * P.mass[i] * vd[a] / (P.rho[i] + P.rho[j]) * w[k];
            }
        }
        // main pair loop (:169-336), no free surface
        std::vector<T> cont(n, T(0.0)), a0(n, T(0.0)), a1(n, T(0.0));
        for (size_t k = 0; k < np; ++k) {
            const int i = pi[k], j = pj[k];
            const T Vi = vol[i], Vj = vol[j], ri = P.rho[i], rj = P.rho[j];
            const T cbar = (c[i] + c[j]) / 2.0, rbar = (ri + rj) / 2.0;
            const T Pbar = (p[i] + p[j]) / 2.0;
            const T vbar0 = (P.u[i] + P.u[j]) / 2.0, vbar1 = (P.v[i] + P.v[j]) / 2.0;
            const T r2 = dx0[k] * dx0[k] + dx1[k] * dx1[k];
            const T d = sqrt(r2);
            const T e0 = -dx0[k] / d, e1 = -dx1[k] / d;
            T vs0, vs1, Ps;
            if (C.solver == SPH_SOLVER_MS_HLLC_DELTA) {
                const T vI[2] = {P.u[i], P.v[i]}, vJ[2] = {P.u[j], P.v[j]}, vb[2] = {vbar0, vbar1}, ee[2] = {e0, e1};
                T vs[2];
                hllc_state_t(C, vI, vJ, vb, ee, ri, rj, c[i], c[j], p[i], p[j], vs, Ps);
                vs0 = vs[0]; vs1 = vs[1];
            } else {
                const T UL = P.u[i] * e0 + P.v[i] * e1, UR = P.u[j] * e0 + P.v[j] * e1;
                const T Ubar = (UL + UR) / 2.0;
                const T Us = Ubar + 0.5 * (p[i] - p[j]) / (rbar * K.sqrt_c0);
                vs0 = (Us - Ubar) * e0 + vbar0; vs1 = (Us - Ubar) * e1 + vbar1;
                const T dU = UL - UR;
                const T m3 = val(dU) > 0.0 ? 3.0 * dU : T(0.0);
                const T bR = val(m3) < val(cbar) ? m3 : cbar;
                Ps = Pbar + 0.5 * bR * rbar * dU;
            }
            const T vdi0 = P.u[i] - vs0 + avg[0][i] - avg[0][j], vdi1 = P.v[i] - vs1 + avg[1][i] - avg[1][j];
            const T vdj0 = P.u[j] - vs0 + avg[0][j] - avg[0][i], vdj1 = P.v[j] - vs1 + avg[1][j] - avg[1][i];
            const T tmi = vdi0 * ni0[k] + vdi1 * ni1[k];
            const T tmj = -(vdj0 * nj0[k] + vdj1 * nj1[k]);
            cont[i] += 2.0 * ri * Vj * tmi;
            cont[j] += 2.0 * rj * Vi * tmj;
            const T rij = 1.0 / (ri * rj);
            a0[i] += P.mass[j] * (-2.0 * Ps * ni0[k] * rij);
            a1[i] += P.mass[j] * (-2.0 * Ps * ni1[k] * rij);
            a0[j] += -(P.mass[i] * (-2.0 * Ps * nj0[k] * rij));
            a1[j] += -(P.mass[i] * (-2.0 * Ps * nj1[k] * rij));
            const T vij0 = P.u[i] - P.u[j], vij1 = P.v[i] - P.v[j];
            const T vx = vij0 * dx0[k] + vij1 * dx1[k];
            if (val(vx) < 0.0) {
                const double fh = C.fai * hb;
                const T phi = hb * vx / (r2 + fh * fh);
                const T Pi = (-C.alpha * cbar * phi + C.beta * (phi * phi)) / rbar;
                a0[i] += P.mass[j] * (-Pi * ni0[k]); a1[i] += P.mass[j] * (-Pi * ni1[k]);
                a0[j] += -(P.mass[i] * (-Pi * nj0[k])); a1[j] += -(P.mass[i] * (-Pi * nj1[k]));
            }
            const T rdi = dx0[k] * ni0[k] + dx1[k] * ni1[k], rdj = dx0[k] * nj0[k] + dx1[k] * nj1[k];
            a0[i] += Vj * 2.0 * nu * rdi / r2 * vij0; a1[i] += Vj * 2.0 * nu * rdi / r2 * vij1;
            a0[j] += -(Vi * 2.0 * nu * rdj / r2 * vij0); a1[j] += -(Vi * 2.0 * nu * rdj / r2 * vij1);
            const T tt = C.delta_alpha * hb * cbar * vx / r2;
            a0[i] += tt * ni0[k] * C.rho0 / ri * Vj; a1[i] += tt * ni1[k] * C.rho0 / ri * Vj;
            a0[j] += -(tt * nj0[k] * C.rho0 / rj * Vi); a1[j] += -(tt * nj1[k] * C.rho0 / rj * Vi);
        }
        // delta-SPH (:531-545)
        std::vector<T> corr(n, T(0.0));
        for (size_t k = 0; k < np; ++k) {
            const int i = pi[k], j = pj[k];
            const T pd0 = -dx0[k], pd1 = -dx1[k];
            const T r2 = pd0 * pd0 + pd1 * pd1;
            const T dr = -(P.rho[i] - P.rho[j]);
            const T cbar = (c[i] + c[j]) / 2.0;
            const T psi = dr - 0.5 * ((g0[i] + g0[j]) * pd0 + (g1[i] + g1[j]) * pd1);
            const T tmi = (pd0 * ni0[k] + pd1 * ni1[k]) / r2, tmj = (pd0 * nj0[k] + pd1 * nj1[k]) / r2;
            corr[i] += 2.0 * C.delta * hb * cbar * psi * tmi * vol[j];
            corr[j] += -(2.0 * C.delta * hb * cbar * psi * tmj * vol[i]);
        }
        drho.assign(n, T(0.0)); acc[0].assign(n, T(0.0)); acc[1].assign(n, T(0.0));
        for (int i = 0; i < n; ++i) {
            drho[i] = cont[i];
            if (P.type[i] != SPH_TYPE_WATER) continue;
            acc[0][i] = a0[i]; acc[1][i] = a1[i];
            drho[i] = drho[i] + corr[i];
        }
        if (sh) {
            // the particle shift on this RHS's pairs (Shift_particle_position.f90:56-100),
            // sh[0..1][i] = -beta h^2 sum_j (1 + R (w/w_dx)^4) V_j B_i^-1 grad_i W, and
            // the normalised density gradient gr[0..1]
            sh[0].assign(n, T(0.0)); sh[1].assign(n, T(0.0));
            const double h2 = C.h * C.h;
            for (size_t k = 0; k < np; ++k) {
                const int i = pi[k], j = pj[k];
                const T r = w[k] / K.w_dx;
                const T r2 = r * r;
                const T f = C.shift_beta * h2 * (1.0 + C.shift_R * (r2 * r2));
                sh[0][i] += -(f * ni0[k] * vol[j]); sh[1][i] += -(f * ni1[k] * vol[j]);
                sh[0][j] += f * nj0[k] * vol[i]; sh[1][j] += f * nj1[k] * vol[i];
            }
            gr[0] = g0; gr[1] = g1;
        }
        if (fx) {
            // Calculate_Body_Force, x component of the total (Morris laplacian)
            std::vector<T> bp(n, T(0.0)), bv(n, T(0.0));
            std::vector<int> nearb(n, 0);
            for (size_t k = 0; k < np; ++k) {
                const int i = pi[k], j = pj[k];
                if (P.itype[i] != SPH_TYPE_BODY && P.itype[j] != SPH_TYPE_BODY) continue;
                const T vij0 = P.u[i] - P.u[j];
                const T r2 = dx0[k] * dx0[k] + dx1[k] * dx1[k];
                if (P.itype[j] == SPH_TYPE_BODY) {
                    nearb[i] = 1;
                    bp[i] = bp[i] - vol[j] * (p[i] + p[j]) * ni0[k];
                    const T rd = dx0[k] * ni0[k] + dx1[k] * ni1[k];
                    bv[i] = bv[i] + P.rho[i] * vol[j] * 2.0 * nu * rd / r2 * vij0;
                }
                if (P.itype[i] == SPH_TYPE_BODY) {
                    nearb[j] = 1;
                    bp[j] = bp[j] + vol[i] * (p[i] + p[j]) * nj0[k];
                    const T rd = dx0[k] * nj0[k] + dx1[k] * nj1[k];
                    bv[j] = bv[j] - P.rho[j] * vol[i] * 2.0 * nu * rd / r2 * vij0;
                }
            }
            T f(0.0);
            for (int i = 0; i < n; ++i)
                if (nearb[i]) f = f + vol[i] * (bp[i] + bv[i] + 0.0);
            *fx = f;
        }
        return SPH_OK;
    }
};

// nsteps Euler predictor-corrector steps of the moving square; motion[4s..4s+3]
// is step s's body velocity and acceleration.  Returns the final state in H and
// the drag impulse sum_s dt F_x(s) in drag.
template <class T>
int run_ms(const sph_config& cfg, MSParts<T>& H, const T& nu, const std::vector<T>& motion, double t0, int nsteps,
           double dt, T& drag) {
    MSModel<T> S;
    S.M.C = cfg;
    S.M.K = derive(cfg);
    S.M.nu = nu;
    const int n = H.n;
    std::vector<T> rdrho, racc[2], ravg[2];
    double t = t0;
    drag = T(0.0);
    for (int s = 0; s < nsteps; ++s) {
        t += dt;
        S.t = t;
        S.bvel[0] = motion[4 * s]; S.bvel[1] = motion[4 * s + 1];
        S.bacc[0] = motion[4 * s + 2]; S.bacc[1] = motion[4 * s + 3];
        if (cfg.ghost_assign)
            for (int i = 0; i < n; ++i)
                if (H.itype[i] == SPH_TYPE_BODY) { H.x[i] = H.x[i] + S.bvel[0] * dt; H.y[i] = H.y[i] + S.bvel[1] * dt; }
        MSParts<T> P = H;
        const MSParts<T> B0 = H;
        std::vector<T> dr, a[2], g[2];
        int rc;
        if (s == 0) {
            if ((rc = S.rhs(P, dr, a, g, nullptr))) return rc;
        } else {
            dr = rdrho; a[0] = racc[0]; a[1] = racc[1]; g[0] = ravg[0]; g[1] = ravg[1];
        }
        const std::vector<T> td = dr, ta0 = a[0], ta1 = a[1], tv0 = P.u, tv1 = P.v;
        for (int i = 0; i < n; ++i) {
            if (P.type[i] != SPH_TYPE_WATER) continue;
            P.rho[i] = B0.rho[i] + dr[i] * dt;
            P.x[i] = B0.x[i] + dt * (P.u[i] + g[0][i]) + 0.5 * a[0][i] * (dt * dt);
            P.y[i] = B0.y[i] + dt * (P.v[i] + g[1][i]) + 0.5 * a[1][i] * (dt * dt);
            P.u[i] = B0.u[i] + dt * a[0][i];
            P.v[i] = B0.v[i] + dt * a[1][i];
        }
        T fx;
        std::vector<T> sh[2], gr[2], o1;
        const bool mls_step = cfg.mls_order != 0 && (s + 1) % cfg.mls_every == 0;
        if ((rc = S.rhs(P, dr, a, g, &fx, cfg.shifting ? sh : nullptr, gr,
                        mls_step && cfg.mls_order == 1 ? &o1 : nullptr)))
            return rc;
        drag = drag + dt * fx;
        for (int i = 0; i < n; ++i) {
            if (P.type[i] != SPH_TYPE_WATER) continue;
            P.rho[i] = B0.rho[i] + 0.5 * (dr[i] + td[i]) * dt;
            P.x[i] = B0.x[i] + 0.5 * dt * (P.u[i] + tv0[i]) + g[0][i] * dt + 0.5 * a[0][i] * (dt * dt);
            P.y[i] = B0.y[i] + 0.5 * dt * (P.v[i] + tv1[i]) + g[1][i] * dt + 0.5 * a[1][i] * (dt * dt);
            P.u[i] = B0.u[i] + 0.5 * dt * (a[0][i] + ta0[i]);
            P.v[i] = B0.v[i] + 0.5 * dt * (a[1][i] + ta1[i]);
        }
        // density re-initialisation after every mls_every-th step (1-based), before
        // the shift
        if (mls_step) {
            if (cfg.mls_order == 1) {
                for (int i = 0; i < n; ++i)
                    if (P.type[i] == SPH_TYPE_WATER) P.rho[i] = o1[i];
            } else {
                S.mls(P);
            }
        }
        if (cfg.shifting) {
            // the capped shift of the water particles (none is near a free surface
            // here) and the first-order density correction
            for (int i = 0; i < n; ++i) {
                if (P.type[i] != SPH_TYPE_WATER) continue;
                T s0 = sh[0][i], s1 = sh[1][i];
                const T amp = sqrt(s0 * s0 + s1 * s1);
                if (val(amp) > cfg.shift_max) { s0 = s0 / amp * cfg.shift_max; s1 = s1 / amp * cfg.shift_max; }
                P.x[i] = P.x[i] + s0; P.y[i] = P.y[i] + s1;
                P.rho[i] = P.rho[i] + gr[0][i] * s0;
                P.rho[i] = P.rho[i] + gr[1][i] * s1;
            }
        }
        rdrho = dr; racc[0] = a[0]; racc[1] = a[1]; ravg[0] = g[0]; ravg[1] = g[1];
        for (int i = 0; i < n; ++i) {
            H.x[i] = P.x[i]; H.y[i] = P.y[i]; H.u[i] = P.u[i]; H.v[i] = P.v[i]; H.rho[i] = P.rho[i];
        }
    }
    return SPH_OK;
}

}  // namespace

extern "C" {

// nsteps time steps from (pos, vel, rho) along the tangent direction
// (dpos, dvel, drho, dnu) (any of the arrays may be NULL = zero).  out[0] = loss
// of the final state (SPH_LOSS_*; target_vel for the misfit), out[1] = its
// directional derivative.  The final state (values) goes to pos_out, vel_out,
// rho_out when they are given.  Arrays are column-major (n,2) like the ABI's.
int oracle_tangent(const sph_config* cfg, int n, const double* pos, const double* vel, const double* rho,
                   const double* mass, const int* type, const double* dpos, const double* dvel, const double* drho,
                   double dnu, int nsteps, double dt, int loss, const double* target_vel, double* out,
                   double* pos_out, double* vel_out, double* rho_out) {
    if (!cfg || !pos || !vel || !rho || !mass || !type || !out || n <= 0 || nsteps <= 0) return SPH_E_ARG;
    if ((cfg->solver != SPH_SOLVER_MODLR_DELTA_SPS && cfg->solver != SPH_SOLVER_MUSCL_DELTA_SPS &&
         cfg->solver != SPH_SOLVER_DELTA_SPS) ||
        cfg->integrator != SPH_INTEGRATOR_RK4_REUSE ||
        cfg->xsph_eps != 0.0 || cfg->pair_rule != SPH_PAIRS_ONE_FLUID)
        return SPH_E_CONFIG;
    if (loss == SPH_LOSS_VELOCITY_MISFIT && !target_vel) return SPH_E_ARG;
    std::vector<Dual> x(n), y(n), u(n), v(n), r(n);
    for (int i = 0; i < n; ++i) {
        x[i] = Dual(pos[i], dpos ? dpos[i] : 0.0);
        y[i] = Dual(pos[n + i], dpos ? dpos[n + i] : 0.0);
        u[i] = Dual(vel[i], dvel ? dvel[i] : 0.0);
        v[i] = Dual(vel[n + i], dvel ? dvel[n + i] : 0.0);
        r[i] = Dual(rho[i], drho ? drho[i] : 0.0);
    }
    std::vector<Dual> st[5];
    int rc = run<Dual>(*cfg, n, x.data(), y.data(), u.data(), v.data(), r.data(), mass, type, Dual(cfg->nu, dnu),
                       nsteps, dt, st);
    if (rc) return rc;
    Dual L(0.0, 0.0);
    for (int i = 0; i < n; ++i) {
        if (type[i] != SPH_TYPE_WATER) continue;
        if (loss == SPH_LOSS_VELOCITY_MISFIT) {
            const Dual a = st[2][i] - target_vel[i], b = st[3][i] - target_vel[n + i];
            L += a * a + b * b;
        } else {
            L += 0.5 * mass[i] * (st[2][i] * st[2][i] + st[3][i] * st[3][i]);
        }
    }
    out[0] = L.v;
    out[1] = L.d;
    for (int i = 0; i < n; ++i) {
        if (pos_out) { pos_out[i] = st[0][i].v; pos_out[n + i] = st[1][i].v; }
        if (vel_out) { vel_out[i] = st[2][i].v; vel_out[n + i] = st[3][i].v; }
        if (rho_out) rho_out[i] = st[4][i].v;
    }
    return SPH_OK;
}

// The moving-square tangent-linear model: nsteps steps from (pos, vel, rho) at
// time t0 with the initial types, wall labels and per-step body motion
// (motion[4*nsteps]), along the direction (dpos, dvel, drho, dnu, dmotion) (any
// array may be NULL = zero).  out[0] = loss (SPH_LOSS_KINETIC_ENERGY,
// SPH_LOSS_VELOCITY_MISFIT or SPH_LOSS_DRAG), out[1] = its directional derivative.
int oracle_tangent_ms(const sph_config* cfg, int n, const double* pos, const double* vel, const double* rho,
                      const double* mass, const int* type, const int* itype, const int* labels, double t0,
                      int nsteps, double dt, const double* motion, int loss, const double* target_vel,
                      const double* dpos, const double* dvel, const double* drho, double dnu, const double* dmotion,
                      double* out) {
    if (!cfg || !pos || !vel || !rho || !mass || !type || !itype || !motion || !out || n <= 0 || nsteps <= 0)
        return SPH_E_ARG;
    if ((cfg->solver != SPH_SOLVER_MS_MODLR_DELTA && cfg->solver != SPH_SOLVER_MS_HLLC_DELTA) ||
        cfg->integrator != SPH_INTEGRATOR_EULER_PC || (cfg->shifting && cfg->shift_n != 4) ||
        cfg->laplacian != 1 || cfg->free_surface || cfg->periodic)
        return SPH_E_CONFIG;
    for (int i = 0; i < n; ++i)
        if (type[i] <= SPH_TYPE_INLET) return SPH_E_CONFIG;
    if (loss == SPH_LOSS_VELOCITY_MISFIT && !target_vel) return SPH_E_ARG;
    MSParts<Dual> H;
    H.n = n;
    for (int i = 0; i < n; ++i) {
        H.x.push_back(Dual(pos[i], dpos ? dpos[i] : 0.0));
        H.y.push_back(Dual(pos[n + i], dpos ? dpos[n + i] : 0.0));
        H.u.push_back(Dual(vel[i], dvel ? dvel[i] : 0.0));
        H.v.push_back(Dual(vel[n + i], dvel ? dvel[n + i] : 0.0));
        H.rho.push_back(Dual(rho[i], drho ? drho[i] : 0.0));
        H.mass.push_back(Dual(mass[i], 0.0));
        H.type.push_back(type[i]);
        H.itype.push_back(itype[i]);
        H.label.push_back(labels ? labels[i] : 0);
    }
    std::vector<Dual> mo(4 * (size_t)nsteps);
    for (size_t k = 0; k < mo.size(); ++k) mo[k] = Dual(motion[k], dmotion ? dmotion[k] : 0.0);
    Dual drag;
    int rc = run_ms<Dual>(*cfg, H, Dual(cfg->nu, dnu), mo, t0, nsteps, dt, drag);
    if (rc) return rc;
    Dual L(0.0, 0.0);
    if (loss == SPH_LOSS_DRAG) {
        L = drag;
    } else {
        for (int i = 0; i < n; ++i) {
            if (type[i] != SPH_TYPE_WATER) continue;
            if (loss == SPH_LOSS_VELOCITY_MISFIT) {
                const Dual a = H.u[i] - target_vel[i], b = H.v[i] - target_vel[n + i];
                L += a * a + b * b;
            } else {
                L += 0.5 * mass[i] * (H.u[i] * H.u[i] + H.v[i] * H.v[i]);
            }
        }
    }
    out[0] = L.v;
    out[1] = L.d;
    return SPH_OK;
}

}  // extern "C"
