// adjoint.cuh -- reverse kernels of the discrete adjoint of one time step.
//
// The forward RHS of the normalised modified linear Riemann delta-SPH + SPS
// solver (pass A, pass C; Solver_Normalized_Modified_Linear_Riemann_Delta_SPS.f90)
// is differentiated by hand, in FP64, for a pair set held fixed.  Written with
// r = x_a - x_b, d = |r|, grad_a W_ab = G(d) r and n = B_a^-1 r, the
// contribution of neighbour b to particle a is orientation-free:
//
//   w      = (u_a - u_b)/2 + (p_a - p_b) r / (2 rbar c0 d)          (not near a surface)
//   P*     = pbar + bR rbar dU / 2,  dU = -(u_a - u_b).r/d,  bR = min(3 max(dU,0), cbar)
//   drho_a += 2 rho_a V_b G (w.n) + 2 delta h cbar V_b psi (-G r.n/d^2),
//             psi = -(rho_a - rho_b) + (grad rho_a + grad rho_b).r/2
//   acc_a  += C G n + 2 nu V_b G (r.n)/d^2 (u_a - u_b) + SPS(tau_a + tau_b),
//             C = -2 P* m_b/(rho_a rho_b) - [v.r<0] m_b Pi_ab + delta_alpha h rho0 cbar (v.r) V_b/(d^2 rho_a)
//
// (the same terms pass C evaluates in the reference's pair orientation).  The
// reverse kernels are gathers over the pair list of the RHS being reversed:
// thread c adds the derivative of its own sum with respect to its own inputs
// and the derivative of each neighbour's sum with respect to c's inputs, so no
// atomics are needed and the result does not depend on thread timing.
//
//   k_adj_c     reverse of pass C: adjoints of x, u, rho (with p(rho), c(rho),
//               V = m/rho folded in), of B^-1, grad rho and tau; dL/dnu partials
//   k_adj_point reverse of tau = SPS(grad u, grad v, rho) and of grad = B^-1 g,
//               B^-1 = inv(B): the adjoints mu of the raw gradient sums and M of B
//   k_adj_a     reverse of the raw sums g = sum (phi_b - phi_a) V_b G r and
//               B = -sum V_b G r r^T of pass A, fused with the reverse of the
//               RK4 stage that produced the state (stage_reverse)
//   k_adj_stage3 reverse of the step end, with the reused K1
#pragma once
#include "update.cuh"

namespace sph {

// Device arrays of the adjoint (sorted slots unless noted).
struct Adj {
    double* lr[4];       // adjoint of drho/dt of the k-th RHS of the step (K1..K4)
    double2* la[4];      // adjoint of the acceleration of the k-th RHS
    double2* lxe;        // adjoint of the step-end position
    double2* ax0;        // adjoint of the step-start state: position,
    double2* av0;        //   velocity,
    double* ar0;         //   density
    double2* sx;         // adjoint of the state the reversed RHS was evaluated on
    double2* su;
    double* sr;
    double4* gbinv;      // adjoint of B^-1 (11, 12, 21, 22)
    double2* ggr;        // adjoint of grad rho
    double4* gtau;       // adjoint of tau (xx, xy, yy, -)
    double4* mu1;        // adjoint of the raw sums: (g_rho x, y, g_u x, y)
    double4* mu2;        //   (g_v x, y, B 11, B 12)
    double2* mu3;        //   (B 21, B 22)
    double* nu_part;     // per-block partial sums of dL/dnu, one block of slots per RHS of the step
    double* nu_acc;      // [1] dL/dnu
    double* irho;        // 1/rho of the state the reversed RHS was evaluated on (k_adj_c)
    // MUSCL: adjoints of the normalised grad p, u, v from the pass C reverse, and
    // the multipliers of pass A's raw grad p sums
    double2* ggp;
    double2* ggu;
    double2* ggv;
    double2* mu4;
    // particle shifting of the step end (last RHS of a step)
    double2* ssum;       // the shifting sum s = sum_b (1 + R (W/W_dx)^4) V_b G r, recomputed
    double2* smu;        // its adjoint
    double2* shgr;       // adjoint of grad rho from the density correction
    double4* shbi;       // adjoint of B^-1 from delta = -beta h^2 B^-1 s
    // id order, n_host + images: adjoint of the step-start state carried from
    // step to step, and (host particles) of the rates reused as K1
    double2* lx;
    double2* lv;
    double* lrho;
    double* lk_r;
    double2* lk_a;
    // moving-square path (Euler predictor-corrector, ghost assignment)
    double2* lg[2];      // adjoint of the XSPH velocity of RHS k of the step
    double2* lk_g;       // id order: of the carried XSPH velocity
    double2* gavg;       // adjoint of avg from the pass C reverse
    double* sm;          // adjoint of the mass of the state the reversed RHS was evaluated on
    double4* glam;       // ghost Shepard multipliers (p, u, v, m) / sum W
    double* glamw;       //   and of the normalisation
    double4* gint;       // the forward's interpolated ghost (p, u, v, m) of the reversed RHS
    double* gsw;         //   and its weight sum sum W V
    double* mo_part;     // per-block partials of the body-motion adjoints
    double* g_motion;    // [4 nsteps] dL/d(body velocity, body acceleration) of each step
};

constexpr int kAdjThreads = 128;

// G(d) of grad_a W = G(d) (x_a - x_b) and dG/dd.
// Gaussian: G = -2 k exp(-q^2)/h^2; Wendland C2: G = -5 k (1 - q/2)^3 / h^2.
// (1/h is loop-invariant: the compiler hoists it out of the pair loops.)
__device__ __forceinline__ void kernel_g(const Params& P, double d, double& G, double& dG) {
    const double ih = 1.0 / P.h, q = d * ih, kf = P.kfactor, ih2 = ih * ih;
    if (P.kernel_model == SPH_KERNEL_GAUSSIAN) {
        const double ex = exp(-(q * q));
        G = -2.0 * kf * ex * ih2;
        dG = 4.0 * kf * q * ex * (ih2 * ih);
    } else {
        const double t = 1.0 - 0.5 * q;
        G = -5.0 * kf * t * t * t * ih2;
        dG = 7.5 * kf * t * t * (ih2 * ih);
    }
}

// kernel_g and the kernel value W(d) of compute_kernel (whose d-derivative is
// G(d) d) from one exponential.
__device__ __forceinline__ void kernel_gw(const Params& P, double d, double& G, double& dG, double& W) {
    const double ih = 1.0 / P.h, q = d * ih, kf = P.kfactor, ih2 = ih * ih;
    if (P.kernel_model == SPH_KERNEL_GAUSSIAN) {
        const double ex = exp(-(q * q));
        G = -2.0 * kf * ex * ih2;
        dG = 4.0 * kf * q * ex * (ih2 * ih);
        W = (ex - P.gauss_e9) * kf;
    } else {
        const double t = 1.0 - 0.5 * q;
        const double t2 = t * t;
        G = -5.0 * kf * t2 * t * ih2;
        dG = 7.5 * kf * t2 * (ih2 * ih);
        W = kf * (1.0 + 2.0 * q) * (t2 * t2);
    }
}

// dp/drho and dc/drho of eos64.
__device__ __forceinline__ void eos_deriv(const Params& P, double rho, double& dp, double& dc) {
    const double r = rho / P.rho0;
    if (P.eos == SPH_EOS_TAIT) dp = 7.0 * P.eos_b * pw3(r) * pw3(r) / P.rho0;
    else dp = P.c0sq;
    dc = 3.0 * P.sqrt_c0 * r * r / P.rho0;
}

// One particle's inputs to a pair term.
struct PSide {
    double2 x;
    double u, v, rho, p, c, V, m, sm;
    double ir;            // 1 / rho
    double t0, t1, t2;    // tau xx, xy, yy
    double g0, g1;        // grad rho
    double ax, ay;        // XSPH average velocity (moving-square solver)
    double gp0, gp1, gu0, gu1, gv0, gv1;   // normalised grad p, u, v (MUSCL)
    double4 bi;           // B^-1
    bool water, near;
};

template <typename R, bool MS = false, bool MUSCL = false>
__device__ __forceinline__ PSide load_side(const Sorted<R>& D, int s) {
    PSide o;
    o.x = D.pos[s];
    const double4 k = D.kin[s];
    o.u = k.x; o.v = k.y; o.rho = k.z; o.p = k.w;
    const typename VT<R>::V4 ax = D.aux[s];
    o.m = D.mass[s];
    o.ir = 1.0 / o.rho;
    o.V = o.m * o.ir;
    o.c = (double)ax.z;
    o.sm = (double)ax.w;
    const typename VT<R>::V4 n1 = D.nb1[s];
    const double gs = grad_scale<R>();
    o.t0 = (double)n1.x; o.t1 = (double)n1.y; o.t2 = (double)n1.z; o.g0 = gs * n1.w;
    o.g1 = gs * D.nb2[s].x;
    o.bi = D.binv64[s];
    o.water = D.type[s] == SPH_TYPE_WATER;
    o.near = (D.flags[s] & 2) != 0;
    o.ax = o.ay = 0.0;
    o.gp0 = o.gp1 = o.gu0 = o.gu1 = o.gv0 = o.gv1 = 0.0;
    if (MUSCL) {
        // nb2 = (grad rho y, grad p x, grad p y, grad u x), nb3 = (grad u y, grad v x, grad v y, .)
        const typename VT<R>::V4 n2 = D.nb2[s], n3 = D.nb3[s];
        o.gp0 = gs * n2.y; o.gp1 = gs * n2.z; o.gu0 = gs * n2.w; o.gu1 = gs * n3.x;
        o.gv0 = gs * n3.y; o.gv1 = gs * n3.z;
    }
    if (MS) {
        const typename VT<R>::V2 g = D.avg[s];
        o.ax = (double)g.x; o.ay = (double)g.y;
    }
    return o;
}

// Adjoints of one pair term's inputs.  x: d/dx_a (d/dx_b is its negative);
// u, v: d/du_a (d/du_b is the negative); tau, grad rho: of the pair sums
// tau_a + tau_b and grad rho_a + grad rho_b.
struct PBar {
    double x0, x1, u, v;
    double pa, pb, ca, cb, ra, rb, Vb;
    double t0, t1, t2, g0, g1;
    double bi0, bi1, bi2, bi3;
    double nu;
    double avg0, avg1;    // of avg_a - avg_b (MS)
    double mb;            // of m_b (explicit; V_b = m_b/rho_b is in Vb)
    // MUSCL: of the normalised grad p, u, v of a and of b
    double gpa0, gpa1, gua0, gua1, gva0, gva1, gpb0, gpb1, gub0, gub1, gvb0, gvb1;
};

// Reverse of muscl_limiter on the branch the forward took: lim is one of 0,
// 1.3 di, dj, di, 1.3 dj (the min / max chain), or the large-jump branch gives
// dij/2 to one side.  From the adjoints (lib, ljb) of (li, lj), the adjoints of
// (di, dj, dij).
__device__ __forceinline__ void muscl_limiter_rev(double di, double dj, double dij, double lib, double ljb,
                                                  double& dib, double& djb, double& dijb) {
    const double b = 1.3, bdi = b * di, bdj = b * dj;
    const bool pos = dj > 0.0;
    double lim, cdi = 0.0, cdj = 0.0;            // lim = cdi di + cdj dj on the taken branch
    if (pos) {
        // max(0, max(min(bdi, dj), min(di, bdj)))
        const bool m1a = bdi <= dj;
        const double m1 = m1a ? bdi : dj, m1i = m1a ? b : 0.0, m1j = m1a ? 0.0 : 1.0;
        const bool m2a = di <= bdj;
        const double m2 = m2a ? di : bdj, m2i = m2a ? 1.0 : 0.0, m2j = m2a ? 0.0 : b;
        const bool mm1 = m1 >= m2;
        const double mm = mm1 ? m1 : m2;
        lim = mm > 0.0 ? mm : 0.0;
        if (mm > 0.0) { cdi = mm1 ? m1i : m2i; cdj = mm1 ? m1j : m2j; }
    } else {
        // min(0, min(max(bdi, dj), max(di, bdj)))
        const bool m1a = bdi >= dj;
        const double m1 = m1a ? bdi : dj, m1i = m1a ? b : 0.0, m1j = m1a ? 0.0 : 1.0;
        const bool m2a = di >= bdj;
        const double m2 = m2a ? di : bdj, m2i = m2a ? 1.0 : 0.0, m2j = m2a ? 0.0 : b;
        const bool mm1 = m1 <= m2;
        const double mm = mm1 ? m1 : m2;
        lim = mm < 0.0 ? mm : 0.0;
        if (mm < 0.0) { cdi = mm1 ? m1i : m2i; cdj = mm1 ? m1j : m2j; }
    }
    const double half = 0.5 * dij;
    const bool big = (pos ? (lim > half) : (lim < half)) && fabs(lim) > 0.0;
    dib = djb = dijb = 0.0;
    if (big) {
        const bool first = pos ? (di > dj) : (di < dj);
        dijb = 0.5 * (first ? lib : ljb);
    } else {
        const double l = lib + ljb;
        dib = cdi * l; djb = cdj * l;
    }
}

// Reverse of the contribution of b to particle a (a water particle) with the
// adjoints lr (of drho_a) and (l0, l1) (of acc_a).  MS: the moving-square
// solvers (Moving_Square.../Solver_Normalized_Modified_Linear_Riemann_Delta.f90
// :169-230, and with P.hllc Solver_Normalized_HLLC_Riemann_Delta.f90:207-322):
// w also carries avg_a - avg_b (XSPH inside the continuity flux), no SPS.
// MUSCL: the MUSCL linear-Riemann solver (Solver_Normalized_MUSCL_Linear_Riemann_Delta_SPS.f90:
// 470-502): the limited reconstructions of p, u, v enter U_L - U_R, P_L - P_R and
// this side's v - v*; a_lower: a is the reference's pair index i (the lower id),
// which fixes the limiter's sides.
template <bool MS = false, bool MUSCL = false, bool HLLC = false>
__device__ __forceinline__ void rev_pair(const Params& P, const PSide& A, const PSide& B, double lr, double l0,
                                         double l1, PBar& o, bool a_lower = true) {
    const double r0 = A.x.x - B.x.x, r1 = A.x.y - B.x.y;
    const double d2 = r0 * r0 + r1 * r1, d = sqrt(d2), id = 1.0 / d, id2 = id * id;
    double G, dG;
    kernel_g(P, d, G, dG);
    const double n0 = A.bi.x * r0 + A.bi.y * r1, n1 = A.bi.z * r0 + A.bi.w * r1;
    const double s = r0 * n0 + r1 * n1;
    const double du0 = A.u - B.u, du1 = A.v - B.v, dp = A.p - B.p, drho = A.rho - B.rho;
    const double vx = du0 * r0 + du1 * r1;
    // MUSCL reconstruction increments on the reference's i / j sides
    const double sI = a_lower ? 1.0 : -1.0;
    double lpi = 0, lpj = 0, lui = 0, luj = 0, lvi = 0, lvj = 0;
    double xj0 = 0, xj1 = 0, dpi = 0, dpj = 0, dui = 0, duj = 0, dvi = 0, dvj = 0;
    double gIp0 = 0, gIp1 = 0, gJp0 = 0, gJp1 = 0, gIu0 = 0, gIu1 = 0, gJu0 = 0, gJu1 = 0;
    double gIv0 = 0, gIv1 = 0, gJv0 = 0, gJv1 = 0;
    if (MUSCL) {
        xj0 = -sI * r0; xj1 = -sI * r1;                       // x_j - x_i
        gIp0 = a_lower ? A.gp0 : B.gp0; gIp1 = a_lower ? A.gp1 : B.gp1;
        gJp0 = a_lower ? B.gp0 : A.gp0; gJp1 = a_lower ? B.gp1 : A.gp1;
        gIu0 = a_lower ? A.gu0 : B.gu0; gIu1 = a_lower ? A.gu1 : B.gu1;
        gJu0 = a_lower ? B.gu0 : A.gu0; gJu1 = a_lower ? B.gu1 : A.gu1;
        gIv0 = a_lower ? A.gv0 : B.gv0; gIv1 = a_lower ? A.gv1 : B.gv1;
        gJv0 = a_lower ? B.gv0 : A.gv0; gJv1 = a_lower ? B.gv1 : A.gv1;
        dpi = 0.5 * (gIp0 * xj0 + gIp1 * xj1); dpj = -0.5 * (gJp0 * xj0 + gJp1 * xj1);
        dui = 0.5 * (gIu0 * xj0 + gIu1 * xj1); duj = -0.5 * (gJu0 * xj0 + gJu1 * xj1);
        dvi = 0.5 * (gIv0 * xj0 + gIv1 * xj1); dvj = -0.5 * (gJv0 * xj0 + gJv1 * xj1);
        muscl_limiter<double>(dpi, dpj, -sI * dp, lpi, lpj);
        muscl_limiter<double>(dui, duj, -sI * du0, lui, luj);
        muscl_limiter<double>(dvi, dvj, -sI * du1, lvi, lvj);
    }
    const double Su = lui + luj, Sv = lvi + lvj, Sp = lpi + lpj;
    // U_L - U_R = -(v_a - v_b + sI (l_i + l_j)).r / d
    const double vxm = MUSCL ? (du0 + sI * Su) * r0 + (du1 + sI * Sv) * r1 : vx;
    const double dU = -vxm * id;
    const double rbar = 0.5 * (A.rho + B.rho), cbar = 0.5 * (A.c + B.c);
    const double irbar = 1.0 / rbar, ic0 = 1.0 / P.sqrt_c0;
    const double Pbar = 0.5 * (A.p + B.p);
    // Riemann state
    double PA, w0, w1, bR = 0.0, kk = 0.0;
    bool take_m3 = false;
    // this side's reconstruction increment: + l_i as i, - l_j as j
    const double su = MUSCL ? (a_lower ? lui : -luj) : 0.0, sv = MUSCL ? (a_lower ? lvi : -lvj) : 0.0;
    // HLLC (moving-square solver, Moving_Square.../Solver_Normalized_HLLC_Riemann_Delta.f90:
    // 207-322), written in differences: with the pair frame e = (x_j - x_i)/d,
    // t = (-e1, e0), dV = VR0 - VL0 = (u_a - u_b).r/d and tdv = VR1 - VL1 =
    // (r0 (v_a - v_b) - r1 (u_a - u_b))/d (both independent of the orientation),
    // C_K = rho_K c_K, the contact speed U* = (VR0 C_L + VL0 C_R + P_L - P_R)/(C_L + C_R):
    //   sL = U* - VL0 = (C_L dV + dp_ij)/(C_L + C_R), sR = U* - VR0 = (dp_ij - C_R dV)/(C_L + C_R);
    // the state sampled at the mean normal velocity in one of four regions (taken
    // as the forward took it; the shock factor is 1, its branch being unreachable
    // when the pressure follows the density), rho_HLLC - rho0 = rho_K - rho0
    // [+ rho_K (U* - V_K0)/(S_K - U*)], and v_a - v* = al e + be t.
    const bool hllc = MS && HLLC && !A.near;
    const double sIh = a_lower ? 1.0 : -1.0;
    double hdVh = 0, htdv = 0, hrL = 0, hrR = 0, hcL = 0, hcR = 0, hCL = 0, hCR = 0, hiC = 0, hsL = 0, hsR = 0;
    double hal = 0, hbe = 0, he0 = 0, he1 = 0;
    int hreg = 0;
    if (hllc) {
        hdVh = vx * id;
        htdv = (r0 * du1 - r1 * du0) * id;
        const double dpp = sIh * dp;
        hrL = a_lower ? A.rho : B.rho; hrR = a_lower ? B.rho : A.rho;
        hcL = a_lower ? A.c : B.c; hcR = a_lower ? B.c : A.c;
        hCL = hrL * hcL; hCR = hrR * hcR; hiC = 1.0 / (hCL + hCR);
        hsL = (hCL * hdVh + dpp) * hiC;
        hsR = (dpp - hCR * hdVh) * hiC;
        const double hh = 0.5 * hdVh;
        hreg = (-hcL > hh) ? 0 : (hsL - hh >= 0.0 && hh >= -hcL) ? 1 : (hcR >= -hh && hsL - hh <= 0.0) ? 2 : 3;
        double dH, aI, bI, aJ, bJ;
        if (hreg == 0) { dH = hrL - P.rho0; aI = 0.0; bI = 0.0; aJ = hdVh; bJ = htdv; }
        else if (hreg == 1) { dH = hrL - P.rho0 + hrL * hsL / (-hcL - hsL); aI = -hsL; bI = 0.0; aJ = -hsR; bJ = htdv; }
        else if (hreg == 2) { dH = hrR - P.rho0 + hrR * hsR / (hcR - hsR); aI = -hsL; bI = -htdv; aJ = -hsR; bJ = 0.0; }
        else { dH = hrR - P.rho0; aI = -hdVh; bI = -htdv; aJ = 0.0; bJ = 0.0; }
        hal = a_lower ? aI : aJ; hbe = a_lower ? bI : bJ;
        he0 = -sIh * r0 * id; he1 = -sIh * r1 * id;
        PA = P.c0sq * dH + P.pb;
        w0 = hal * he0 - hbe * he1;
        w1 = hal * he1 + hbe * he0;
    } else if (A.near || P.dsph) {
        // the pair-mean state: near the free surface, and for every pair of the
        // plain delta-SPH method (Solver_Normalized_Delta_SPH_SPS.f90:335-374)
        PA = Pbar; w0 = 0.5 * du0 + su; w1 = 0.5 * du1 + sv;
    } else {
        const double m3 = 3.0 * fmax(dU, 0.0);
        take_m3 = m3 < cbar;
        bR = take_m3 ? m3 : cbar;
        PA = Pbar + 0.5 * bR * rbar * dU;
        kk = (MUSCL ? dp + sI * Sp : dp) * (0.5 * irbar * ic0) * id;
        w0 = 0.5 * du0 + su + kk * r0; w1 = 0.5 * du1 + sv + kk * r1;
    }
    if (MS) { w0 += A.ax - B.ax; w1 += A.ay - B.ay; }
    const double rhoij = A.ir * B.ir;
    const double fp = -2.0 * PA * B.m * rhoij;
    const bool av = vx < 0.0;
    const double fh2 = (P.fai * P.h) * (P.fai * P.h);
    const double den_phi = d2 + fh2;
    double phi = 0.0, Pi = 0.0, iden = 0.0;
    if (av) {
        iden = 1.0 / den_phi;
        phi = P.h * vx * iden;
        Pi = (-P.alpha * cbar * phi + P.beta * (phi * phi)) * irbar;
    }
    const double Kt = P.delta_alpha * P.h * P.rho0;
    const double tt = Kt * cbar * vx * id2 * A.ir * B.V;
    const double Cn = fp - (av ? B.m * Pi : 0.0) + tt;
    const double lf = 2.0 * P.nu * B.V * G * s * id2;
    const double Ln = l0 * n0 + l1 * n1;

    double Gb = 0, n0b = 0, n1b = 0, sb = 0, db = 0, r0b = 0, r1b = 0;
    double du0b = 0, du1b = 0, dpb = 0, rab = 0, rbb = 0, Pbarb = 0, rbarb = 0, cbarb = 0, Vbb = 0, vxb = 0, dUb = 0;
    o.t0 = o.t1 = o.t2 = o.g0 = o.g1 = 0.0;
    // acc = Cn G n + lf (u_a - u_b) + SPS
    const double Cnb = G * Ln;
    o.mb = Cnb * (-2.0 * PA * rhoij - (av ? Pi : 0.0));
    Gb += Cn * Ln;
    n0b += Cn * G * l0; n1b += Cn * G * l1;
    const double lfb = l0 * du0 + l1 * du1;
    du0b += lf * l0; du1b += lf * l1;
    if (!MS) {
        // SPS: acc_x += sm rho_ij G Q, acc_y += sm rho_ij G (q rho_ij Q + Rr), q = 1 with the
        // reference's temp_p carry-over
        const double sxx = A.t0 + B.t0, sxy = A.t1 + B.t1, syy = A.t2 + B.t2;
        const double Q = sxx * r0 + sxy * r1, Rr = syy * r1 + sxy * r0;
        const double q = P.quirks ? 1.0 : 0.0;
        const double cx = rhoij * (l0 + q * rhoij * l1), cy = rhoij * l1;
        Gb += B.sm * (cx * Q + cy * Rr);
        const double Qb = B.sm * G * cx, Rb = B.sm * G * cy;
        const double rhoijb = B.sm * G * (l0 * Q + l1 * (2.0 * q * rhoij * Q + Rr));
        o.t0 = Qb * r0; o.t1 = Qb * r1 + Rb * r0; o.t2 = Rb * r1;
        r0b += Qb * sxx + Rb * sxy; r1b += Qb * sxy + Rb * syy;
        rab -= rhoijb * rhoij * A.ir; rbb -= rhoijb * rhoij * B.ir;
    }
    // C = fp - [av] m_b Pi + tt
    const double PAb0 = -2.0 * B.m * rhoij * Cnb;
    rab -= fp * A.ir * Cnb; rbb -= fp * B.ir * Cnb;
    if (av) {
        const double Pib = -B.m * Cnb;
        cbarb += -P.alpha * phi * irbar * Pib;
        const double phib = (-P.alpha * cbar + 2.0 * P.beta * phi) * irbar * Pib;
        rbarb -= Pi * irbar * Pib;
        vxb += P.h * iden * phib;
        db -= phi * 2.0 * d * iden * phib;
    }
    {
        const double base = Kt * id2 * A.ir;
        cbarb += base * vx * B.V * Cnb;
        vxb += base * cbar * B.V * Cnb;
        Vbb += base * cbar * vx * Cnb;
        db -= 2.0 * tt * id * Cnb;
        rab -= tt * A.ir * Cnb;
    }
    // Morris laplacian factor lf = 2 nu V_b G s / d^2
    o.nu = 2.0 * B.V * G * s * id2 * lfb;
    Vbb += 2.0 * P.nu * G * s * id2 * lfb;
    Gb += 2.0 * P.nu * B.V * s * id2 * lfb;
    sb += 2.0 * P.nu * B.V * G * id2 * lfb;
    db -= 2.0 * lf * id * lfb;
    // continuity and delta-SPH
    double w0b = 0.0, w1b = 0.0;
    if (lr != 0.0) {
        const double WN = w0 * n0 + w1 * n1;
        const double k2 = 2.0 * A.rho * B.V * G * lr;
        rab += 2.0 * B.V * G * WN * lr;
        Vbb += 2.0 * A.rho * G * WN * lr;
        Gb += 2.0 * A.rho * B.V * WN * lr;
        w0b = k2 * n0; w1b = k2 * n1;
        n0b += k2 * w0; n1b += k2 * w1;
        if (A.water && P.dsph) {
            // Antuono form (Solver_Normalized_Delta_SPH_SPS.f90:610-636) in a's frame:
            // D_a += delta h cbar G V_b Y, Y = 2 (rho_a - rho_b) s/d^2 - (grad rho_a + grad rho_b).n
            const double K = P.delta * P.h * lr;
            const double sg0 = A.g0 + B.g0, sg1 = A.g1 + B.g1;
            const double Y = 2.0 * drho * s * id2 - (sg0 * n0 + sg1 * n1);
            cbarb += K * G * B.V * Y;
            Gb += K * cbar * B.V * Y;
            Vbb += K * cbar * G * Y;
            const double Yb = K * cbar * G * B.V;
            rab += 2.0 * s * id2 * Yb; rbb -= 2.0 * s * id2 * Yb;
            sb += 2.0 * drho * id2 * Yb;
            db -= 4.0 * drho * s * id2 * id * Yb;
            o.g0 = -n0 * Yb; o.g1 = -n1 * Yb;
            n0b -= sg0 * Yb; n1b -= sg1 * Yb;
        } else if (A.water) {
            const double T2 = 2.0 * P.delta * P.h * lr;
            const double sg0 = A.g0 + B.g0, sg1 = A.g1 + B.g1;
            const double psi = -drho + 0.5 * (sg0 * r0 + sg1 * r1);
            const double X = -G * s * id2;
            cbarb += T2 * psi * X * B.V;
            const double psib = T2 * cbar * X * B.V;
            const double Xb = T2 * cbar * psi * B.V;
            Vbb += T2 * cbar * psi * X;
            Gb -= s * id2 * Xb; sb -= G * id2 * Xb; db -= 2.0 * X * id * Xb;
            rab -= psib; rbb += psib;
            o.g0 = 0.5 * psib * r0; o.g1 = 0.5 * psib * r1;
            r0b += 0.5 * psib * sg0; r1b += 0.5 * psib * sg1;
        }
    }
    if (!hllc) { du0b += 0.5 * w0b; du1b += 0.5 * w1b; }
    o.avg0 = w0b; o.avg1 = w1b;
    double luib = 0, lujb = 0, lvib = 0, lvjb = 0, Spb = 0, Sub = 0, Svb = 0;
    if (MUSCL) {
        if (a_lower) { luib += w0b; lvib += w1b; } else { lujb -= w0b; lvjb -= w1b; }
    }
    double hcab = 0.0, hcbb = 0.0;
    if (hllc) {
        // reverse of the HLLC state above, region as taken
        const double dHb = P.c0sq * PAb0;
        const double alb = w0b * he0 + w1b * he1, beb = -w0b * he1 + w1b * he0;
        const double e0b = w0b * hal + w1b * hbe, e1b = -w0b * hbe + w1b * hal;
        double sLb = 0, sRb = 0, dVb = 0, tdvb = 0, rLb = 0, rRb = 0, cLb = 0, cRb = 0;
        if (hreg == 0) {
            rLb += dHb;
            if (!a_lower) { dVb += alb; tdvb += beb; }
        } else if (hreg == 1) {
            const double Dd = -hcL - hsL, iD2 = 1.0 / (Dd * Dd);
            rLb += dHb * (1.0 + hsL / Dd);
            sLb += dHb * hrL * (-hcL) * iD2;
            cLb += dHb * hrL * hsL * iD2;
            if (a_lower) sLb -= alb; else { sRb -= alb; tdvb += beb; }
        } else if (hreg == 2) {
            const double Dd = hcR - hsR, iD2 = 1.0 / (Dd * Dd);
            rRb += dHb * (1.0 + hsR / Dd);
            sRb += dHb * hrR * hcR * iD2;
            cRb -= dHb * hrR * hsR * iD2;
            if (a_lower) { sLb -= alb; tdvb -= beb; } else sRb -= alb;
        } else {
            rRb += dHb;
            if (a_lower) { dVb -= alb; tdvb -= beb; }
        }
        dVb += (sLb * hCL - sRb * hCR) * hiC;
        const double dppb = (sLb + sRb) * hiC;
        const double CLb = (sLb * (hdVh - hsL) - sRb * hsR) * hiC;
        const double CRb = (-sLb * hsL - sRb * (hdVh + hsR)) * hiC;
        rLb += CLb * hcL; cLb += CLb * hrL;
        rRb += CRb * hcR; cRb += CRb * hrR;
        dpb += sIh * dppb;
        vxb += dVb * id;
        db -= hdVh * id * dVb;
        du1b += tdvb * r0 * id; du0b -= tdvb * r1 * id;
        r0b += tdvb * du1 * id; r1b -= tdvb * du0 * id;
        db -= htdv * id * tdvb;
        r0b -= sIh * id * e0b; r1b -= sIh * id * e1b;
        db += sIh * (r0 * e0b + r1 * e1b) * id * id;
        if (a_lower) { rab += rLb; rbb += rRb; hcab = cLb; hcbb = cRb; }
        else { rab += rRb; rbb += rLb; hcab = cRb; hcbb = cLb; }
    } else {
        Pbarb += PAb0;
    }
    if (!A.near && !P.dsph && !hllc) {
        const double kkb = w0b * r0 + w1b * r1;
        r0b += kk * w0b; r1b += kk * w1b;
        dpb += kkb * (0.5 * irbar * ic0) * id;
        if (MUSCL) Spb += sI * kkb * (0.5 * irbar * ic0) * id;
        rbarb -= kk * irbar * kkb;
        db -= kk * id * kkb;
        const double bRb = 0.5 * rbar * dU * PAb0;
        rbarb += 0.5 * bR * dU * PAb0;
        dUb += 0.5 * bR * rbar * PAb0;
        if (take_m3) { if (dU > 0.0) dUb += 3.0 * bRb; }
        else cbarb += bRb;
    }
    // dU = -vxm/d
    {
        const double vxmb = -dUb * id;
        db += vxm * id2 * dUb;
        du0b += vxmb * r0; du1b += vxmb * r1;
        if (MUSCL) {
            r0b += vxmb * (du0 + sI * Su); r1b += vxmb * (du1 + sI * Sv);
            Sub += sI * vxmb * r0; Svb += sI * vxmb * r1;
        } else {
            r0b += vxmb * du0; r1b += vxmb * du1;
        }
    }
    // vx = (u_a - u_b).r (artificial viscosity, delta-alpha)
    du0b += vxb * r0; du1b += vxb * r1;
    r0b += vxb * du0; r1b += vxb * du1;
    if (MUSCL) {
        // the limiters: inputs di = (grad_i . x_ji)/2, dj = -(grad_j . x_ji)/2, dij = phi_j - phi_i
        const double lpib = Spb, lpjb = Spb;
        luib += Sub; lujb += Sub; lvib += Svb; lvjb += Svb;
        double dib, djb, dijb, xjb0 = 0.0, xjb1 = 0.0;
        double gIpb0, gIpb1, gJpb0, gJpb1, gIub0, gIub1, gJub0, gJub1, gIvb0, gIvb1, gJvb0, gJvb1;
        muscl_limiter_rev(dpi, dpj, -sI * dp, lpib, lpjb, dib, djb, dijb);
        dpb -= sI * dijb;
        gIpb0 = 0.5 * dib * xj0; gIpb1 = 0.5 * dib * xj1; gJpb0 = -0.5 * djb * xj0; gJpb1 = -0.5 * djb * xj1;
        xjb0 += 0.5 * dib * gIp0 - 0.5 * djb * gJp0; xjb1 += 0.5 * dib * gIp1 - 0.5 * djb * gJp1;
        muscl_limiter_rev(dui, duj, -sI * du0, luib, lujb, dib, djb, dijb);
        du0b -= sI * dijb;
        gIub0 = 0.5 * dib * xj0; gIub1 = 0.5 * dib * xj1; gJub0 = -0.5 * djb * xj0; gJub1 = -0.5 * djb * xj1;
        xjb0 += 0.5 * dib * gIu0 - 0.5 * djb * gJu0; xjb1 += 0.5 * dib * gIu1 - 0.5 * djb * gJu1;
        muscl_limiter_rev(dvi, dvj, -sI * du1, lvib, lvjb, dib, djb, dijb);
        du1b -= sI * dijb;
        gIvb0 = 0.5 * dib * xj0; gIvb1 = 0.5 * dib * xj1; gJvb0 = -0.5 * djb * xj0; gJvb1 = -0.5 * djb * xj1;
        xjb0 += 0.5 * dib * gIv0 - 0.5 * djb * gJv0; xjb1 += 0.5 * dib * gIv1 - 0.5 * djb * gJv1;
        r0b -= sI * xjb0; r1b -= sI * xjb1;                   // x_j - x_i = -sI r
        if (a_lower) {
            o.gpa0 = gIpb0; o.gpa1 = gIpb1; o.gua0 = gIub0; o.gua1 = gIub1; o.gva0 = gIvb0; o.gva1 = gIvb1;
            o.gpb0 = gJpb0; o.gpb1 = gJpb1; o.gub0 = gJub0; o.gub1 = gJub1; o.gvb0 = gJvb0; o.gvb1 = gJvb1;
        } else {
            o.gpa0 = gJpb0; o.gpa1 = gJpb1; o.gua0 = gJub0; o.gua1 = gJub1; o.gva0 = gJvb0; o.gva1 = gJvb1;
            o.gpb0 = gIpb0; o.gpb1 = gIpb1; o.gub0 = gIub0; o.gub1 = gIub1; o.gvb0 = gIvb0; o.gvb1 = gIvb1;
        }
    }
    // s = r.n, n = B^-1 r
    r0b += sb * n0; r1b += sb * n1;
    n0b += sb * r0; n1b += sb * r1;
    o.bi0 = n0b * r0; o.bi1 = n0b * r1; o.bi2 = n1b * r0; o.bi3 = n1b * r1;
    r0b += A.bi.x * n0b + A.bi.z * n1b;
    r1b += A.bi.y * n0b + A.bi.w * n1b;
    // G(d), d = |r|
    db += dG * Gb;
    r0b += db * r0 * id; r1b += db * r1 * id;
    o.x0 = r0b; o.x1 = r1b;
    o.u = du0b; o.v = du1b;
    o.pa = 0.5 * Pbarb + dpb; o.pb = 0.5 * Pbarb - dpb;
    o.ca = 0.5 * cbarb + hcab; o.cb = 0.5 * cbarb + hcbb;
    o.ra = rab + 0.5 * rbarb; o.rb = rbb + 0.5 * rbarb;
    o.Vb = Vbb;
}

// Reverse of pass C for the RHS whose rate adjoints are (lr, la).  Four
// consecutive lanes share a particle c: lane bit 0 picks the role (0: the
// derivative of c's own sum, 1: the derivatives of the neighbours' sums with
// respect to c's inputs), lane bit 1 the pairs (even or odd list positions).
// Each lane inlines one pair reverse, so the register count stays low and a
// small particle count still fills the GPU; the four partial sums are combined
// by shuffles in a fixed order.
#ifndef SPH_ADJ_LANES
#define SPH_ADJ_LANES 4
#endif
#ifndef SPH_ADJ_C_MIN_BLOCKS
#define SPH_ADJ_C_MIN_BLOCKS 3       // 168 registers: 3 blocks of 128 per SM
#endif
#ifndef SPH_ADJ_C_MUSCL_MIN_BLOCKS
#define SPH_ADJ_C_MUSCL_MIN_BLOCKS 2 // the limiter reverses need more than 168
#endif
constexpr int kAdjLanes = SPH_ADJ_LANES;     // 2 or 4
// HLLC: the moving-square HLLC solver (a variant of its own, so that the
// modified solver's reverse carries none of its registers).
template <typename R, bool MS = false, bool MUSCL = false, bool HLLC = false>
__global__ void __launch_bounds__(kAdjThreads, MUSCL ? SPH_ADJ_C_MUSCL_MIN_BLOCKS : SPH_ADJ_C_MIN_BLOCKS) k_adj_c(Params P, Sorted<R> D, Adj A, const double* lr,
                                                        const double2* la, double* nu_part) {
    __shared__ double red[kAdjThreads];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = t / kAdjLanes;
    const int role = t & 1, par = (t >> 1) & (kAdjLanes / 2 - 1);
    double nu_sum = 0.0;
    // every lane of the warp takes part in the shuffles below
    const bool live = c < P.n_tot;
    // 0-16 as below; MS: 17-18 avg, 19 mass; MUSCL: 17-22 grad p, u, v
    constexpr int NV = MS ? 20 : (MUSCL ? 23 : 17);
    double v[23];
#pragma unroll
    for (int q = 0; q < 23; ++q) v[q] = 0.0;
    if (live) {
        const int nn = D.npairs[c];
        // both roles run the same instructions: the two sides are loaded by
        // index (c's records stay in L1), not branched on
        const double sg = role ? -1.0 : 1.0;
        for (int e = par; e < nn; e += kAdjLanes / 2) {
            const unsigned ent = D.pairs[(size_t)e * P.nbr_stride + c];
            const int b = (int)(ent & 0x7fffffffu);
            const int acc_at = role ? b : c;         // the particle whose sum is differentiated
            const bool c_lower = (ent >> 31) != 0;  // c has the lower id of the pair
            const int other = role ? c : b;
            if (D.type[acc_at] != SPH_TYPE_WATER) continue;
            const double l_r = lr[acc_at];
            const double2 l_a = la[acc_at];
            if (l_r == 0.0 && l_a.x == 0.0 && l_a.y == 0.0) continue;
            const PSide Sa = load_side<R, MS, MUSCL>(D, acc_at);
            const PSide Sb = load_side<R, MS, MUSCL>(D, other);
            PBar o;
            rev_pair<MS, MUSCL, HLLC>(P, Sa, Sb, l_r, l_a.x, l_a.y, o, role ? !c_lower : c_lower);
            v[0] += sg * o.x0; v[1] += sg * o.x1; v[2] += sg * o.u; v[3] += sg * o.v;
            v[4] += role ? o.pb : o.pa;
            v[5] += role ? o.cb : o.ca;
            v[6] += role ? o.rb : o.ra;
            v[7] += role ? o.Vb : 0.0;
            v[8] += o.t0; v[9] += o.t1; v[10] += o.t2; v[11] += o.g0; v[12] += o.g1;
            if (!role) {
                v[13] += o.bi0; v[14] += o.bi1; v[15] += o.bi2; v[16] += o.bi3;
                nu_sum += o.nu;
            }
            if (MS) {
                v[17] += sg * o.avg0; v[18] += sg * o.avg1;
                v[19] += role ? o.mb : 0.0;
            }
            if (MUSCL) {
                v[17] += role ? o.gpb0 : o.gpa0; v[18] += role ? o.gpb1 : o.gpa1;
                v[19] += role ? o.gub0 : o.gua0; v[20] += role ? o.gub1 : o.gua1;
                v[21] += role ? o.gvb0 : o.gva0; v[22] += role ? o.gvb1 : o.gva1;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        v[q] += __shfl_xor_sync(0xffffffffu, v[q], 1);
        if (kAdjLanes == 4) v[q] += __shfl_xor_sync(0xffffffffu, v[q], 2);
    }
    if (live && (t & (kAdjLanes - 1)) == 0) {
        const double4 k = D.kin[c];
        const double rho = k.z, ir = 1.0 / rho, V = D.mass[c] * ir;
        A.irho[c] = ir;
        double dp, dc;
        eos_deriv(P, rho, dp, dc);
        A.sx[c] = make_double2(v[0], v[1]);
        A.su[c] = make_double2(v[2], v[3]);
        A.sr[c] = v[6] + dp * v[4] + dc * v[5] - V / rho * v[7];
        A.gbinv[c] = make_double4(v[13], v[14], v[15], v[16]);
        A.ggr[c] = make_double2(v[11], v[12]);
        A.gtau[c] = make_double4(v[8], v[9], v[10], 0.0);
        if (MS) {
            A.gavg[c] = make_double2(v[17], v[18]);
            A.sm[c] = v[19] + v[7] / rho;       // V = m / rho
        }
        if (MUSCL) {
            A.ggp[c] = make_double2(v[17], v[18]);
            A.ggu[c] = make_double2(v[19], v[20]);
            A.ggv[c] = make_double2(v[21], v[22]);
        }
    }
    red[threadIdx.x] = nu_sum;
    __syncthreads();
    for (int w = kAdjThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) nu_part[blockIdx.x] = red[0];
}

// dL/dnu += sum of the block partials, in block order.
// Sum over one block (any multiple of 32 threads up to 1024) in a fixed order:
// shuffles within each warp, then over the warp sums.  The result is in thread 0.
__device__ __forceinline__ double block_sum(double s, double* red32) {
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) red32[w] = s;
    __syncthreads();
    s = 0.0;
    if (w == 0) {
        s = lane < (int)(blockDim.x >> 5) ? red32[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    }
    __syncthreads();
    return s;
}

__global__ void k_adj_nu_sum(int nparts, const double* part, double* acc) {
    __shared__ double red[32];
    double s = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) s += part[i];
    s = block_sum(s, red);
    if (threadIdx.x == 0) acc[0] += s;
}

// Reverse of the per-particle end of pass A.  shift: the RHS is the last of a
// step with particle shifting, whose step-end reverse left adjoints of grad rho
// and B^-1 in shgr / shbi.
template <typename R>
__global__ void k_adj_point(Params P, Sorted<R> D, Adj A, int shift) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= P.n_tot) return;
    const int ta = D.type[a];
    const double4 bi = D.binv64[a];
    const typename VT<R>::V4 n1 = D.nb1[a], n2 = D.nb2[a], n3 = D.nb3[a];
    // normalised gradients of pass A: rho (n1.w, n2.x), u (n2.w, n3.x), v (n3.y, n3.z)
    const double gs = grad_scale<R>();
    const double gr0 = gs * n1.w, gr1 = gs * n2.x;
    const double gu0 = gs * n2.w, gu1 = gs * n3.x;
    const double gv0 = gs * n3.y, gv1 = gs * n3.z;
    double2 ggr = A.ggr[a];
    double4 gbs = make_double4(0, 0, 0, 0);
    if (shift) {
        const double2 sg = A.shgr[a];
        ggr.x += sg.x; ggr.y += sg.y;
        gbs = A.shbi[a];
    }
    double Gr0 = ggr.x, Gr1 = ggr.y, Gu0 = 0, Gu1 = 0, Gv0 = 0, Gv1 = 0, Gp0 = 0, Gp1 = 0;
    if (P.muscl) {
        const double2 gp = A.ggp[a], gu = A.ggu[a], gv = A.ggv[a];
        Gp0 = gp.x; Gp1 = gp.y; Gu0 = gu.x; Gu1 = gu.y; Gv0 = gv.x; Gv1 = gv.y;
    }
    double rho_b = 0.0;
    if (ta == SPH_TYPE_WATER && !P.ms) {
        // tau = SPS(grad u, grad v) rho (Solver_..._SPS.f90:256-296)
        const double4 T = A.gtau[a];
        const double rho = D.kin[a].z;
        const double sxx = gu0, sxy = gu1 + gv0, syy = gv1;
        const double abs2 = 2 * (sxx * sxx + syy * syy) + sxy * sxy;
        const double sq = sqrt(abs2);
        const double DL = P.sps_dl;
        const double t = P.sps_c012 * DL;
        const double nut = (t * t) * sq;
        const double kk = P.sps_23 * nut * (sxx + syy);
        const double blin = P.sps_blin * (DL * DL) * abs2;
        rho_b = T.x * (2 * nut * sxx - kk - blin) + T.y * (nut * sxy) + T.z * (2 * nut * syy - kk - blin);
        const double Axx = T.x * rho, Axy = T.y * rho, Ayy = T.z * rho;
        const double kkb = -(Axx + Ayy), blinb = -(Axx + Ayy);
        double sxxb = 2 * nut * Axx + P.sps_23 * nut * kkb;
        double syyb = 2 * nut * Ayy + P.sps_23 * nut * kkb;
        double sxyb = nut * Axy;
        const double nutb = 2 * sxx * Axx + sxy * Axy + 2 * syy * Ayy + P.sps_23 * (sxx + syy) * kkb;
        double abs2b = P.sps_blin * (DL * DL) * blinb;
        if (sq > 0.0) abs2b += (t * t) * nutb / (2.0 * sq);
        sxxb += 4 * sxx * abs2b; syyb += 4 * syy * abs2b; sxyb += 2 * sxy * abs2b;
        Gu0 += sxxb; Gu1 += sxyb; Gv0 += sxyb; Gv1 += syyb;
    }
    // grad = B^-1 g: adjoint of g = B^-T adjoint of grad
    auto mt = [&](double x, double y, double& ox, double& oy) {
        ox = bi.x * x + bi.z * y;
        oy = bi.y * x + bi.w * y;
    };
    double m0, m1, m2, m3, m4, m5, m6 = 0.0, m7 = 0.0;
    mt(Gr0, Gr1, m0, m1);
    mt(Gu0, Gu1, m2, m3);
    mt(Gv0, Gv1, m4, m5);
    if (P.muscl) mt(Gp0, Gp1, m6, m7);
    const double gp0n = (double)n2.y, gp1n = (double)n2.z;    // normalised grad p (MUSCL)
    double M00 = 0, M01 = 0, M10 = 0, M11 = 0;
    const bool inverted = (ta == SPH_TYPE_WATER || (P.ms && ta == -202)) && P.renorm &&
                          !(bi.x == 1.0 && bi.y == 0.0 && bi.z == 0.0 && bi.w == 1.0);
    if (inverted) {
        // raw sums g = B grad with B = inv(B^-1)
        const double det = bi.x * bi.w - bi.y * bi.z;
        const double B00 = bi.w / det, B01 = -bi.y / det, B10 = -bi.z / det, B11 = bi.x / det;
        auto raw = [&](double x, double y, double& ox, double& oy) {
            ox = B00 * x + B01 * y;
            oy = B10 * x + B11 * y;
        };
        double qr0, qr1, qu0, qu1, qv0, qv1, qp0 = 0.0, qp1 = 0.0;
        raw(gr0, gr1, qr0, qr1);
        raw(gu0, gu1, qu0, qu1);
        raw(gv0, gv1, qv0, qv1);
        if (P.muscl) raw(gp0n, gp1n, qp0, qp1);
        double4 gb = A.gbinv[a];
        gb.x += gbs.x; gb.y += gbs.y; gb.z += gbs.z; gb.w += gbs.w;
        // adjoint of B^-1: from pass C and from grad = B^-1 g
        const double Y00 = gb.x + Gr0 * qr0 + Gu0 * qu0 + Gv0 * qv0 + Gp0 * qp0;
        const double Y01 = gb.y + Gr0 * qr1 + Gu0 * qu1 + Gv0 * qv1 + Gp0 * qp1;
        const double Y10 = gb.z + Gr1 * qr0 + Gu1 * qu0 + Gv1 * qv0 + Gp1 * qp0;
        const double Y11 = gb.w + Gr1 * qr1 + Gu1 * qu1 + Gv1 * qv1 + Gp1 * qp1;
        // adjoint of B = -B^-T Y B^-T
        const double T00 = Y00 * bi.x + Y01 * bi.y, T01 = Y00 * bi.z + Y01 * bi.w;
        const double T10 = Y10 * bi.x + Y11 * bi.y, T11 = Y10 * bi.z + Y11 * bi.w;
        M00 = -(bi.x * T00 + bi.z * T10);
        M01 = -(bi.x * T01 + bi.z * T11);
        M10 = -(bi.y * T00 + bi.w * T10);
        M11 = -(bi.y * T01 + bi.w * T11);
    }
    A.mu1[a] = make_double4(m0, m1, m2, m3);
    A.mu2[a] = make_double4(m4, m5, M00, M01);
    A.mu3[a] = make_double2(M10, M11);
    if (P.muscl) A.mu4[a] = make_double2(m6, m7);
    A.sr[a] += rho_b;
}

// Reverse of stage k = 2, 1, 0:  x_k = x0 + f u_k, u_k = v0 + f a_k, rho_k = rho0 + f d_k
// (f = dt for k = 2, dt/2 otherwise); u_k also enters x' with weight dt/3 (k = 1, 2)
// or dt/6 (k = 0).  (sx, su, sr) is the adjoint of the state the RHS after stage k
// was evaluated on.  For k = -1 that state is the step-start state itself (the
// first step's fresh K1); so it is for particles the stages do not move.
template <typename R>
__device__ __forceinline__ void stage_reverse(const Params& P, const Sorted<R>& D, const Adj& A, int s, int k,
                                              double dt, double2 sx, double2 su, double sr) {
    double2 ax = A.ax0[s], av = A.av0[s];
    double ar = A.ar0[s];
    if (k >= 0 && D.id[s] < P.n_host && integrated(P, D.type[s])) {
        const double f = k == 2 ? dt : 0.5 * dt;
        const double w = k == 0 ? dt / 6.0 : dt / 3.0;
        const double2 le = A.lxe[s];
        const double lu0 = su.x + f * sx.x + w * le.x, lu1 = su.y + f * sx.y + w * le.y;
        ax.x += sx.x; ax.y += sx.y;
        av.x += lu0; av.y += lu1;
        ar += sr;
        const double2 la = A.la[k][s];
        A.la[k][s] = make_double2(la.x + f * lu0, la.y + f * lu1);
        A.lr[k][s] += f * sr;
    } else {
        ax.x += sx.x; ax.y += sx.y;
        av.x += su.x; av.y += su.y;
        ar += sr;
    }
    A.ax0[s] = ax; A.av0[s] = av; A.ar0[s] = ar;
}

// f = V_b G(d) [sum_phi (phi_b - phi_a) mu_phi.r - r^T M r]: the adjoint-weighted
// pair term of pass A's raw sums at particle a, with G = G(d), dG = G'(d),
// id = 1/|r|.  Returns f / V_b and its gradient with respect to r divided by V_b.
__device__ __forceinline__ void rev_rawsum(double r0, double r1, double id, double G, double dG, double dr,
                                           double du, double dv, const double4& m1, const double4& m2,
                                           const double2& m3, double& S_G, double& fr0, double& fr1,
                                           double dpp = 0.0, double2 m4 = make_double2(0.0, 0.0)) {
    // sum_phi dphi mu_phi; MUSCL adds the grad p sum (dpp, m4)
    const double c0 = dr * m1.x + du * m1.z + dv * m2.x + dpp * m4.x;
    const double c1 = dr * m1.y + du * m1.w + dv * m2.y + dpp * m4.y;
    const double Mr0 = m2.z * r0 + m2.w * r1, Mr1 = m3.x * r0 + m3.y * r1;
    const double MTr0 = m2.z * r0 + m3.x * r1, MTr1 = m2.w * r0 + m3.y * r1;
    const double S = c0 * r0 + c1 * r1 - (r0 * Mr0 + r1 * Mr1);
    S_G = S;
    const double k = dG * S * id;
    fr0 = k * r0 + G * (c0 - Mr0 - MTr0);
    fr1 = k * r1 + G * (c1 - Mr1 - MTr1);
}

// Reverse of pass A's raw pair sums, then of the stage that produced the
// state this RHS was evaluated on.  MS: also the reverse of the XSPH velocity
//   avg_a = eps sum_b m_b (v_b - v_a) W_ab / (rho_a + rho_b)
// (Moving_Square.../Solver_Normalized_Modified_Linear_Riemann_Delta.f90:114-121)
// with the adjoint lg + gavg of avg; the totals of the state adjoint (x, u, rho,
// m) are written to sx, su, sr, sm for the ghost reverse and the stage reverse
// that follow.
// MUSCL: also pass A's raw grad p sum, p = p(rho) by the equation of state.
// kAdjLanes lanes per particle: lane q takes pairs q, q + kAdjLanes, ...; the
// lanes' partial sums are added by shuffles in a fixed order.
template <typename R, bool MS = false, bool MUSCL = false>
__global__ void __launch_bounds__(kAdjThreads) k_adj_a(Params P, Sorted<R> D, Adj A, int stage, double dt,
                                                       const double2* lg) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int c0 = t / kAdjLanes, lane = t & (kAdjLanes - 1);
    // every lane of the warp takes part in the shuffles below
    const bool live = c0 < P.n_tot;
    const int c = live ? c0 : 0;
    const double2 xc = D.pos[c];
    const double4 kc = D.kin[c];
    const double mc = D.mass[c];
    const double Vc = mc / kc.z;
    const double4 mc1 = A.mu1[c], mc2 = A.mu2[c];
    const double2 mc3 = A.mu3[c];
    const double2 mc4 = MUSCL ? A.mu4[c] : make_double2(0.0, 0.0);
    double x0b = 0, x1b = 0, ub = 0, vb = 0, rb = 0, Vb = 0, mb_ = 0, pb_ = 0;
    double2 lac = make_double2(0.0, 0.0);
    if (MS) {
        const double2 g = A.gavg[c], l = lg[c];
        lac = make_double2(g.x + l.x, g.y + l.y);
    }
    const int nn = live ? D.npairs[c] : 0;
    for (int e = lane; e < nn; e += kAdjLanes) {
        const int b = (int)(D.pairs[(size_t)e * P.nbr_stride + c] & 0x7fffffffu);
        const double2 xb = D.pos[b];
        const double4 kb = D.kin[b];
        const double r0 = xc.x - xb.x, r1 = xc.y - xb.y;
        const double d = sqrt(r0 * r0 + r1 * r1), id = 1.0 / d;
        double G, dG, W;
        kernel_gw(P, d, G, dG, W);
        if (MS) {
            const double mb = D.mass[b];
            const double rs = kc.z + kb.z, irs = 1.0 / rs;
            const double2 g = A.gavg[b], l = lg[b];
            const double lb0 = g.x + l.x, lb1 = g.y + l.y;
            // own sum: f = eps m_b W / rs times (v_b - v_c)
            const double f = P.eps * mb * W * irs;
            const double S = lac.x * (kb.x - kc.x) + lac.y * (kb.y - kc.y);
            ub -= f * lac.x; vb -= f * lac.y;
            rb -= S * f * irs;
            const double Wb = S * P.eps * mb * irs;
            // the neighbour's sum: f' = eps m_c W / rs times (v_c - v_b)
            const double f2 = P.eps * mc * W * irs;
            const double S2 = lb0 * (kc.x - kb.x) + lb1 * (kc.y - kb.y);
            ub += f2 * lb0; vb += f2 * lb1;
            rb -= S2 * f2 * irs;
            mb_ += S2 * P.eps * W * irs;
            const double Wb2 = S2 * P.eps * mc * irs;
            // dW/dx_c = G r
            x0b += (Wb + Wb2) * G * r0; x1b += (Wb + Wb2) * G * r1;
        }
        // own sums: phi_b - phi_c, weight V_b
        {
            const double Vbn = D.mass[b] * A.irho[b];
            double S, f0, f1;
            rev_rawsum(r0, r1, id, G, dG, kb.z - kc.z, kb.x - kc.x, kb.y - kc.y, mc1, mc2, mc3, S, f0, f1,
                       MUSCL ? kb.w - kc.w : 0.0, mc4);
            x0b += Vbn * f0; x1b += Vbn * f1;
            rb -= Vbn * G * (mc1.x * r0 + mc1.y * r1);
            if (MUSCL) pb_ -= Vbn * G * (mc4.x * r0 + mc4.y * r1);
            ub -= Vbn * G * (mc1.z * r0 + mc1.w * r1);
            vb -= Vbn * G * (mc2.x * r0 + mc2.y * r1);
        }
        // neighbour's sums: phi_c - phi_b at r' = -r, weight V_c
        {
            const double4 mb1 = A.mu1[b], mb2 = A.mu2[b];
            const double2 mb3 = A.mu3[b];
            const double2 mb4 = MUSCL ? A.mu4[b] : make_double2(0.0, 0.0);
            double S, f0, f1;
            rev_rawsum(-r0, -r1, id, G, dG, kc.z - kb.z, kc.x - kb.x, kc.y - kb.y, mb1, mb2, mb3, S, f0, f1,
                       MUSCL ? kc.w - kb.w : 0.0, mb4);
            x0b -= Vc * f0; x1b -= Vc * f1;
            rb -= Vc * G * (mb1.x * r0 + mb1.y * r1);
            if (MUSCL) pb_ -= Vc * G * (mb4.x * r0 + mb4.y * r1);
            ub -= Vc * G * (mb1.z * r0 + mb1.w * r1);
            vb -= Vc * G * (mb2.x * r0 + mb2.y * r1);
            Vb += G * S;
        }
    }
    double v[8] = {x0b, x1b, ub, vb, rb, Vb, mb_, pb_};
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        if (!MS && q == 6) continue;
        if (!MUSCL && q == 7) continue;
        v[q] += __shfl_xor_sync(0xffffffffu, v[q], 1);
        if (kAdjLanes == 4) v[q] += __shfl_xor_sync(0xffffffffu, v[q], 2);
    }
    if (!live || lane != 0) return;
    x0b = v[0]; x1b = v[1]; ub = v[2]; vb = v[3]; rb = v[4]; Vb = v[5]; mb_ = v[6]; pb_ = v[7];
    const double2 sx = A.sx[c], su = A.su[c];
    if (MS) {
        A.sx[c] = make_double2(sx.x + x0b, sx.y + x1b);
        A.su[c] = make_double2(su.x + ub, su.y + vb);
        A.sr[c] += rb - Vc / kc.z * Vb;
        A.sm[c] += mb_ + Vb / kc.z;
        return;
    }
    if (MUSCL) {
        double dpd, dcd;
        eos_deriv(P, kc.z, dpd, dcd);
        rb += dpd * pb_;
    }
    stage_reverse(P, D, A, c, stage, dt, make_double2(sx.x + x0b, sx.y + x1b), make_double2(su.x + ub, su.y + vb),
                  A.sr[c] + rb - Vc / kc.z * Vb);
}

// The shifting sum of particle a over the pairs of the RHS state D, in FP64
// (the forward forms it in the last pass C of a step, k_pass_c<..., SHIFT>, or
// in k_shift_gather on the mixed Taylor-Green path):
//   s_a = sum_b phi(d) V_b r,  phi = (1 + R (W/W_dx)^4) G,  r = x_a - x_b.
template <typename R>
__global__ void k_shift_sum(Params P, Sorted<R> D, Adj A) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= P.n_tot) return;
    const double2 xa = D.pos[a];
    const double iwdx = 1.0 / P.w_dx;
    double s0 = 0.0, s1 = 0.0;
    const int nn = D.npairs[a];
    for (int e = 0; e < nn; ++e) {
        const int b = (int)(D.pairs[(size_t)e * P.nbr_stride + a] & 0x7fffffffu);
        const double2 xb = D.pos[b];
        const double r0 = xa.x - xb.x, r1 = xa.y - xb.y;
        const double d = sqrt(r0 * r0 + r1 * r1);
        double G, dG, W;
        kernel_gw(P, d, G, dG, W);
        const double q = W * iwdx, q2 = q * q;
        const double f = (1.0 + P.shift_R * (q2 * q2)) * G * (D.mass[b] / D.kin[b].z);
        s0 += f * r0; s1 += f * r1;
    }
    A.ssum[a] = make_double2(s0, s1);
}

// Reverse of the shifting sums with their adjoints mu (smu): particle c adds
// d(mu_c . s_c)/dx_c (its own sum) and d(mu_b . s_b)/d(x_c, rho_c) over its pair
// neighbours b (their sums, through r and V_c = m_c / rho_c) to sx, sr.
template <typename R>
__global__ void k_adj_shift(Params P, Sorted<R> D, Adj A) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n_tot) return;
    const double2 xc = D.pos[c];
    const double2 mc = A.smu[c];
    const double Vc = D.mass[c] * A.irho[c];
    const double iwdx = 1.0 / P.w_dx;
    double x0b = 0, x1b = 0, Vb_ = 0;
    const int nn = D.npairs[c];
    for (int e = 0; e < nn; ++e) {
        const int b = (int)(D.pairs[(size_t)e * P.nbr_stride + c] & 0x7fffffffu);
        const double2 mb = A.smu[b];
        if (mc.x == 0.0 && mc.y == 0.0 && mb.x == 0.0 && mb.y == 0.0) continue;
        const double2 xb = D.pos[b];
        const double r0 = xc.x - xb.x, r1 = xc.y - xb.y;
        const double d = sqrt(r0 * r0 + r1 * r1), id = 1.0 / d;
        double G, dG, W;
        kernel_gw(P, d, G, dG, W);
        const double q = W * iwdx, q2 = q * q, q4 = q2 * q2;
        const double phi = (1.0 + P.shift_R * q4) * G;
        // dphi/dd: dW/dd = G d
        const double dphi = 4.0 * P.shift_R * q2 * q * (G * d * iwdx) * G + (1.0 + P.shift_R * q4) * dG;
        const double Vb = D.mass[b] * A.irho[b];
        // own sum: mu_c . V_b phi r, r = x_c - x_b
        const double rm = r0 * mc.x + r1 * mc.y;
        x0b += Vb * (phi * mc.x + dphi * rm * r0 * id);
        x1b += Vb * (phi * mc.y + dphi * rm * r1 * id);
        // the neighbour's sum: mu_b . V_c phi r', r' = -r
        const double rmb = -(r0 * mb.x + r1 * mb.y);
        x0b -= Vc * (phi * mb.x - dphi * rmb * r0 * id);
        x1b -= Vc * (phi * mb.y - dphi * rmb * r1 * id);
        Vb_ += phi * rmb;
    }
    const double2 sx = A.sx[c];
    A.sx[c] = make_double2(sx.x + x0b, sx.y + x1b);
    A.sr[c] -= Vc * A.irho[c] * Vb_;
    // the moving square's assigned ghosts also carry a mass adjoint (V = m / rho)
    if (P.ms) A.sm[c] += Vb_ * A.irho[c];
}

// Reverse of the step end's capped shift and density correction for slot s
// (x' = x + dc, rho' = rho + grad rho.dc, dc the capped shift of the last RHS):
// the adjoints of the shift sum, grad rho and B^-1 go to smu, shgr, shbi.
template <typename R>
__device__ __forceinline__ void shift_reverse(const Params& P, const Sorted<R>& D, const Adj& A, int s, int i,
                                              double2 lx, double lrho) {
    // (the shift moves the water particles that are not near the surface)
    {
        double2 mu = make_double2(0, 0), sg = make_double2(0, 0);
        double4 sb = make_double4(0, 0, 0, 0);
        if (i < P.n_host && D.type[s] == SPH_TYPE_WATER && !(D.flags[s] & 2)) {
            const double2 ss = A.ssum[s];
            const double4 bi = D.binv64[s];
            const double c = -P.shift_beta * (P.h * P.h);
            const double d0 = c * (bi.x * ss.x + bi.y * ss.y), d1 = c * (bi.z * ss.x + bi.w * ss.y);
            const double amp = sqrt(d0 * d0 + d1 * d1);
            const bool capped = amp > P.shift_max;
            const double dc0 = capped ? d0 / amp * P.shift_max : d0, dc1 = capped ? d1 / amp * P.shift_max : d1;
            const double g0 = grad_scale<R>() * D.nb1[s].w, g1 = grad_scale<R>() * D.nb2[s].x;
            // x' = x + dc, rho' = rho + g.dc
            const double b0 = lx.x + lrho * g0, b1 = lx.y + lrho * g1;
            sg = make_double2(lrho * dc0, lrho * dc1);
            double e0 = b0, e1 = b1;
            if (capped) {
                const double k = P.shift_max / amp, h0 = d0 / amp, h1 = d1 / amp;
                const double hb = h0 * b0 + h1 * b1;
                e0 = k * (b0 - h0 * hb); e1 = k * (b1 - h1 * hb);
            }
            // delta = c B^-1 s
            mu = make_double2(c * (bi.x * e0 + bi.z * e1), c * (bi.y * e0 + bi.w * e1));
            sb = make_double4(c * e0 * ss.x, c * e0 * ss.y, c * e1 * ss.x, c * e1 * ss.y);
        }
        A.smu[s] = mu; A.shgr[s] = sg; A.shbi[s] = sb;
    }
}

// Reverse of stage 3 (the step end) from the id-order adjoints of the end state
// and of the carried rates.  Non-integrated host particles keep their state.
// With shift: the step end also moved the water particles that are not near
// the surface by the capped shift cap(delta), delta = -beta h^2 B^-1 s (s from
// k_shift_sum), and corrected rho by grad rho . cap(delta)
// (Shift_particle_position.f90:97-136): its reverse leaves the adjoints of s
// (smu), grad rho (shgr) and B^-1 (shbi) of the last RHS; the cap is the branch
// the forward took.
template <typename R>
__global__ void k_adj_stage3(Params P, Sorted<R> D, Adj A, double dt, int shift, const double2* ox = nullptr,
                             const double* orho = nullptr) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.n_tot) return;
    const int i = D.id[s];
    double2 lx = make_double2(0, 0), lv = make_double2(0, 0);
    double lrho = 0.0;
    if (i < P.n_host) { lx = A.lx[i]; lv = A.lv[i]; lrho = A.lrho[i]; }
    // ox / orho: the adjoint of the last stage's positions and densities when the
    // step ended with the density re-initialisation (its reverse and that of the
    // shift after it already ran: k_adj_mls_end, k_adj_mls_own, k_adj_mls_nbr)
    if (ox) { lx = ox[s]; lrho = orho[s]; shift = 0; }
    if (shift) shift_reverse<R>(P, D, A, s, i, lx, lrho);
    for (int k = 0; k < 4; ++k) { A.lr[k][s] = 0.0; A.la[k][s] = make_double2(0, 0); }
    A.lxe[s] = make_double2(0, 0);
    if (i < P.n_host && integrated(P, D.type[s])) {
        // x' = x0 + (u1 + 2 u2 + 2 u3 + u') dt/6 + dt^2 a4/2,
        // u' = v0 + (a1 + 2 a2 + 2 a3 + a4) dt/6, rho' = rho0 + (d1 + 2 d2 + 2 d3 + d4) dt/6
        const double w6 = dt / 6.0, w3 = dt / 3.0;
        const double2 lu = make_double2(lv.x + w6 * lx.x, lv.y + w6 * lx.y);
        A.ax0[s] = lx;
        A.av0[s] = lu;
        A.ar0[s] = lrho;
        A.lxe[s] = lx;
        const double2 lka = A.lk_a[i];
        A.la[0][s] = make_double2(w6 * lu.x, w6 * lu.y);
        A.la[1][s] = make_double2(w3 * lu.x, w3 * lu.y);
        A.la[2][s] = make_double2(w3 * lu.x, w3 * lu.y);
        A.la[3][s] = make_double2(w6 * lu.x + 0.5 * dt * dt * lx.x + lka.x, w6 * lu.y + 0.5 * dt * dt * lx.y + lka.y);
        A.lr[0][s] = w6 * lrho;
        A.lr[1][s] = w3 * lrho;
        A.lr[2][s] = w3 * lrho;
        A.lr[3][s] = w6 * lrho + A.lk_r[i];
    } else {
        A.ax0[s] = lx;
        A.av0[s] = lv;
        A.ar0[s] = lrho;
    }
}


// ---- reverse of the density re-initialisation (moving least squares) -------
// The forward (k_mls, Taylor-Green variant) forms, for a water host a and its
// neighbours b within the support at the state the step's last stage produced,
//   A = sum W_b p_b p_b^T + alpha^3 I,  r = sum rho_b W_b p_b,  rho_a' = c.r,  A c = e_1,
// p_b = (1, dx, dy[, dx^2, dx dy, dy^2]), (dx, dy) = (x_b - x_a)/h, W_b = W(|x_a - x_b|),
// or rho_a' = sum rho_b W_b / S, S = sum W_b, when A is singular or (order 6) a
// has at most 8 neighbours.  With lam the adjoint of rho_a' and y = A^-1 (lam r):
//   rho_b-bar += lam W_b (c.p_b),   W_b-bar = (c.p_b)(lam rho_b - y.p_b),
//   p_b-bar = lam rho_b W_b c - W_b ((c.p_b) y + (y.p_b) c)
// (Shepard: rho_b-bar += lam W_b / S, W_b-bar = lam (rho_b - rho_a') / S), then
// through p_b to x_b - x_a and through W_b to |x_a - x_b|.
// The moving-square variant weights by W_b V_b, V_b = m_b / rho_b, counts a
// itself (distance 0: no position derivative), tests only d <= r_cut, has no
// few-neighbour fallback and keeps rho_a where the result is NaN: the formulas
// above with W_b V_b in place of W_b, whose adjoint then reaches W_b (times
// V_b), rho_b (times -W_b V_b / rho_b) and m_b (times W_b / rho_b; the ghosts'
// assigned mass).

// The Cholesky factor of k_mls's solve (the same operations in the same order,
// so c = A^-1 e_1 takes the forward's bits) and a solve with it.
template <int M>
__device__ __forceinline__ bool mls_chol(const double (&A)[M * (M + 1) / 2], double (&L)[M * (M + 1) / 2]) {
#pragma unroll
    for (int i = 0; i < M; ++i) {
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            double sum = A[i * (i + 1) / 2 + j];
#pragma unroll
            for (int k = 0; k < j; ++k) sum -= L[i * (i + 1) / 2 + k] * L[j * (j + 1) / 2 + k];
            if (i == j) {
                if (!(sum > 0.0)) return false;
                L[i * (i + 1) / 2 + i] = sqrt(sum);
            } else {
                L[i * (i + 1) / 2 + j] = sum / L[j * (j + 1) / 2 + j];
            }
        }
    }
    return true;
}

template <int M>
__device__ __forceinline__ void mls_solve(const double (&L)[M * (M + 1) / 2], const double (&b)[M], double (&x)[M]) {
    double y[M];
#pragma unroll
    for (int i = 0; i < M; ++i) {
        double sum = b[i];
#pragma unroll
        for (int k = 0; k < i; ++k) sum -= L[i * (i + 1) / 2 + k] * y[k];
        y[i] = sum / L[i * (i + 1) / 2 + i];
    }
#pragma unroll
    for (int i = M - 1; i >= 0; --i) {
        double sum = y[i];
#pragma unroll
        for (int k = i + 1; k < M; ++k) sum -= L[k * (k + 1) / 2 + i] * x[k];
        x[i] = sum / L[i * (i + 1) / 2 + i];
    }
}

// p-bar -> (dx, dy)-bar
template <int M>
__device__ __forceinline__ void mls_pbar_to_d(const double (&pb)[6], double dx, double dy, double& dxb, double& dyb) {
    dxb = pb[1];
    dyb = pb[2];
    if (M == 6) {
        dxb += 2.0 * dx * pb[3] + dy * pb[4];
        dyb += dx * pb[4] + 2.0 * dy * pb[5];
    }
}

// The step end's adjoint split for the reverse of a step that ended with the
// density re-initialisation: the shift after it reversed (as in k_adj_stage3),
// then the positions' adjoint (xe) and the adjoint of the re-initialised
// density (lam) per slot.
template <typename R>
__global__ void k_adj_mls_end(Params P, Sorted<R> D, Adj A, int shift, double2* xe, double* lam) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.n_tot) return;
    const int i = D.id[s];
    double2 lx = make_double2(0, 0);
    double lrho = 0.0;
    if (i < P.n_host) { lx = A.lx[i]; lrho = A.lrho[i]; }
    if (shift) shift_reverse<R>(P, D, A, s, i, lx, lrho);
    xe[s] = lx;
    lam[s] = lrho;
}

// The pair test of the re-initialisation: the support of the pair search, or
// (moving square) d <= r_cut alone.
__device__ __forceinline__ bool mls_in(const Params& P, double px, double py, double& d) {
    const bool in = in_support(P, px, py, d);
    return P.ms ? d <= P.r_cut : in;
}

// Per owner a (a water host): A, r and the solve of k_mls on the state V the
// last stage produced, y = A^-1 (lam_a r), and the adjoint of x_a through its
// own sum.  cy[16 a ..]: c (0-5), y (6-11), mode (12: 0 not an owner or the
// density kept, 1 the moving-least-squares weights, 2 Shepard), S (13),
// rho_a' (14), the adjoint of rho_a through a's own term (15, moving square).
template <typename R, int M>
__global__ void k_adj_mls_own(Params P, Sorted<R> V, const double* lam, double* cy, double2* xown) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= P.n_tot) return;
    double* o = cy + (size_t)16 * a;
    o[12] = 0.0;
    o[15] = 0.0;
    xown[a] = make_double2(0.0, 0.0);
    if (V.type[a] != SPH_TYPE_WATER || V.id[a] >= P.n_host) return;
    const double2 xa = V.pos[a];
    const double inv_h = 1.0 / P.h;
    double Am[M * (M + 1) / 2], r[M];
#pragma unroll
    for (int k = 0; k < M * (M + 1) / 2; ++k) Am[k] = 0.0;
#pragma unroll
    for (int k = 0; k < M; ++k) r[k] = 0.0;
    double sw = 0.0, srw = 0.0;
    int cnt = 0;
    const int nn = V.nnbr[a];
    // (the moving-square variant: a itself first, e = -1)
    for (int e = P.ms ? -1 : 0; e < nn; ++e) {
        const int b = e < 0 ? a : (int)(V.nbr[(size_t)e * P.nbr_stride + a] & 0x7fffffffu);
        const double2 xb = V.pos[b];
        const double px = xa.x - xb.x, py = xa.y - xb.y;
        double d;
        if (!mls_in(P, px, py, d)) continue;
        double w, gx, gy;
        kernel_w_dw<double>(P, d, px, py, w, gx, gy);
        const double rho_b = V.kin[b].z;
        if (P.ms) w *= V.mass[b] / rho_b;
        double p[M];
        const double dx = -px * inv_h, dy = -py * inv_h;
        p[0] = 1.0; p[1] = dx; p[2] = dy;
        if (M == 6) { p[3 % M] = dx * dx; p[4 % M] = dx * dy; p[5 % M] = dy * dy; }
#pragma unroll
        for (int i = 0; i < M; ++i) {
            const double wp = w * p[i];
#pragma unroll
            for (int j = 0; j <= i; ++j) Am[i * (i + 1) / 2 + j] += wp * p[j];
            r[i] += rho_b * wp;
        }
        sw += w;
        srw += rho_b * w;
        ++cnt;
    }
#pragma unroll
    for (int i = 0; i < M; ++i) Am[i * (i + 1) / 2 + i] += P.mls_alpha3;
    const double lm = lam[a];
    double L[M * (M + 1) / 2], c[M], y[M];
    const bool ok = !(!P.ms && M == 6 && cnt <= 8) && mls_chol<M>(Am, L);
    const double out = srw / sw;
    if (ok) {
        double e1[M], lr[M];
#pragma unroll
        for (int i = 0; i < M; ++i) { e1[i] = i == 0 ? 1.0 : 0.0; lr[i] = lm * r[i]; }
        mls_solve<M>(L, e1, c);
        mls_solve<M>(L, lr, y);
        double cr = 0.0;
#pragma unroll
        for (int i = 0; i < M; ++i) { o[i] = c[i]; o[6 + i] = y[i]; cr += c[i] * r[i]; }
        o[12] = 1.0;
        // (the moving square keeps the old density where the result is NaN)
        if (P.ms && isnan(cr)) { o[12] = 0.0; return; }
    } else {
        if (P.ms && isnan(out)) return;
        o[12] = 2.0;
        o[13] = sw;
        o[14] = out;
    }
    if (P.ms) {
        // a's own term: W(0) V_a with p = e_1, no position derivative
        double d0;
        mls_in(P, 0.0, 0.0, d0);
        double w, gx, gy;
        kernel_w_dw<double>(P, d0, 0.0, 0.0, w, gx, gy);
        const double rho_a = V.kin[a].z;
        const double wt = w * (V.mass[a] / rho_a);
        const double Wt = ok ? c[0] * (lm * rho_a - y[0]) : lm * (rho_a - out) / sw;
        o[15] = (ok ? lm * wt * c[0] : lm * wt / sw) - Wt * wt / rho_a;
    }
    double xb0 = 0.0, xb1 = 0.0;
    for (int e = 0; e < nn; ++e) {
        const int b = (int)(V.nbr[(size_t)e * P.nbr_stride + a] & 0x7fffffffu);
        const double2 xb = V.pos[b];
        const double px = xa.x - xb.x, py = xa.y - xb.y;
        double d;
        if (!mls_in(P, px, py, d)) continue;
        double w, gx, gy;
        kernel_w_dw<double>(P, d, px, py, w, gx, gy);
        const double rho_b = V.kin[b].z;
        const double f = P.ms ? V.mass[b] / rho_b : 1.0;     // the weight W f
        const double wt = w * f;
        double Wb;
        if (ok) {
            const double dx = -px * inv_h, dy = -py * inv_h;
            double p[6] = {1.0, dx, dy, dx * dx, dx * dy, dy * dy};
            double cp = 0.0, yp = 0.0;
#pragma unroll
            for (int i = 0; i < M; ++i) { cp += c[i] * p[i]; yp += y[i] * p[i]; }
            Wb = cp * (lm * rho_b - yp) * f;
            double pb[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
            for (int i = 0; i < M; ++i) pb[i] = lm * rho_b * wt * c[i] - wt * (yp * c[i] + cp * y[i]);
            double dxb, dyb;
            mls_pbar_to_d<M>(pb, dx, dy, dxb, dyb);
            xb0 -= dxb * inv_h; xb1 -= dyb * inv_h;       // (dx, dy) = (x_b - x_a)/h
        } else {
            Wb = lm * (rho_b - out) / sw * f;
        }
        xb0 += Wb * gx; xb1 += Wb * gy;                   // grad_a W = (gx, gy)
    }
    xown[a] = make_double2(xb0, xb1);
}

// Per particle q: its position and density adjoints through the re-initialised
// densities of the owners a it is a neighbour of (gathered over q's list, which
// holds every such a), plus the step end's (xe) and the owner's own part (xown);
// a particle that is not an owner keeps its density, rho' = rho.  Moving
// square: an owner's own term (cy[16 q + 15]) is added, and for the ghosts the
// adjoints of the density and mass they carried (as the corrector RHS assigned
// them) go to gm instead of orho (their density passes through: orho = lam).
template <typename R, int M>
__global__ void k_adj_mls_nbr(Params P, Sorted<R> V, const double* lam, const double* cy, const double2* xown,
                              const double2* xe, double2* ox, double* orho, double2* gm) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= P.n_tot) return;
    const double2 xq = V.pos[q];
    const double rho_q = V.kin[q].z;
    const bool water = V.type[q] == SPH_TYPE_WATER;
    const bool owner = water && V.id[q] < P.n_host && cy[(size_t)16 * q + 12] != 0.0;
    const double fq = P.ms ? V.mass[q] / rho_q : 1.0;
    const double inv_h = 1.0 / P.h;
    const double2 x0 = xe[q], x1 = xown[q];
    double xb0 = x0.x + x1.x, xb1 = x0.y + x1.y;
    double rb = 0.0, mb = 0.0;
    const int nn = V.nnbr[q];
    for (int e = 0; e < nn; ++e) {
        const int a = (int)(V.nbr[(size_t)e * P.nbr_stride + q] & 0x7fffffffu);
        const double* o = cy + (size_t)16 * a;
        const double mode = o[12];
        if (mode == 0.0) continue;
        const double2 xa = V.pos[a];
        const double px = xa.x - xq.x, py = xa.y - xq.y;
        double d;
        if (!mls_in(P, px, py, d)) continue;
        double w, gx, gy;
        kernel_w_dw<double>(P, d, px, py, w, gx, gy);
        const double wt = w * fq;
        const double lm = lam[a];
        double Wt;                                         // the adjoint of the weight W fq
        if (mode == 1.0) {
            const double dx = -px * inv_h, dy = -py * inv_h;
            double p[6] = {1.0, dx, dy, dx * dx, dx * dy, dy * dy};
            double c[M], y[M];
            double cp = 0.0, yp = 0.0;
#pragma unroll
            for (int i = 0; i < M; ++i) { c[i] = o[i]; y[i] = o[6 + i]; cp += c[i] * p[i]; yp += y[i] * p[i]; }
            rb += lm * wt * cp;
            Wt = cp * (lm * rho_q - yp);
            double pb[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
            for (int i = 0; i < M; ++i) pb[i] = lm * rho_q * wt * c[i] - wt * (yp * c[i] + cp * y[i]);
            double dxb, dyb;
            mls_pbar_to_d<M>(pb, dx, dy, dxb, dyb);
            xb0 += dxb * inv_h; xb1 += dyb * inv_h;
        } else {
            const double S = o[13], out = o[14];
            rb += lm * wt / S;
            Wt = lm * (rho_q - out) / S;
        }
        if (P.ms) {
            rb -= Wt * wt / rho_q;                         // V_q = m_q / rho_q
            mb += Wt * w / rho_q;
        }
        const double Wb = Wt * fq;
        xb0 -= Wb * gx; xb1 -= Wb * gy;                   // grad_q W = -grad_a W
    }
    if (owner) rb += cy[(size_t)16 * q + 15];
    ox[q] = make_double2(xb0, xb1);
    if (P.ms && !water) {
        orho[q] = lam[q];
        gm[q] = make_double2(rb, mb);
    } else {
        orho[q] = owner ? rb : rb + lam[q];
        if (gm) gm[q] = make_double2(0.0, 0.0);
    }
}

// The moving square's ghosts: the adjoints of the density and mass they carried
// into the re-initialisation (gm) join those of the corrector RHS that assigned
// them, after k_adj_c has formed the latter.
template <typename R>
__global__ void k_adj_add_ghost_rm(Params P, Sorted<R> D, Adj A, const double2* gm) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.n_tot || D.type[s] == SPH_TYPE_WATER) return;
    const double2 g = gm[s];
    A.sr[s] += g.x;
    A.sm[s] += g.y;
}

// ---- reverse of the order-1 re-initialisation --------------------------------
// The forward (k_mls1) forms, on the state of the step's last RHS and over its
// pair list, for a water host a:
//   rho_a' = S_m / S_w,  S_m = sum_b m_b W_ab,  S_w = sum_b W_ab V_b,  V_b = m_b / rho_b,
// over the pairs with a neighbour b of a's type; the stage that ends the step
// then discards a's integrated density.  With lam the adjoint of rho_a':
//   W_ab-bar = lam m_b (1 - rho_a' / rho_b) / S_w,
//   rho_b-bar += lam rho_a' W_ab m_b / (S_w rho_b^2).

// The step end's split: the positions' adjoint passes through to the last
// stage, a water host's density adjoint goes to the re-initialisation alone
// (its integrated density was replaced), the others' pass through.
template <typename R>
__global__ void k_adj_mls1_end(Params P, Sorted<R> D, const double2* xe, const double* lam, double2* ox,
                               double* orho) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.n_tot) return;
    ox[s] = xe[s];
    orho[s] = (D.type[s] == SPH_TYPE_WATER && D.id[s] < P.n_host) ? 0.0 : lam[s];
}

// Per owner a on the last RHS's state V: S_w and rho_a' with k_mls1's operations
// (cy[16 a ..]: mode 12 = 2 for an owner, S_w 13, rho_a' 14).
template <typename R>
__global__ void k_adj_mls1_own(Params P, Sorted<R> V, double* cy) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= P.n_tot) return;
    double* o = cy + (size_t)16 * a;
    o[12] = 0.0;
    const int ta = V.type[a];
    if (ta != SPH_TYPE_WATER || V.id[a] >= P.n_host) return;
    const double2 xa = V.pos[a];
    double sw = 0.0, sm = 0.0;
    const int nn = V.npairs[a];
    for (int e = 0; e < nn; ++e) {
        const int b = (int)(V.pairs[(size_t)e * P.nbr_stride + a] & 0x7fffffffu);
        if (V.type[b] != ta) continue;
        const double2 xb = V.pos[b];
        const double px = xa.x - xb.x, py = xa.y - xb.y;
        const double d = __dsqrt_rn(__dadd_rn(__dmul_rn(px, px), __dmul_rn(py, py)));
        double w, gx, gy;
        kernel_w_dw<double>(P, d, px, py, w, gx, gy);
        const double mb = V.mass[b];
        sw += w * (mb / V.kin[b].z);
        sm += mb * w;
    }
    o[12] = 2.0;
    o[13] = sw;
    o[14] = sm / sw;
}

// Per particle q of the last RHS's state: the adjoints of its position and
// density through its own order-1 density and those of the owners in its pair
// list, added to sx and sr (after k_adj_c has formed the RHS's own).
template <typename R>
__global__ void k_adj_mls1_nbr(Params P, Sorted<R> V, Adj A, const double* lam, const double* cy) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= P.n_tot) return;
    const int tq = V.type[q];
    const double2 xq = V.pos[q];
    const double rho_q = V.kin[q].z, m_q = V.mass[q];
    const double* oq = cy + (size_t)16 * q;
    const bool own = oq[12] != 0.0;
    const double lq = own ? lam[q] : 0.0, swq = own ? oq[13] : 1.0, rq = own ? oq[14] : 0.0;
    double x0b = 0.0, x1b = 0.0, rb = 0.0;
    const int nn = V.npairs[q];
    for (int e = 0; e < nn; ++e) {
        const int b = (int)(V.pairs[(size_t)e * P.nbr_stride + q] & 0x7fffffffu);
        if (V.type[b] != tq) continue;
        const double* ob = cy + (size_t)16 * b;
        const bool bown = ob[12] != 0.0;
        if (!own && !bown) continue;
        const double2 xb = V.pos[b];
        const double px = xq.x - xb.x, py = xq.y - xb.y;
        const double d = __dsqrt_rn(__dadd_rn(__dmul_rn(px, px), __dmul_rn(py, py)));
        double w, gx, gy;
        kernel_w_dw<double>(P, d, px, py, w, gx, gy);      // grad_q W = (gx, gy)
        double Wb = 0.0;
        if (own) {
            const double rho_b = V.kin[b].z;
            Wb += lq * V.mass[b] * (1.0 - rq / rho_b) / swq;
        }
        if (bown) {
            const double lb = lam[b], swb = ob[13], rbp = ob[14];
            Wb += lb * m_q * (1.0 - rbp / rho_q) / swb;
            rb += lb * rbp * w * m_q / (swb * (rho_q * rho_q));
        }
        x0b += Wb * gx;
        x1b += Wb * gy;
    }
    const double2 sx = A.sx[q];
    A.sx[q] = make_double2(sx.x + x0b, sx.y + x1b);
    A.sr[q] += rb;
}

// Sorted step-start adjoints -> id order; the K1 adjoint goes to the previous step.
template <typename R>
__global__ void k_adj_scatter(Params P, Sorted<R> D, Adj A, int first) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.n_tot) return;
    const int i = D.id[s];
    A.lx[i] = A.ax0[s];
    A.lv[i] = A.av0[s];
    A.lrho[i] = A.ar0[s];
    if (i < P.n_host) {
        A.lk_r[i] = first ? 0.0 : A.lr[0][s];
        A.lk_a[i] = first ? make_double2(0, 0) : A.la[0][s];
        if (A.lk_g) A.lk_g[i] = first ? make_double2(0, 0) : A.lg[0][s];
    }
}

// Image adjoints to their sources (the images are copies of the step-start
// state, shifted by a period): bottom/top images first, since their sources
// include left/right images, then left/right images to the host particles.
__global__ void k_adj_route(int n_src, int base, const int* cnt, const int* off, Adj A) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_src) return;
    const int c = cnt[s];
    if (c == 0) return;
    double2 x = A.lx[s], v = A.lv[s];
    double r = A.lrho[s];
    for (int k = 0; k < c; ++k) {
        const int j = base + off[s] + k;
        const double2 xj = A.lx[j], vj = A.lv[j];
        x.x += xj.x; x.y += xj.y; v.x += vj.x; v.y += vj.y; r += A.lrho[j];
    }
    A.lx[s] = x; A.lv[s] = v; A.lrho[s] = r;
}

// The hi/lo records of the mixed path formed from the FP64 state of V (as the
// forward's stages write them).
template <typename R>
__global__ void k_resplit(int n, Sorted<R> D) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    store_split(D, s, D.pos[s], D.kin[s]);
}

// Stage state -> the arrays the RHS reads (positions, kinematic and auxiliary records).
template <typename R>
__global__ void k_adj_load(Params P, Sorted<R> D, const double2* pos, const double4* kin) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.n_tot) return;
    const double2 x = pos ? pos[s] : D.pos0[s];
    double4 k;
    if (kin) k = kin[s];
    else {
        const double2 v = D.vel0[s];
        double p, c;
        eos64(P, D.rho0[s], p, c);
        k = make_double4(v.x, v.y, D.rho0[s], p);
    }
    double p, c;
    eos64(P, k.z, p, c);
    const double m = D.mass[s];
    D.pos[s] = x;
    D.kin[s] = k;
    D.aux[s] = mk4<R>((R)m, (R)(m / k.z), (R)c, (R)D.smass[s]);
    store_split(D, s, x, k);
}

// Copies of the state a step starts from (id order, host particles) into or out
// of a snapshot slot, as one launch.
struct SnapPtrs {
    double2 *pos, *vel, *r_acc, *r_avg;
    double *rho, *r_drho;
};
__global__ void k_snap_copy(int n, SnapPtrs dst, SnapPtrs src) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    dst.pos[i] = src.pos[i]; dst.vel[i] = src.vel[i]; dst.rho[i] = src.rho[i];
    dst.r_drho[i] = src.r_drho[i]; dst.r_acc[i] = src.r_acc[i]; dst.r_avg[i] = src.r_avg[i];
}

// The sorted step-start state a reversed step needs (what prepare wrote: the
// permutation, the sorted master state and records, the cell ranges and the
// neighbour lists, and the id-order image routing), kept per step of a segment
// while the segment is re-run and restored by the reverse step instead of
// re-sorting.  One descriptor per array (a neighbour-list row is an array):
// words = 4-byte words per particle (per_particle = 1, times n_tot) or in all.
struct PrepDesc {
    unsigned* field;
    long long off;        // word offset in a slot
    int per_particle;
    int words;
    long long pitch;      // > 0: the neighbour lists, row e of particle a at e * pitch + a
};

// save = 1: arrays -> slot; save = 0: slot -> arrays.  blockIdx.y = descriptor.
// cnt: the list lengths (the live ones when saving, the slot's copy when
// restoring, so no launch reads counts it is writing); each particle copies its
// own entries only.  Arrays whose size is a multiple of 16 bytes move in 16-byte
// words (the arrays and the slot offsets are 256-byte aligned).
__global__ void k_prep_copy(const PrepDesc* d, int n_tot, unsigned* slot, int save, const int* cnt) {
    const PrepDesc c = d[blockIdx.y];
    unsigned* s = slot + c.off;
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long stride = (long long)gridDim.x * blockDim.x;
    if (c.pitch > 0) {
        for (long long a = t0; a < n_tot; a += stride) {
            const int n = cnt[a];
            for (int e = 0; e < n; ++e) {
                const long long k = (long long)e * c.pitch + a;
                if (save) s[k] = c.field[k];
                else c.field[k] = s[k];
            }
        }
        return;
    }
    const long long total = c.per_particle ? (long long)n_tot * c.words : (long long)c.words;
    if ((total & 3) == 0) {
        uint4* f4 = reinterpret_cast<uint4*>(c.field);
        uint4* s4 = reinterpret_cast<uint4*>(s);
        for (long long w = t0; w < total / 4; w += stride) {
            if (save) s4[w] = f4[w];
            else f4[w] = s4[w];
        }
    } else {
        for (long long w = t0; w < total; w += stride) {
            if (save) s[w] = c.field[w];
            else c.field[w] = s[w];
        }
    }
}

// Copy of the stage state (positions and records) into the stage store.
template <typename R>
__global__ void k_keep_stage(int n, Sorted<R> D, double2* pos, double4* kin, typename VT<R>::V4* aux) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    pos[s] = D.pos[s]; kin[s] = D.kin[s]; aux[s] = D.aux[s];
}

// Loss of the final state (id order, host water particles): per-block partials.
__global__ void k_adj_loss(int n, int kind, const int* type, const double2* vel, const double* mass,
                           const double2* target, double* part) {
    __shared__ double red[256];
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (type[i] != SPH_TYPE_WATER || kind == SPH_LOSS_DRAG) continue;
        const double2 v = vel[i];
        if (kind == SPH_LOSS_VELOCITY_MISFIT) {
            const double2 t = target[i];
            s += (v.x - t.x) * (v.x - t.x) + (v.y - t.y) * (v.y - t.y);
        } else {
            s += 0.5 * mass[i] * (v.x * v.x + v.y * v.y);
        }
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// Adjoint of the final state: dL/dv scaled by dloss; the positions, densities
// and carried rates do not enter the loss (nor the final state the drag loss,
// whose terms enter step by step in the reverse sweep).
__global__ void k_adj_seed(int n, int kind, double dloss, const int* type, const double2* vel, const double* mass,
                           const double2* target, Adj A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double2 g = make_double2(0, 0);
    if (type[i] == SPH_TYPE_WATER && kind != SPH_LOSS_DRAG) {
        const double2 v = vel[i];
        if (kind == SPH_LOSS_VELOCITY_MISFIT) {
            const double2 t = target[i];
            g = make_double2(2.0 * dloss * (v.x - t.x), 2.0 * dloss * (v.y - t.y));
        } else {
            g = make_double2(dloss * mass[i] * v.x, dloss * mass[i] * v.y);
        }
    }
    A.lv[i] = g;
    A.lx[i] = make_double2(0, 0);
    A.lrho[i] = 0.0;
    A.lk_r[i] = 0.0;
    A.lk_a[i] = make_double2(0, 0);
    if (A.lk_g) A.lk_g[i] = make_double2(0, 0);
}

// ---------------------------------------------------------------------------
// Moving-square path: Euler predictor-corrector with carried rates, ghost
// assignment, body motion and the drag loss.
// ---------------------------------------------------------------------------

// Reverse of the drag loss term w * F_x of one RHS, F = the total body force of
// k_body_force (Calculate_Body_Force.f90:53-142, Morris laplacian):
//   F_x = sum_a V_a sum_{b in body} T_ab,
//   T_ab = V_b [ -(p_a + p_b) G L0 + 2 nu rho_a G Q (u_a - u_b) / d^2 ],
// r = x_a - x_b, L = B_a^-1 r, Q = r.L.  Thread c adds the derivative with
// respect to its inputs as particle a (its body neighbours b) and, for a body
// particle, as particle b (its neighbours a), to the state adjoints of the RHS;
// dL/dnu partials per block into nu_part.  Only body particles and the
// particles k_mark_body_nbrs flagged (nflag == 2) have terms.
template <typename R>
__global__ void __launch_bounds__(kAdjThreads) k_adj_drag(Params P, Sorted<R> D, Adj A, double w, double* nu_part) {
    __shared__ double red[kAdjThreads];
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    double nu_sum = 0.0;
    if (c < P.n_tot && (D.itype[c] == SPH_TYPE_BODY || D.nflag[c] == 2)) {
        const bool cbody = D.itype[c] == SPH_TYPE_BODY;
        const double2 xc = D.pos[c];
        const double4 kc = D.kin[c];
        const double Vc = D.mass[c] * A.irho[c];
        const double4 bic = D.binv64[c];
        double x0b = 0, x1b = 0, ub = 0, pb = 0, rb = 0, Vb_ = 0;
        double4 gb = make_double4(0, 0, 0, 0);
        const int nn = D.npairs[c];
        for (int e = 0; e < nn; ++e) {
            const int b = (int)(D.pairs[(size_t)e * P.nbr_stride + c] & 0x7fffffffu);
            const bool bbody = D.itype[b] == SPH_TYPE_BODY;
            if (!bbody && !cbody) continue;
            const double2 xb = D.pos[b];
            const double4 kb = D.kin[b];
            const double Vb = D.mass[b] * A.irho[b];
            // the term of pair (a, b): a = c when b is the body particle, else a = b
            const bool c_is_a = bbody;
            const double4 bi = c_is_a ? bic : D.binv64[b];
            const double4 ka = c_is_a ? kc : kb, kbb = c_is_a ? kb : kc;
            const double Va = c_is_a ? Vc : Vb, Vbb = c_is_a ? Vb : Vc;
            const double r0 = c_is_a ? xc.x - xb.x : xb.x - xc.x, r1 = c_is_a ? xc.y - xb.y : xb.y - xc.y;
            const double d2 = r0 * r0 + r1 * r1, d = sqrt(d2), id = 1.0 / d, id2 = id * id;
            double G, dG;
            kernel_g(P, d, G, dG);
            const double L0 = bi.x * r0 + bi.y * r1, L1 = bi.z * r0 + bi.w * r1;
            const double Q = r0 * L0 + r1 * L1;
            const double P2 = ka.w + kbb.w, du = ka.x - kbb.x;
            const double K = 2.0 * P.nu * ka.z;
            const double Tin = -P2 * G * L0 + K * du * G * Q * id2;
            const double wv = w * Va * Vbb;
            // d/dr of Tin
            const double gq0 = L0 + bi.x * r0 + bi.z * r1, gq1 = L1 + bi.y * r0 + bi.w * r1;
            const double kd = dG * id;
            const double t1 = K * du * id2;
            const double Tr0 = -P2 * (kd * r0 * L0 + G * bi.x) + t1 * (kd * r0 * Q + G * gq0 - 2.0 * G * Q * r0 * id2);
            const double Tr1 = -P2 * (kd * r1 * L0 + G * bi.y) + t1 * (kd * r1 * Q + G * gq1 - 2.0 * G * Q * r1 * id2);
            const double sg = c_is_a ? 1.0 : -1.0;
            x0b += sg * wv * Tr0; x1b += sg * wv * Tr1;
            ub += sg * wv * K * G * Q * id2;
            pb += -wv * G * L0;
            if (c_is_a) {
                rb += wv * 2.0 * P.nu * G * Q * du * id2;
                Vb_ += w * Vbb * Tin;
                nu_sum += wv * 2.0 * ka.z * G * Q * du * id2;
                gb.x += wv * (-P2 * G * r0 + t1 * G * r0 * r0);
                gb.y += wv * (-P2 * G * r1 + t1 * G * r0 * r1);
                gb.z += wv * (t1 * G * r1 * r0);
                gb.w += wv * (t1 * G * r1 * r1);
            } else {
                Vb_ += w * Va * Tin;
            }
        }
        if (nn > 0) {
            double dp, dc;
            eos_deriv(P, kc.z, dp, dc);
            const double2 sx = A.sx[c], su = A.su[c];
            A.sx[c] = make_double2(sx.x + x0b, sx.y + x1b);
            A.su[c] = make_double2(su.x + ub, su.y);
            A.sr[c] += rb + dp * pb - Vc / kc.z * Vb_;
            if (A.sm) A.sm[c] += Vb_ / kc.z;
            const double4 g = A.gbinv[c];
            A.gbinv[c] = make_double4(g.x + gb.x, g.y + gb.y, g.z + gb.z, g.w + gb.w);
        }
    }
    red[threadIdx.x] = nu_sum;
    __syncthreads();
    for (int k = kAdjThreads / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) nu_part[blockIdx.x] = red[0];
}

// Flags the pair neighbours of the body particles (nflag = 2; the flags are
// cleared before and the ghost flags written after this kernel's use).
template <typename R>
__global__ void k_mark_body_nbrs(Params P, Sorted<R> D) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= P.n_tot || D.itype[b] != SPH_TYPE_BODY) return;
    const int nn = D.npairs[b];
    for (int e = 0; e < nn; ++e) D.nflag[(int)(D.pairs[(size_t)e * P.nbr_stride + b] & 0x7fffffffu)] = 2;
}

// Reverse of k_assign_ghosts, ghost side, one warp per ghost as in the forward
// kernel.  For ghost s with the adjoints of its assigned state (u, v from su; rho
// from sr, i.e. p through rho = (p - pb)/c0^2 + rho0; m from sm) form the
// multipliers of the Shepard sums
//   lam_phi = phibar_int / sum W  (phi = p, u, v, m),
//   lam_w   = -sum_phi lam_phi phi_int        (the normalisation),
// after the reverse of the label mirror and of the shock-release branch (whose
// characteristic form returns the interpolated values for labels -6/-7 and
// pressure 0 for other labels).  Body ghosts: u, v are the body velocity, whose
// adjoint is summed per block with the adjoint of the body acceleration (the
// g.(x - x_j) pressure term) into part[4 blocks].  A second gather gives the
// ghost's position adjoint and flags (nflag = 1) the particles it interpolates
// from for k_adj_ghost_water.  The ghost's su, sr, sm are consumed (the ghost
// state a step starts from is overwritten before use).  Only launched with the
// library's ghost assignment: caller-given ghost states are constant from step
// to step and their adjoints pass through to the step start untouched.
template <typename R>
__global__ void __launch_bounds__(kAdjThreads) k_adj_ghost_lambda(Params P, Sorted<R> D, Adj A,
                                                                  const int* ghost_ids, int n_ghost, double t,
                                                                  double bax, double bay, double* part) {
    __shared__ double red[4][kAdjThreads / 32];
    const int wg = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double bu = 0, bv = 0, ba0 = 0, ba1 = 0;
    if (wg < n_ghost) {
        const int s = D.slot_of[ghost_ids[wg]];
        const bool body = D.itype[s] == SPH_TYPE_BODY;
        const double gxe = P.grav[0] + (body ? bax : 0.0), gye = P.grav[1] + (body ? bay : 0.0);
        // the interpolated values and the weight sum, as the forward assignment of
        // this RHS formed them (k_assign_ghosts kept them in gint / gsw)
        const double4 gi = A.gint[s];
        const double sw = A.gsw[s];
        const double pint = gi.x, uint = gi.y, vint = gi.z, m = gi.w;
        double lp = 0, lu = 0, lv = 0, lm = 0, lw = 0, xs0 = 0, xs1 = 0;
        if (m != 0.0) {
            const double2 ou = A.su[s];
            double pbar = A.sr[s] / P.c0sq, ubar = 0.0, vbar = 0.0;
            if (body) {
                bu = ou.x; bv = ou.y;
            } else {
                const int lab = D.blabel[s];
                double fu = 1.0, fv = 1.0;
                if (lab == -6) { if (P.wall_bc == 1) fv = -1.0; else { fu = -1.0; fv = -1.0; } }
                else if (lab == -7) { fu = -1.0; fv = -1.0; }
                else if (lab == -8) { if (P.wall_bc == 1) fu = -1.0; else { fu = -1.0; fv = -1.0; } }
                ubar = fu * ou.x; vbar = fv * ou.y;
                if (0.0 < t && t <= P.shock_t && lab != -6 && lab != -7) pbar = 0.0;
            }
            const double inv = 1.0 / sw;
            lp = pbar * inv; lu = ubar * inv; lv = vbar * inv; lm = A.sm[s] * inv;
            lw = -(lp * pint + lu * uint + lv * vint + lm * m);
            double a0 = 0.0, a1 = 0.0;
            ghost_visit_warp(P, D, s, [&](int b, double dx, double dy, double q, double w) {
                const double4 kb = D.kin[b];
                const double mb = D.mass[b];
                const double Vb = mb / kb.z, W = w * Vb;
                const double Wb = lp * (kb.w + kb.z * (gxe * dx + gye * dy)) + lu * kb.x + lv * kb.y + lm * mb + lw;
                const double k = Wb * Vb * ghost_dw_over_d(P, q);
                const double cg = lp * kb.z * W;
                xs0 += k * dx + cg * gxe;
                xs1 += k * dy + cg * gye;
                a0 += cg * dx; a1 += cg * dy;
                D.nflag[b] = 1;
            });
            xs0 = warp_sum(xs0); xs1 = warp_sum(xs1);
            a0 = warp_sum(a0); a1 = warp_sum(a1);
            if (body) { ba0 = a0; ba1 = a1; }
        }
        if (lane == 0) {
            A.glam[s] = make_double4(lp, lu, lv, lm);
            A.glamw[s] = lw;
            const double2 sx = A.sx[s];
            A.sx[s] = make_double2(sx.x + xs0, sx.y + xs1);
            A.su[s] = make_double2(0, 0);
            A.sr[s] = 0.0;
            A.sm[s] = 0.0;
        }
    }
    if (lane == 0) { red[0][wib] = bu; red[1][wib] = bv; red[2][wib] = ba0; red[3][wib] = ba1; }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int q = 0; q < 4; ++q) {
            double acc = 0.0;
            for (int w = 0; w < kAdjThreads / 32; ++w) acc += red[q][w];
            part[(size_t)q * gridDim.x + blockIdx.x] = acc;
        }
}

// k_adj_ghost_water for one flagged particle j (all 32 lanes of the warp).
template <typename R>
__device__ __forceinline__ void ghost_water_one(const Params& P, const Sorted<R>& D, const Adj& A, int j, double bax,
                                                double bay) {
    const int lane = threadIdx.x & 31;
    const double2 xj = D.pos[j], x0 = D.pos0[j];
    const int cx = (int)floor((x0.x - P.gx0) / P.cs), cy = (int)floor((x0.y - P.gy0) / P.cs);
    const double4 kj = D.kin[j];
    const double mj = D.mass[j], Vj = mj / kj.z;
    const double hg = P.ghost_h;
    double x0b = 0, x1b = 0, ub = 0, vb = 0, pb = 0, rb = 0;
    const int gx0 = max(cx - P.ghost_cells, 0), gx1 = min(cx + P.ghost_cells, P.gnx - 1);
    for (int gy = max(cy - P.ghost_cells, 0); gy <= min(cy + P.ghost_cells, P.gny - 1); ++gy) {
        const int row = gy * P.gnx;
        int lo = -1, hi = -1;
        for (int gx = gx0; gx <= gx1; ++gx) {
            const int b0 = D.cell_start[row + gx];
            if (b0 < 0) continue;
            if (lo < 0) lo = b0;
            hi = D.cell_end[row + gx];
        }
        if (lo < 0) continue;
        for (int s = lo + lane; s < hi; s += 32) {
            if (D.type[s] != SPH_TYPE_FIX_GHOST || D.id[s] >= P.n_host) continue;
            const double2 x = D.pos[s];
            const double dx = x.x - xj.x, dy = x.y - xj.y;
            const double d = sqrt(dx * dx + dy * dy);
            if (!(d <= P.ghost_r)) continue;
            const double4 lam = A.glam[s];
            const double lw = A.glamw[s];
            if (lam.x == 0.0 && lam.y == 0.0 && lam.z == 0.0 && lam.w == 0.0 && lw == 0.0) continue;
            const double q = d / hg;
            double w;
            if (P.kernel_model == SPH_KERNEL_GAUSSIAN) {
                w = (exp(-(q * q)) - P.gauss_e9) * P.ghost_kf;
            } else {
                const double tq = 1.0 - q / 2.0;
                const double t2 = tq * tq;
                w = P.ghost_kf * (1.0 + 2.0 * q) * (t2 * t2);
            }
            const bool body = D.itype[s] == SPH_TYPE_BODY;
            const double gxe = P.grav[0] + (body ? bax : 0.0), gye = P.grav[1] + (body ? bay : 0.0);
            const double ge = gxe * dx + gye * dy;
            const double W = w * Vj;
            ub += lam.y * W; vb += lam.z * W; pb += lam.x * W;
            rb += lam.x * W * ge;
            const double Wb = lam.x * (kj.w + kj.z * ge) + lam.y * kj.x + lam.z * kj.y + lam.w * mj + lw;
            rb -= Wb * W / kj.z;
            const double k = Wb * Vj * ghost_dw_over_d(P, q);
            const double cg = lam.x * kj.z * W;
            x0b -= k * dx + cg * gxe;
            x1b -= k * dy + cg * gye;
        }
    }
    x0b = warp_sum(x0b); x1b = warp_sum(x1b); ub = warp_sum(ub); vb = warp_sum(vb);
    pb = warp_sum(pb); rb = warp_sum(rb);
    if (lane != 0) return;
    double dp, dc;
    eos_deriv(P, kj.z, dp, dc);
    const double2 sx = A.sx[j], su = A.su[j];
    A.sx[j] = make_double2(sx.x + x0b, sx.y + x1b);
    A.su[j] = make_double2(su.x + ub, su.y + vb);
    A.sr[j] += rb + dp * pb;
}

// Reverse of k_assign_ghosts, interpolated side, one warp per flagged particle j
// (a fixed grid of warps strides over the slots and skips the unflagged ones):
// the lanes split the ghosts of the window around j's list-build cell whose own
// window and radius j falls in (the same cells and the same distance test as the
// forward), adding d(sum_s lam_s . sums_s)/d(x_j, u_j, v_j, rho_j); p_j enters
// through the equation of state, V_j = m_j / rho_j.
template <typename R>
__global__ void __launch_bounds__(kAdjThreads) k_adj_ghost_water(Params P, Sorted<R> D, Adj A, double bax,
                                                                 double bay) {
    // a fixed grid of warps strides over the slots; only the flagged ones work
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < P.n_tot; j += nw) {
        if (D.nflag[j] == 0 || D.type[j] == SPH_TYPE_FIX_GHOST) continue;    // whole warps
        ghost_water_one(P, D, A, j, bax, bay);
    }
}

// Reverse of the step end of the Euler predictor-corrector (stage 11,
// SPH_Time_Iteration.f90:313-394) from the id-order adjoints of the end state
// and of the carried rates:
//   rho' = rho0 + (d1 + d2) dt/2,  u' = v0 + (a1 + a2) dt/2,
//   x'   = x0 + (up + v0) dt/2 + g2 dt + a2 dt^2/2,   carried (d2, a2, g2),
// up the predicted velocity.  Rates of RHS 0 (the predictor's, K1) and RHS 1
// (the corrector's); lxe keeps the adjoint of up for the predictor reverse.
// With shift: the step end then moved the water particles by the capped shift
// of the corrector RHS and corrected their density (as at the end of the
// Runge-Kutta step, k_adj_stage3); its reverse leaves smu, shgr, shbi, and D
// carries that RHS's pass-A outputs.
template <typename R>
__global__ void k_adj_stage_end_ms(Params P, Sorted<R> D, Adj A, double dt, int shift, const double2* ox = nullptr,
                                   const double* orho = nullptr) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.n_tot) return;
    const int i = D.id[s];
    double2 lx = make_double2(0, 0), lv = make_double2(0, 0);
    double lrho = 0.0;
    if (i < P.n_host) { lx = A.lx[i]; lv = A.lv[i]; lrho = A.lrho[i]; }
    // ox / orho: the adjoint of the corrected positions and densities when the
    // step ended with the density re-initialisation (as in k_adj_stage3)
    if (ox) { lx = ox[s]; lrho = orho[s]; shift = 0; }
    if (shift) shift_reverse<R>(P, D, A, s, i, lx, lrho);
    for (int k = 0; k < 2; ++k) {
        A.lr[k][s] = 0.0; A.la[k][s] = make_double2(0, 0); A.lg[k][s] = make_double2(0, 0);
    }
    A.lxe[s] = make_double2(0, 0);
    A.ax0[s] = lx;
    A.ar0[s] = lrho;
    if (i < P.n_host && integrated(P, D.type[s])) {
        const double h2 = 0.5 * dt;
        A.av0[s] = make_double2(lv.x + h2 * lx.x, lv.y + h2 * lx.y);
        A.lxe[s] = make_double2(h2 * lx.x, h2 * lx.y);
        const double2 lka = A.lk_a[i], lkg = A.lk_g[i];
        A.lr[0][s] = h2 * lrho;
        A.la[0][s] = make_double2(h2 * lv.x, h2 * lv.y);
        A.lr[1][s] = h2 * lrho + A.lk_r[i];
        A.la[1][s] = make_double2(h2 * lv.x + h2 * dt * lx.x + lka.x, h2 * lv.y + h2 * dt * lx.y + lka.y);
        A.lg[1][s] = make_double2(dt * lx.x + lkg.x, dt * lx.y + lkg.y);
    } else {
        A.av0[s] = lv;
    }
}

// Reverse of the predictor (stage 10) with the adjoint (sx, su, sr) of the
// predicted state:  xp = x0 + (v0 + g1) dt + a1 dt^2/2,  up = v0 + a1 dt,
// rho_p = rho0 + d1 dt (pred = 1); or, for the state a step starts from (the
// first step's fresh RHS, pred = 0), the plain accumulation.
template <typename R>
__global__ void k_adj_stage_ms(Params P, Sorted<R> D, Adj A, int pred, double dt) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.n_tot) return;
    const double2 sx = A.sx[s], su = A.su[s];
    const double sr = A.sr[s];
    double2 ax = A.ax0[s], av = A.av0[s];
    double ar = A.ar0[s];
    ax.x += sx.x; ax.y += sx.y;
    ar += sr;
    if (pred && D.id[s] < P.n_host && integrated(P, D.type[s])) {
        const double2 le = A.lxe[s];
        const double lu0 = su.x + le.x, lu1 = su.y + le.y;
        av.x += dt * sx.x + lu0; av.y += dt * sx.y + lu1;
        const double2 la = A.la[0][s], lg = A.lg[0][s];
        const double q = 0.5 * dt * dt;
        A.la[0][s] = make_double2(la.x + q * sx.x + dt * lu0, la.y + q * sx.y + dt * lu1);
        A.lg[0][s] = make_double2(lg.x + dt * sx.x, lg.y + dt * sx.y);
        A.lr[0][s] += dt * sr;
    } else {
        av.x += su.x; av.y += su.y;
    }
    A.ax0[s] = ax; A.av0[s] = av; A.ar0[s] = ar;
}

// Per-block sums of the step-start position adjoint of the body particles
// (the body moves by u_body dt at the step start, so dL/du_body += dt times this).
template <typename R>
__global__ void k_adj_body_pos(Params P, Sorted<R> D, Adj A, double* part) {
    __shared__ double red[2][256];
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    double x = 0.0, y = 0.0;
    if (s < P.n_tot && D.itype[s] == SPH_TYPE_BODY && D.id[s] < P.n_host) {
        const double2 a = A.ax0[s];
        x = a.x; y = a.y;
    }
    red[0][threadIdx.x] = x; red[1][threadIdx.x] = y;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if (threadIdx.x < k) { red[0][threadIdx.x] += red[0][threadIdx.x + k]; red[1][threadIdx.x] += red[1][threadIdx.x + k]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) { part[blockIdx.x] = red[0][0]; part[gridDim.x + blockIdx.x] = red[1][0]; }
}

// out[q] += scale * sum_i part[q nparts + i], q < nq, in block order.
__global__ void k_adj_motion_sum(int nparts, int nq, const double* part, double scale, double* out) {
    __shared__ double red[32];
    for (int q = 0; q < nq; ++q) {
        double s = 0.0;
        for (int i = threadIdx.x; i < nparts; i += blockDim.x) s += part[(size_t)q * nparts + i];
        s = block_sum(s, red);
        if (threadIdx.x == 0) out[q] += scale * s;
    }
}

// Drag loss accumulation of the forward run: acc += w * F_x.
__global__ void k_drag_acc(const double* force, double w, double* acc) {
    if (threadIdx.x == 0 && blockIdx.x == 0) acc[0] += w * force[4];
}

}  // namespace sph
