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
    // id order, n_host + images: adjoint of the step-start state carried from
    // step to step, and (host particles) of the rates reused as K1
    double2* lx;
    double2* lv;
    double* lrho;
    double* lk_r;
    double2* lk_a;
};

constexpr int kAdjThreads = 128;

// G(d) of grad_a W = G(d) (x_a - x_b) and dG/dd.
// Gaussian: G = -2 k exp(-q^2)/h^2; Wendland C2: G = -5 k (1 - q/2)^3 / h^2.
__device__ __forceinline__ void kernel_g(const Params& P, double d, double& G, double& dG) {
    const double h = P.h, q = d / h, kf = P.kfactor;
    if (P.kernel_model == SPH_KERNEL_GAUSSIAN) {
        const double ex = exp(-(q * q));
        G = -2.0 * kf * ex / (h * h);
        dG = 4.0 * kf * q * ex / (h * h * h);
    } else {
        const double t = 1.0 - 0.5 * q;
        G = -5.0 * kf * t * t * t / (h * h);
        dG = 7.5 * kf * t * t / (h * h * h);
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
    double t0, t1, t2;    // tau xx, xy, yy
    double g0, g1;        // grad rho
    double4 bi;           // B^-1
    bool water, near;
};

template <typename R>
__device__ __forceinline__ PSide load_side(const Sorted<R>& D, int s) {
    PSide o;
    o.x = D.pos[s];
    const double4 k = D.kin[s];
    o.u = k.x; o.v = k.y; o.rho = k.z; o.p = k.w;
    const typename VT<R>::V4 ax = D.aux[s];
    o.m = D.mass[s];
    o.V = o.m / o.rho;
    o.c = (double)ax.z;
    o.sm = (double)ax.w;
    const typename VT<R>::V4 n1 = D.nb1[s];
    o.t0 = (double)n1.x; o.t1 = (double)n1.y; o.t2 = (double)n1.z; o.g0 = (double)n1.w;
    o.g1 = (double)D.nb2[s].x;
    o.bi = D.binv64[s];
    o.water = D.type[s] == SPH_TYPE_WATER;
    o.near = (D.flags[s] & 2) != 0;
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
};

// Reverse of the contribution of b to particle a (a water particle) with the
// adjoints lr (of drho_a) and (l0, l1) (of acc_a).
__device__ __forceinline__ void rev_pair(const Params& P, const PSide& A, const PSide& B, double lr, double l0,
                                         double l1, PBar& o) {
    const double r0 = A.x.x - B.x.x, r1 = A.x.y - B.x.y;
    const double d2 = r0 * r0 + r1 * r1, d = sqrt(d2), id = 1.0 / d, id2 = id * id;
    double G, dG;
    kernel_g(P, d, G, dG);
    const double n0 = A.bi.x * r0 + A.bi.y * r1, n1 = A.bi.z * r0 + A.bi.w * r1;
    const double s = r0 * n0 + r1 * n1;
    const double du0 = A.u - B.u, du1 = A.v - B.v, dp = A.p - B.p, drho = A.rho - B.rho;
    const double vx = du0 * r0 + du1 * r1;
    const double dU = -vx * id;
    const double rbar = 0.5 * (A.rho + B.rho), cbar = 0.5 * (A.c + B.c);
    const double c0 = P.sqrt_c0;
    const double Pbar = 0.5 * (A.p + B.p);
    // Riemann state
    double PA, w0, w1, bR = 0.0, kk = 0.0;
    bool take_m3 = false;
    if (A.near) {
        PA = Pbar; w0 = 0.5 * du0; w1 = 0.5 * du1;
    } else {
        const double m3 = 3.0 * fmax(dU, 0.0);
        take_m3 = m3 < cbar;
        bR = take_m3 ? m3 : cbar;
        PA = Pbar + 0.5 * bR * rbar * dU;
        kk = dp / (2.0 * rbar * c0 * d);
        w0 = 0.5 * du0 + kk * r0; w1 = 0.5 * du1 + kk * r1;
    }
    const double rhoij = 1.0 / (A.rho * B.rho);
    const double fp = -2.0 * PA * B.m * rhoij;
    const bool av = vx < 0.0;
    const double fh2 = (P.fai * P.h) * (P.fai * P.h);
    const double den_phi = d2 + fh2;
    double phi = 0.0, Pi = 0.0;
    if (av) {
        phi = P.h * vx / den_phi;
        Pi = (-P.alpha * cbar * phi + P.beta * (phi * phi)) / rbar;
    }
    const double Kt = P.delta_alpha * P.h * P.rho0;
    const double tt = Kt * cbar * vx * id2 / A.rho * B.V;
    const double Cn = fp - (av ? B.m * Pi : 0.0) + tt;
    const double lf = 2.0 * P.nu * B.V * G * s * id2;
    const double Ln = l0 * n0 + l1 * n1;

    double Gb = 0, n0b = 0, n1b = 0, sb = 0, db = 0, r0b = 0, r1b = 0;
    double du0b = 0, du1b = 0, dpb = 0, rab = 0, rbb = 0, Pbarb = 0, rbarb = 0, cbarb = 0, Vbb = 0, vxb = 0, dUb = 0;
    o.t0 = o.t1 = o.t2 = o.g0 = o.g1 = 0.0;
    // acc = Cn G n + lf (u_a - u_b) + SPS
    const double Cnb = G * Ln;
    Gb += Cn * Ln;
    n0b += Cn * G * l0; n1b += Cn * G * l1;
    const double lfb = l0 * du0 + l1 * du1;
    du0b += lf * l0; du1b += lf * l1;
    {
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
        rab -= rhoijb * rhoij / A.rho; rbb -= rhoijb * rhoij / B.rho;
    }
    // C = fp - [av] m_b Pi + tt
    const double PAb0 = -2.0 * B.m * rhoij * Cnb;
    rab -= fp / A.rho * Cnb; rbb -= fp / B.rho * Cnb;
    if (av) {
        const double Pib = -B.m * Cnb;
        cbarb += -P.alpha * phi / rbar * Pib;
        const double phib = (-P.alpha * cbar + 2.0 * P.beta * phi) / rbar * Pib;
        rbarb -= Pi / rbar * Pib;
        vxb += P.h / den_phi * phib;
        db -= phi * 2.0 * d / den_phi * phib;
    }
    {
        const double base = Kt * id2 / A.rho;
        cbarb += base * vx * B.V * Cnb;
        vxb += base * cbar * B.V * Cnb;
        Vbb += base * cbar * vx * Cnb;
        db -= 2.0 * tt * id * Cnb;
        rab -= tt / A.rho * Cnb;
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
        if (A.water) {
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
    du0b += 0.5 * w0b; du1b += 0.5 * w1b;
    Pbarb += PAb0;
    if (!A.near) {
        const double kkb = w0b * r0 + w1b * r1;
        r0b += kk * w0b; r1b += kk * w1b;
        dpb += kkb / (2.0 * rbar * c0 * d);
        rbarb -= kk / rbar * kkb;
        db -= kk * id * kkb;
        const double bRb = 0.5 * rbar * dU * PAb0;
        rbarb += 0.5 * bR * dU * PAb0;
        dUb += 0.5 * bR * rbar * PAb0;
        if (take_m3) { if (dU > 0.0) dUb += 3.0 * bRb; }
        else cbarb += bRb;
    }
    // dU = -vx/d, vx = (u_a - u_b).r
    vxb -= dUb * id;
    db += vx * id2 * dUb;
    du0b += vxb * r0; du1b += vxb * r1;
    r0b += vxb * du0; r1b += vxb * du1;
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
    o.ca = 0.5 * cbarb; o.cb = 0.5 * cbarb;
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
constexpr int kAdjLanes = SPH_ADJ_LANES;     // 2 or 4
template <typename R>
__global__ void __launch_bounds__(kAdjThreads, SPH_ADJ_C_MIN_BLOCKS) k_adj_c(Params P, Sorted<R> D, Adj A, const double* lr,
                                                        const double2* la, double* nu_part) {
    __shared__ double red[kAdjThreads];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = t / kAdjLanes;
    const int role = t & 1, par = (t >> 1) & (kAdjLanes / 2 - 1);
    double nu_sum = 0.0;
    // every lane of the warp takes part in the shuffles below
    const bool live = c < P.n_tot;
    double v[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) v[q] = 0.0;
    if (live) {
        const int nn = D.npairs[c];
        // both roles run the same instructions: the two sides are loaded by
        // index (c's records stay in L1), not branched on
        const double sg = role ? -1.0 : 1.0;
        for (int e = par; e < nn; e += kAdjLanes / 2) {
            const int b = (int)(D.pairs[(size_t)e * P.nbr_stride + c] & 0x7fffffffu);
            const int acc_at = role ? b : c;         // the particle whose sum is differentiated
            const int other = role ? c : b;
            if (D.type[acc_at] != SPH_TYPE_WATER) continue;
            const double l_r = lr[acc_at];
            const double2 l_a = la[acc_at];
            if (l_r == 0.0 && l_a.x == 0.0 && l_a.y == 0.0) continue;
            const PSide Sa = load_side(D, acc_at);
            const PSide Sb = load_side(D, other);
            PBar o;
            rev_pair(P, Sa, Sb, l_r, l_a.x, l_a.y, o);
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
        }
    }
#pragma unroll
    for (int q = 0; q < 17; ++q) {
        v[q] += __shfl_xor_sync(0xffffffffu, v[q], 1);
        if (kAdjLanes == 4) v[q] += __shfl_xor_sync(0xffffffffu, v[q], 2);
    }
    if (live && (t & (kAdjLanes - 1)) == 0) {
        const double4 k = D.kin[c];
        const double rho = k.z, V = D.mass[c] / rho;
        double dp, dc;
        eos_deriv(P, rho, dp, dc);
        A.sx[c] = make_double2(v[0], v[1]);
        A.su[c] = make_double2(v[2], v[3]);
        A.sr[c] = v[6] + dp * v[4] + dc * v[5] - V / rho * v[7];
        A.gbinv[c] = make_double4(v[13], v[14], v[15], v[16]);
        A.ggr[c] = make_double2(v[11], v[12]);
        A.gtau[c] = make_double4(v[8], v[9], v[10], 0.0);
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
__global__ void k_adj_nu_sum(int nparts, const double* part, double* acc) {
    __shared__ double red[256];
    double s = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) s += part[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) acc[0] += red[0];
}

// Reverse of the per-particle end of pass A.
template <typename R>
__global__ void k_adj_point(Params P, Sorted<R> D, Adj A) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= P.n_tot) return;
    const int ta = D.type[a];
    const double4 bi = D.binv64[a];
    const typename VT<R>::V4 n1 = D.nb1[a], n2 = D.nb2[a], n3 = D.nb3[a];
    // normalised gradients of pass A: rho (n1.w, n2.x), u (n2.w, n3.x), v (n3.y, n3.z)
    const double gr0 = (double)n1.w, gr1 = (double)n2.x;
    const double gu0 = (double)n2.w, gu1 = (double)n3.x;
    const double gv0 = (double)n3.y, gv1 = (double)n3.z;
    const double2 ggr = A.ggr[a];
    double Gr0 = ggr.x, Gr1 = ggr.y, Gu0 = 0, Gu1 = 0, Gv0 = 0, Gv1 = 0;
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
        Gu0 = sxxb; Gu1 = sxyb; Gv0 = sxyb; Gv1 = syyb;
    }
    // grad = B^-1 g: adjoint of g = B^-T adjoint of grad
    auto mt = [&](double x, double y, double& ox, double& oy) {
        ox = bi.x * x + bi.z * y;
        oy = bi.y * x + bi.w * y;
    };
    double m0, m1, m2, m3, m4, m5;
    mt(Gr0, Gr1, m0, m1);
    mt(Gu0, Gu1, m2, m3);
    mt(Gv0, Gv1, m4, m5);
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
        double qr0, qr1, qu0, qu1, qv0, qv1;
        raw(gr0, gr1, qr0, qr1);
        raw(gu0, gu1, qu0, qu1);
        raw(gv0, gv1, qv0, qv1);
        const double4 gb = A.gbinv[a];
        // adjoint of B^-1: from pass C and from grad = B^-1 g
        const double Y00 = gb.x + Gr0 * qr0 + Gu0 * qu0 + Gv0 * qv0;
        const double Y01 = gb.y + Gr0 * qr1 + Gu0 * qu1 + Gv0 * qv1;
        const double Y10 = gb.z + Gr1 * qr0 + Gu1 * qu0 + Gv1 * qv0;
        const double Y11 = gb.w + Gr1 * qr1 + Gu1 * qu1 + Gv1 * qv1;
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
// pair term of pass A's raw sums at particle a.  Returns f / V_b and its
// gradient with respect to r divided by V_b.
__device__ __forceinline__ void rev_rawsum(const Params& P, double r0, double r1, double dr, double du, double dv,
                                           const double4& m1, const double4& m2, const double2& m3, double& S_G,
                                           double& fr0, double& fr1, double& G) {
    const double d = sqrt(r0 * r0 + r1 * r1);
    double dG;
    kernel_g(P, d, G, dG);
    const double c0 = dr * m1.x + du * m1.z + dv * m2.x;   // sum_phi dphi mu_phi (x)
    const double c1 = dr * m1.y + du * m1.w + dv * m2.y;
    const double Mr0 = m2.z * r0 + m2.w * r1, Mr1 = m3.x * r0 + m3.y * r1;
    const double MTr0 = m2.z * r0 + m3.x * r1, MTr1 = m2.w * r0 + m3.y * r1;
    const double S = c0 * r0 + c1 * r1 - (r0 * Mr0 + r1 * Mr1);
    S_G = S;
    const double k = dG * S / d;
    fr0 = k * r0 + G * (c0 - Mr0 - MTr0);
    fr1 = k * r1 + G * (c1 - Mr1 - MTr1);
}

// Reverse of pass A's raw pair sums, then of the stage that produced the
// state this RHS was evaluated on.
template <typename R>
__global__ void __launch_bounds__(kAdjThreads) k_adj_a(Params P, Sorted<R> D, Adj A, int stage, double dt) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n_tot) return;
    const double2 xc = D.pos[c];
    const double4 kc = D.kin[c];
    const double Vc = D.mass[c] / kc.z;
    const double4 mc1 = A.mu1[c], mc2 = A.mu2[c];
    const double2 mc3 = A.mu3[c];
    double x0b = 0, x1b = 0, ub = 0, vb = 0, rb = 0, Vb = 0;
    const int nn = D.npairs[c];
    for (int e = 0; e < nn; ++e) {
        const int b = (int)(D.pairs[(size_t)e * P.nbr_stride + c] & 0x7fffffffu);
        const double2 xb = D.pos[b];
        const double4 kb = D.kin[b];
        const double r0 = xc.x - xb.x, r1 = xc.y - xb.y;
        // own sums: phi_b - phi_c, weight V_b
        {
            const double Vbn = D.mass[b] / kb.z;
            double S, f0, f1, G;
            rev_rawsum(P, r0, r1, kb.z - kc.z, kb.x - kc.x, kb.y - kc.y, mc1, mc2, mc3, S, f0, f1, G);
            x0b += Vbn * f0; x1b += Vbn * f1;
            rb -= Vbn * G * (mc1.x * r0 + mc1.y * r1);
            ub -= Vbn * G * (mc1.z * r0 + mc1.w * r1);
            vb -= Vbn * G * (mc2.x * r0 + mc2.y * r1);
        }
        // neighbour's sums: phi_c - phi_b at r' = -r, weight V_c
        {
            const double4 mb1 = A.mu1[b], mb2 = A.mu2[b];
            const double2 mb3 = A.mu3[b];
            double S, f0, f1, G;
            rev_rawsum(P, -r0, -r1, kc.z - kb.z, kc.x - kb.x, kc.y - kb.y, mb1, mb2, mb3, S, f0, f1, G);
            x0b -= Vc * f0; x1b -= Vc * f1;
            rb -= Vc * G * (mb1.x * r0 + mb1.y * r1);
            ub -= Vc * G * (mb1.z * r0 + mb1.w * r1);
            vb -= Vc * G * (mb2.x * r0 + mb2.y * r1);
            Vb += G * S;
        }
    }
    const double2 sx = A.sx[c], su = A.su[c];
    stage_reverse(P, D, A, c, stage, dt, make_double2(sx.x + x0b, sx.y + x1b), make_double2(su.x + ub, su.y + vb),
                  A.sr[c] + rb - Vc / kc.z * Vb);
}

// Reverse of stage 3 (the step end) from the id-order adjoints of the end state
// and of the carried rates.  Non-integrated host particles keep their state.
template <typename R>
__global__ void k_adj_stage3(Params P, Sorted<R> D, Adj A, double dt) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.n_tot) return;
    const int i = D.id[s];
    double2 lx = make_double2(0, 0), lv = make_double2(0, 0);
    double lrho = 0.0;
    if (i < P.n_host) { lx = A.lx[i]; lv = A.lv[i]; lrho = A.lrho[i]; }
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
        if (type[i] != SPH_TYPE_WATER) continue;
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
// and carried rates do not enter the loss.
__global__ void k_adj_seed(int n, int kind, double dloss, const int* type, const double2* vel, const double* mass,
                           const double2* target, Adj A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double2 g = make_double2(0, 0);
    if (type[i] == SPH_TYPE_WATER) {
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
}

}  // namespace sph
