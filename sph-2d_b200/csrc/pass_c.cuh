// pass_c.cuh -- neighbour pass C: the fused force pass.  One thread per
// particle gathers, for every pair neighbour, the linear-Riemann flux (with
// optional MUSCL reconstruction), continuity, pressure force, Monaghan
// artificial viscosity, Morris laplacian, delta-alpha term, SPS force, XSPH,
// delta-SPH density diffusion and (on the last RHS of a step) the shifting sum.
//
// Reference loops (all in pair order, scattered to pair_i and pair_j):
//   Solver_Normalized_Modified_Linear_Riemann_Delta_SPS.f90:300-502, 552-583, 627-635
//   Solver_Normalized_MUSCL_Linear_Riemann_Delta_SPS.f90:458-682, 690-721
//   MUSCL_Limiter: function_module.f90:34-80
//   Shift_particle_position.f90:78-103
//   assembly: single_step_compute.f90:152-171
//
// Every pair quantity is evaluated in the reference's own orientation
// (pair_i = the particle with the lower id, bit 31 of the list entry), so the
// flux seen by the two particles of a pair is computed by the identical
// sequence of operations the Fortran uses; each thread then keeps the
// pair_i or pair_j contribution that belongs to its particle.
#pragma once
#include "pass_a.cuh"

namespace sph {

template <typename R>
__device__ __forceinline__ void muscl_limiter(R di, R dj, R dij, R& li, R& lj) {
    const R beta_lim = R(1.3);
    const R diff = R(0.5);
    R fi, fj, lim;
    if (dj > R(0)) {
        lim = max(R(0), max(min(beta_lim * di, dj), min(di, beta_lim * dj)));
        if (lim > R(0.5) * dij && fabs(lim) > R(0)) {
            if (di > dj) { fi = diff; fj = R(0); } else { fi = R(0); fj = diff; }
            li = dij * fi; lj = dij * fj;
        } else { li = lim; lj = lim; }
    } else {
        lim = min(R(0), min(max(beta_lim * di, dj), max(di, beta_lim * dj)));
        if (lim < R(0.5) * dij && fabs(lim) > R(0)) {
            if (di < dj) { fi = diff; fj = R(0); } else { fi = R(0); fj = diff; }
            li = dij * fi; lj = dij * fj;
        } else { li = lim; lj = lim; }
    }
}

// Per-particle state a thread needs for "its" side of a pair.
template <typename R>
struct Side {
    using V4 = typename VT<R>::V4;
    V4 kin;     // u, v, rho-ish, p
    V4 aux;     // m, V, c, smass
    V4 nb1, nb2, nb3;
    R rho;
};

template <typename R, bool MUSCL>
__global__ void __launch_bounds__(128) k_pass_c(Params P, Sorted<R> D, int last_rhs) {
    using V4 = typename VT<R>::V4;
    using V2 = typename VT<R>::V2;
    using A = typename Acc<R>::T;
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= P.n_tot) return;
    const int ta = D.type[a];
    const int nn = D.nnbr[a];
    const double2 xa = D.pos[a];
    Side<R> S;
    S.kin = D.kin[a]; S.aux = D.aux[a]; S.nb1 = D.nb1[a]; S.nb2 = D.nb2[a];
    if (MUSCL) S.nb3 = D.nb3[a];
    S.rho = Dens<R>::rho(S.kin.z, P.rho0);
    const V4 bi = D.binv[a];
    const bool near_a = (D.flags[a] & 2) != 0;

    const R hbar = (R)P.h;
    const R sqc0 = (R)P.sqrt_c0;
    const R nu = (R)P.nu, alpha = (R)P.alpha, beta = (R)P.beta, fai = (R)P.fai;
    const R dlt = (R)P.delta, dla = (R)P.delta_alpha, rho0 = (R)P.rho0, eps = (R)P.eps;
    const R wdx_inv = (R)(1.0 / P.w_dx);
    const R shf = (R)(P.shift_beta * (P.h * P.h));
    const R shR = (R)P.shift_R;

    // accumulators: continuity, delta-SPH, internal, AV, laplacian, art. internal, SPS, XSPH, shift
    A cont, corr, ix, iy, avx, avy, lpx, lpy, arx, ary, spx, spy, xsx, xsy, shx, shy;
    cont.init(); corr.init(); ix.init(); iy.init(); avx.init(); avy.init(); lpx.init(); lpy.init();
    arx.init(); ary.init(); spx.init(); spy.init(); xsx.init(); xsy.init(); shx.init(); shy.init();

    for (int e = 0; e < nn; ++e) {
        const unsigned ent = __ldg(&D.nbr[(size_t)e * P.nbr_stride + a]);
        const int b = (int)(ent & 0x7fffffffu);
        const bool a_is_i = (ent >> 31) != 0;
        const double2 xb = __ldg(&D.pos[b]);
        const double dxd = xa.x - xb.x, dyd = xa.y - xb.y;
        double dd;
        if (!in_support(P, dxd, dyd, dd)) continue;
        Side<R> T;
        T.kin = D.kin[b]; T.aux = D.aux[b]; T.nb1 = D.nb1[b]; T.nb2 = D.nb2[b];
        if (MUSCL) T.nb3 = D.nb3[b];
        T.rho = Dens<R>::rho(T.kin.z, P.rho0);
        // canonical orientation: I = pair_i, J = pair_j
        const Side<R>& I = a_is_i ? S : T;
        const Side<R>& J = a_is_i ? T : S;
        const R sgn = a_is_i ? R(1) : R(-1);
        // position_difference_ij = x_i - x_j, distance, w, dwdx (find_particle_pair.f90:79-107)
        const R xij0 = (R)(a_is_i ? dxd : -dxd), xij1 = (R)(a_is_i ? dyd : -dyd);
        const R d = (R)dd;
        R w, dw0, dw1;
        kernel_w_dw<R>(P, d, xij0, xij1, w, dw0, dw1);
        // Normalized_dwdx of this particle's side: B_a^-1 dwdx(k)
        const R nd0 = bi.x * dw0 + bi.y * dw1;
        const R nd1 = bi.z * dw0 + bi.w * dw1;
        const R cbar = (I.aux.z + J.aux.z) / R(2);
        const R rbar = (I.rho + J.rho) / R(2);
        const R ui = I.kin.x, vi = I.kin.y, uj = J.kin.x, vj = J.kin.y;
        const R pi_ = I.kin.w, pj_ = J.kin.w;
        R PL, PR, Pbar, vI0, vI1, vJ0, vJ1, vb0, vb1, e0, e1;
        if (!MUSCL) {
            PL = pi_; PR = pj_; Pbar = (PL + PR) / R(2);
            vI0 = ui; vI1 = vi; vJ0 = uj; vJ1 = vj;
            vb0 = (vI0 + vJ0) / R(2); vb1 = (vI1 + vJ1) / R(2);
            e0 = -xij0 / d; e1 = -xij1 / d;
        } else {
            const R x0 = -xij0, x1 = -xij1;          // j - i
            e0 = x0 / d; e1 = x1 / d;
            R li, lj;
            // I.nb2 = (grad rho y, grad p x, grad p y, grad u x), I.nb3 = (grad u y, grad v x, grad v y, 0)
            R Di = R(0.5) * (I.nb2.y * x0 + I.nb2.z * x1);
            R Dj = R(-0.5) * (J.nb2.y * x0 + J.nb2.z * x1);
            muscl_limiter<R>(Di, Dj, pj_ - pi_, li, lj);
            PL = pi_ + li; PR = pj_ - lj; Pbar = (pi_ + pj_) / R(2);
            const R vd0 = -(ui - uj), vd1 = -(vi - vj);
            Di = R(0.5) * (I.nb2.w * x0 + I.nb3.x * x1);
            Dj = R(-0.5) * (J.nb2.w * x0 + J.nb3.x * x1);
            muscl_limiter<R>(Di, Dj, vd0, li, lj);
            vI0 = ui + li; vJ0 = uj - lj;
            Di = R(0.5) * (I.nb3.y * x0 + I.nb3.z * x1);
            Dj = R(-0.5) * (J.nb3.y * x0 + J.nb3.z * x1);
            muscl_limiter<R>(Di, Dj, vd1, li, lj);
            vI1 = vi + li; vJ1 = vj - lj;
            vb0 = (ui + uj) / R(2); vb1 = (vi + vj) / R(2);
        }
        const R UL = vI0 * e0 + vI1 * e1;
        const R UR = vJ0 * e0 + vJ1 * e1;
        const R Ubar = (UL + UR) / R(2);
        const R Us = Ubar + R(0.5) * (PL - PR) / (rbar * sqc0);
        const R vs0 = (Us - Ubar) * e0 + vb0, vs1 = (Us - Ubar) * e1 + vb1;
        const R bR = min(R(3) * (max((UL - UR), R(0))), cbar);
        const R Ps = Pbar + R(0.5) * bR * rbar * (UL - UR);
        // this side's star state (near-free-surface particles use the averages)
        const R vA0 = near_a ? vb0 : vs0, vA1 = near_a ? vb1 : vs1, PA = near_a ? Pbar : Ps;
        const R va0 = a_is_i ? vI0 : vJ0, va1 = a_is_i ? vI1 : vJ1;
        const R Vb = T.aux.y, mb = T.aux.x;
        // continuity (:360-369)
        R tm = (va0 - vA0) * nd0 + (va1 - vA1) * nd1;
        if (!a_is_i) tm = -tm;
        cont.add(R(2) * S.rho * Vb * tm);
        // pressure force (:374-388)
        const R rho_ij = R(1) / (I.rho * J.rho);
        ix.add(sgn * (mb * (R(-2) * PA * nd0 * rho_ij)));
        iy.add(sgn * (mb * (R(-2) * PA * nd1 * rho_ij)));
        // artificial viscosity (:392-417)
        const R vij0 = ui - uj, vij1 = vi - vj;
        const R r2 = xij0 * xij0 + xij1 * xij1;
        const R vx = vij0 * xij0 + vij1 * xij1;
        if (vx < R(0)) {
            const R fh = fai * hbar;
            const R phi1 = hbar * vx / (r2 + fh * fh);
            const R Pi = (-alpha * cbar * phi1 + beta * (phi1 * phi1)) / rbar;
            avx.add(sgn * (mb * (-Pi * nd0)));
            avy.add(sgn * (mb * (-Pi * nd1)));
        }
        // Morris laplacian (:432-436)
        const R rd = xij0 * nd0 + xij1 * nd1;
        const R lf = Vb * R(2) * nu * rd / r2;
        lpx.add(sgn * (lf * vij0));
        lpy.add(sgn * (lf * vij1));
        // delta-alpha artificial internal acceleration (:442-446)
        const R tt = dla * hbar * cbar * vx / r2;
        arx.add(sgn * (tt * nd0 * rho0 / S.rho * Vb));
        ary.add(sgn * (tt * nd1 * rho0 / S.rho * Vb));
        // SPS force, unnormalised dwdx and the neighbour's SPS mass (:450-492)
        const R sxx = I.nb1.x + J.nb1.x, sxy = I.nb1.y + J.nb1.y, syy = I.nb1.z + J.nb1.z;
        R tp = (sxx * dw0 + sxy * dw1) * rho_ij;
        const R smb = T.aux.w;
        spx.add(sgn * (smb * tp));
        if (!P.quirks) tp = R(0);
        tp = (tp + syy * dw1 + sxy * dw0) * rho_ij;
        spy.add(sgn * (smb * tp));
        // XSPH average velocity (:495-500; modified solver only)
        if (!MUSCL && P.xsph) {
            const R f = eps * R(2) * mb / (I.rho + J.rho) * w;
            xsx.add(-sgn * (f * vij0));
            xsy.add(-sgn * (f * vij1));
        }
        // delta-SPH density diffusion (:552-583), x_j - x_i and grad rho of both
        {
            const R p0 = -xij0, p1 = -xij1;
            const R drho = sizeof(R) == 8 ? (J.rho - I.rho) : (J.kin.z - I.kin.z);
            const R sg0 = I.nb1.w + J.nb1.w, sg1 = I.nb2.x + J.nb2.x;
            const R psi = drho - R(0.5) * (sg0 * p0 + sg1 * p1);
            const R tma = (p0 * nd0 + p1 * nd1) / r2;
            corr.add(sgn * (R(2) * dlt * hbar * cbar * psi * tma * Vb));
        }
        // particle shifting sum (Shift_particle_position.f90:97-100)
        if (last_rhs) {
            const R r = w * wdx_inv;
            const R f = shf * (R(1) + shR * pw4(r));
            shx.add(-sgn * (f * nd0 * Vb));
            shy.add(-sgn * (f * nd1 * Vb));
        }
    }
    // assembly (single_step_compute.f90:152-171, Solver :627-635)
    R drho = cont.val();
    R ax = R(0), ay = R(0);
    if (ta == SPH_TYPE_WATER) {
        ax = ix.val() + R(0) + avx.val() + arx.val() + spx.val() + lpx.val();
        ay = iy.val() + R(0) + avy.val() + ary.val() + spy.val() + lpy.val();
        drho = drho + corr.val();
    }
    D.drho[a] = drho;
    D.acc[a] = mk2<R>(ax, ay);
    D.avg[a] = mk2<R>(xsx.val(), xsy.val());
    if (last_rhs) D.shift[a] = mk2<R>(shx.val(), shy.val());
}

}  // namespace sph
