// update.cuh -- integrator stages, shifting, diagnostics reductions, pair
// enumeration for the find_particle_pair entry point, and layout conversions.
#pragma once
#include "pass_c.cuh"

namespace sph {

// Runge-Kutta stages of time_iteration.f90 (water particles only; images and
// boundary particles keep their step-start state, as the reference only
// updates type 2 at :944, :978, :1008, :1038):
//   stage 0  rho = rho0 + drhodt*dt/2, v = v0 + 0.5 dt a + avg, x = x0 + 0.5 dt v    K = K1
//   stage 1  same with the second RHS                                          K += 2 K2
//   stage 2  full dt with the third RHS                                        K += 2 K3
//   stage 3  rho = rho0 + (K + drhodt) dt/6, v = v0 + (K_a + a) dt/6 + avg,
//            x = x0 + (K_v + v) dt/6 + 0.5 dt^2 a; then Shift_particle_position.
// Stage 0 uses the rates carried from the previous step (K1 reuse, :940-965)
// unless this is the first step, when a fresh RHS precedes it (:821).
//
// With SPH_INTEGRATOR_EULER_PC (Moving_Square.../SPH_Time_Iteration.f90:304-334) the
// stages are 10 (predictor) and 11 (corrector):
//   predictor  rho = rho0 + drhodt dt, x = x0 + dt (v0 + avg) + 0.5 a dt^2, v = v0 + dt a
//   corrector  rho = rho0 + 0.5 (drhodt + drhodt_p) dt,
//              x = x0 + 0.5 dt (v_p + v0) + avg dt + 0.5 a dt^2, v = v0 + 0.5 dt (a + a_p)
// Shift_particle_position.f90:108-131: the capped displacement of the last RHS's
// shifting sum and the first-order density correction, for water particles
// that are not near the free surface.
template <typename R>
__device__ __forceinline__ void apply_shift(const Params& P, const Sorted<R>& D, int s, double& x, double& y,
                                            double& rho) {
    if (D.type[s] != SPH_TYPE_WATER || (D.flags[s] & 2)) return;
    const double2 sh = D.shift[s];
    double s0 = sh.x, s1 = sh.y;
    const double amp = sqrt(s0 * s0 + s1 * s1);
    if (amp > P.shift_max) { s0 = s0 / amp * P.shift_max; s1 = s1 / amp * P.shift_max; }
    x = x + s0;
    y = y + s1;
    rho = rho + grad_scale<R>() * D.nb1[s].w * s0;
    rho = rho + grad_scale<R>() * D.nb2[s].x * s1;
}

template <typename R>
// to_staging (final stages of the Taylor-Green driver): also write the new
// master state and carried rates of each host particle to the id-order staging
// arrays, exactly what k_unsort would copy there, so the next step's set-up and
// a state read need no unsort pass (static fields are unchanged in staging).
__global__ void k_stage(Params P, Sorted<R> D, int stage, double dt, int use_carried, int do_shift,
                        unsigned* status, Staging S, int to_staging) {
    using V2 = typename VT<R>::V2;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.n_tot) return;
    if (!integrated(P, D.type[s])) return;
    const double2 x0 = D.pos0[s];
    const double2 v0 = D.vel0[s];
    const double r0 = D.rho0[s];
    double dr, ax, ay, gx, gy;
    if ((stage == 0 || stage == 10) && use_carried) {   // the first stage of either driver
        dr = (double)D.c_drho[s]; V2 a = D.c_acc[s], g = D.c_avg[s];
        ax = (double)a.x; ay = (double)a.y; gx = (double)g.x; gy = (double)g.y;
    } else {
        dr = (double)D.drho[s]; V2 a = D.acc[s], g = D.avg[s];
        ax = (double)a.x; ay = (double)a.y; gx = (double)g.x; gy = (double)g.y;
    }
    double rho, u, v, x, y;
    if (stage == 10) {
        rho = r0 + dr * dt;
        x = x0.x + dt * (v0.x + gx) + 0.5 * ax * (dt * dt);
        y = x0.y + dt * (v0.y + gy) + 0.5 * ay * (dt * dt);
        u = v0.x + dt * ax;
        v = v0.y + dt * ay;
        D.ks_r[s] = (R)dr;
        D.ks_a[s] = mk2<R>((R)ax, (R)ay);
        D.ks_v[s] = v0;
    } else if (stage == 11) {
        const double4 kp = D.kin[s];          // predicted velocity
        const V2 ka = D.ks_a[s];
        const double2 kv = D.ks_v[s];
        rho = r0 + 0.5 * (dr + (double)D.ks_r[s]) * dt;
        x = x0.x + 0.5 * dt * (kp.x + kv.x) + gx * dt + 0.5 * ax * (dt * dt);
        y = x0.y + 0.5 * dt * (kp.y + kv.y) + gy * dt + 0.5 * ay * (dt * dt);
        u = v0.x + 0.5 * dt * (ax + (double)ka.x);
        v = v0.y + 0.5 * dt * (ay + (double)ka.y);
        D.c_drho[s] = (R)dr;
        D.c_acc[s] = mk2<R>((R)ax, (R)ay);
        D.c_avg[s] = mk2<R>((R)gx, (R)gy);
    } else if (stage < 3) {
        const double f = stage < 2 ? 0.5 * dt : dt;
        rho = stage < 2 ? r0 + dr * dt / 2 : r0 + dr * dt;
        u = v0.x + f * ax + gx;
        x = x0.x + f * u;
        v = v0.y + f * ay + gy;
        y = x0.y + f * v;
        if (stage == 0) {
            D.ks_r[s] = (R)dr;
            D.ks_a[s] = mk2<R>((R)ax, (R)ay);
            D.ks_v[s] = make_double2(u, v);
        } else {
            D.ks_r[s] = D.ks_r[s] + R(2) * (R)dr;
            V2 ka = D.ks_a[s];
            double2 kv = D.ks_v[s];
            D.ks_a[s] = mk2<R>(ka.x + R(2) * (R)ax, ka.y + R(2) * (R)ay);
            D.ks_v[s] = make_double2(kv.x + 2 * u, kv.y + 2 * v);
        }
    } else {
        const V2 ka = D.ks_a[s];
        const double2 kv = D.ks_v[s];
        rho = r0 + ((double)D.ks_r[s] + dr) * dt / 6.0;
        u = v0.x + ((double)ka.x + ax) * dt / 6.0 + gx;
        x = x0.x + ((double)kv.x + u) * dt / 6.0 + 0.5 * dt * dt * ax;
        v = v0.y + ((double)ka.y + ay) * dt / 6.0 + gy;
        y = x0.y + ((double)kv.y + v) * dt / 6.0 + 0.5 * dt * dt * ay;
        // rates of this last RHS become next step's K1
        D.c_drho[s] = (R)dr;
        D.c_acc[s] = mk2<R>((R)ax, (R)ay);
        D.c_avg[s] = mk2<R>((R)gx, (R)gy);
    }
    // the neighbour lists stay exact while nobody moved more than half the skin
    const double ddx = x - x0.x, ddy = y - x0.y;
    if (ddx * ddx + ddy * ddy > P.skin_half2) atomicOr(status, ST_SKIN);
    const bool final_stage = stage == 3 || stage == 11;
    if (final_stage) {
        if (do_shift) apply_shift(P, D, s, x, y, rho);
        if (!(isfinite(x) && isfinite(y) && isfinite(u) && isfinite(v) && isfinite(rho))) atomicOr(status, ST_NONFINITE);
        D.pos0[s] = make_double2(x, y);
        D.vel0[s] = make_double2(u, v);
        D.rho0[s] = rho;
        D.pos[s] = make_double2(x, y);
        if (to_staging) {
            const int i = D.id[s];
            if (i < P.n_host) {
                S.pos[i] = make_double2(x, y);
                S.vel[i] = make_double2(u, v);
                S.rho[i] = rho;
                // the carried rates as k_unsort reads them back (rounded to R)
                S.r_drho[i] = (double)(R)dr;
                S.r_acc[i] = make_double2((double)(R)ax, (double)(R)ay);
                S.r_avg[i] = make_double2((double)(R)gx, (double)(R)gy);
            }
        }
    } else {
        D.pos[s] = make_double2(x, y);
    }
    double p, c;
    eos64(P, rho, p, c);
    const double m = D.mass[s];
    D.kin[s] = make_double4(u, v, rho, p);
    D.aux[s] = mk4<R>((R)m, (R)(m / rho), (R)c, (R)D.smass[s]);
    store_split(D, s, make_double2(x, y), make_double4(u, v, rho, p));
}

// Density re-initialisation by moving least squares (Reinitialize_particle_density:
// Taylor_Green_Vortex/Reinitialize_particle_density.f90:98-181 with
// MLS_Interpolation_In_Subdomain_Domain.f90:96-285; moving-square variant
// Moving_Square.../Reinitialize_particle_density.f90:92-200 with
// SPH_Subroutine_Module.f90:2565-2792), FP64, on the state after the integrator
// update (images keep the step-start state).  For a water particle i and its
// neighbours j within the support, with W_j the kernel value (the moving-square
// variant: W_j V_j, and i itself counts as a neighbour),
//   p_j = (1, dx, dy[, dx^2, dx dy, dy^2]),  (dx, dy) = (x_j - x_i)/h,
//   A   = sum_j W_j p_j p_j^T + alpha^3 I,
//   rho_i = sum_j rho_j W_j (A^-1 e_1).p_j = c.r,  A c = e_1,  r = sum_j rho_j W_j p_j.
// The reference inverts A (BRINV / the 3x3 adjugate) and forms the same weights;
// here A c = e_1 is solved by an FP64 Cholesky factorisation (A is symmetric and
// positive definite away from degenerate neighbourhoods).  A failed factorisation,
// and with order 6 at most 8 neighbours (Taylor-Green variant), fall back to the
// Shepard weights W_j / sum W, as the reference does.  Non-water particles keep
// their density (the Taylor-Green routine zeroes its periodic images, which are
// regenerated at the next step start).
template <int M>
__device__ __forceinline__ bool chol_solve_e1(double (&A)[M * (M + 1) / 2], double (&c)[M]) {
    // packed lower triangle, row-major: A[i(i+1)/2 + j], j <= i
    double L[M * (M + 1) / 2];
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
    // L y = e_1, L^T c = y
    double y[M];
#pragma unroll
    for (int i = 0; i < M; ++i) {
        double sum = i == 0 ? 1.0 : 0.0;
#pragma unroll
        for (int k = 0; k < i; ++k) sum -= L[i * (i + 1) / 2 + k] * y[k];
        y[i] = sum / L[i * (i + 1) / 2 + i];
    }
#pragma unroll
    for (int i = M - 1; i >= 0; --i) {
        double sum = y[i];
#pragma unroll
        for (int k = i + 1; k < M; ++k) sum -= L[k * (k + 1) / 2 + i] * c[k];
        c[i] = sum / L[i * (i + 1) / 2 + i];
    }
    return true;
}

template <typename R, int M>
__global__ void k_mls(Params P, Sorted<R> D, double* rho_new) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= P.n_tot) return;
    const double rho_a = D.kin[a].z;
    if (D.type[a] != SPH_TYPE_WATER || D.id[a] >= P.n_host) { rho_new[a] = rho_a; return; }
    const double2 xa = D.pos[a];
    const double inv_h = 1.0 / P.h;
    double A[M * (M + 1) / 2], r[M];
#pragma unroll
    for (int k = 0; k < M * (M + 1) / 2; ++k) A[k] = 0.0;
#pragma unroll
    for (int k = 0; k < M; ++k) r[k] = 0.0;
    double sw = 0.0, srw = 0.0;
    int cnt = 0;
    const int nn = D.nnbr[a];
    // the moving-square variant includes the particle itself (distance 0)
    for (int e = (P.ms ? -1 : 0); e < nn; ++e) {
        const int b = e < 0 ? a : (int)(D.nbr[(size_t)e * P.nbr_stride + a] & 0x7fffffffu);
        const double2 xb = D.pos[b];
        const double px = xa.x - xb.x, py = xa.y - xb.y;
        double d;
        const bool in = in_support(P, px, py, d);
        if (P.ms ? !(d <= P.r_cut) : !in) continue;
        double w, gx, gy;
        kernel_w_dw<double>(P, d, px, py, w, gx, gy);
        const double rho_b = D.kin[b].z;
        if (P.ms) w *= D.mass[b] / rho_b;
        double p[M];
        const double dx = -px * inv_h, dy = -py * inv_h;
        p[0] = 1.0; p[1] = dx; p[2] = dy;
        if (M == 6) { p[3 % M] = dx * dx; p[4 % M] = dx * dy; p[5 % M] = dy * dy; }
#pragma unroll
        for (int i = 0; i < M; ++i) {
            const double wp = w * p[i];
#pragma unroll
            for (int j = 0; j <= i; ++j) A[i * (i + 1) / 2 + j] += wp * p[j];
            r[i] += rho_b * wp;
        }
        sw += w;
        srw += rho_b * w;
        ++cnt;
    }
#pragma unroll
    for (int i = 0; i < M; ++i) A[i * (i + 1) / 2 + i] += P.mls_alpha3;
    double c[M];
    double out;
    const bool few = !P.ms && M == 6 && cnt <= 8;
    if (!few && chol_solve_e1<M>(A, c)) {
        out = 0.0;
#pragma unroll
        for (int i = 0; i < M; ++i) out += c[i] * r[i];
    } else {
        out = srw / sw;
    }
    if (P.ms && isnan(out)) out = rho_a;
    rho_new[a] = out;
}

// RefreshDensity_MLS_Order = 1 (Taylor_Green_Vortex/Reinitialize_particle_density.f90:71-92,
// Moving_Square.../Reinitialize_particle_density.f90:66-88), evaluated on the
// step's last RHS (its pair list and state, which the reference's pair arrays
// and volumes still hold when it runs): for a water particle a,
//   rho_a = sum_b m_b W_ab / sum_b W_ab V_b
// over the pairs with a neighbour of a's type (sum_w,
// Define_freesurface_and_Normailized_derivates.f90:87-91), in FP64.
template <typename R>
__global__ void k_mls1(Params P, Sorted<R> D, double* rho_new) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= P.n_tot) return;
    rho_new[a] = D.kin[a].z;
    const int ta = D.type[a];
    if (ta != SPH_TYPE_WATER || D.id[a] >= P.n_host) return;
    const double2 xa = D.pos[a];
    double sw = 0.0, sm = 0.0;
    const int nn = D.npairs[a];
    for (int e = 0; e < nn; ++e) {
        const int b = (int)(D.pairs[(size_t)e * P.nbr_stride + a] & 0x7fffffffu);
        if (D.type[b] != ta) continue;
        const double2 xb = D.pos[b];
        const double px = xa.x - xb.x, py = xa.y - xb.y;
        const double d = __dsqrt_rn(__dadd_rn(__dmul_rn(px, px), __dmul_rn(py, py)));
        double w, gx, gy;
        kernel_w_dw<double>(P, d, px, py, w, gx, gy);
        const double mb = D.mass[b];
        sw += w * (mb / D.kin[b].z);
        sm += mb * w;
    }
    rho_new[a] = sm / sw;
}

// The re-initialised density replaces the integrated one; then the shift of the
// step (when on) is applied, as the reference's driver calls the two in turn.
template <typename R>
__global__ void k_finish_mls(Params P, Sorted<R> D, const double* rho_new, int do_shift, unsigned* status) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.n_tot) return;
    if (!integrated(P, D.type[s]) || D.id[s] >= P.n_host) return;
    const double2 x0 = D.pos0[s];
    double x = x0.x, y = x0.y;
    double rho = D.type[s] == SPH_TYPE_WATER ? rho_new[s] : D.rho0[s];
    if (do_shift) apply_shift(P, D, s, x, y, rho);
    if (!(isfinite(x) && isfinite(y) && isfinite(rho))) atomicOr(status, ST_NONFINITE);
    D.pos0[s] = make_double2(x, y);
    D.pos[s] = make_double2(x, y);
    D.rho0[s] = rho;
    double p, c;
    eos64(P, rho, p, c);
    const double2 v = D.vel0[s];
    const double m = D.mass[s];
    D.kin[s] = make_double4(v.x, v.y, rho, p);
    D.aux[s] = mk4<R>((R)m, (R)(m / rho), (R)c, (R)D.smass[s]);
    store_split(D, s, make_double2(x, y), make_double4(v.x, v.y, rho, p));
}

// Body_Motion_Solver (Moving_Square.../Body_Motion_Solver.f90:187-193): the body
// particles (initial type SPH_TYPE_BODY) move by the step's displacement.
__global__ void k_translate_body(int n, const int* itype, double2* pos, double dx, double dy) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || itype[i] != SPH_TYPE_BODY) return;
    const double2 x = pos[i];
    pos[i] = make_double2(x.x + dx, x.y + dy);
}

// (dw/dd) / d of the ghost kernel at q = d / h_g.
__device__ __forceinline__ double ghost_dw_over_d(const Params& P, double q) {
    const double hg2 = P.ghost_h * P.ghost_h;
    if (P.kernel_model == SPH_KERNEL_GAUSSIAN) return -2.0 * exp(-(q * q)) * P.ghost_kf / hg2;
    const double tq = 1.0 - q / 2.0;
    return -5.0 * (tq * tq * tq) * P.ghost_kf / hg2;
}

// The neighbours the ghost assignment interpolates from for ghost slot s: the
// non-ghost particles within kernel_scale * 1.2 h, found over the window of s's
// cell (the list-build cells, so the window reaches ghost_r plus half the skin).
// The 32 lanes of a warp split the candidates of each window row (the slots of
// a row's window cells are contiguous in the cell-sorted order); fn(b, dx, dy,
// q, w) gets (dx, dy) = x_s - x_b, q = d / h_g and the kernel value w with the
// ghost smoothing length h_g, on the lane that visits b.
template <typename R, typename F>
__device__ __forceinline__ void ghost_visit_warp(const Params& P, const Sorted<R>& D, int s, F&& fn) {
    const int lane = threadIdx.x & 31;
    const double2 x = D.pos[s];
    const int cx = (int)floor((x.x - P.gx0) / P.cs), cy = (int)floor((x.y - P.gy0) / P.cs);
    const double hg = P.ghost_h;
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
        for (int b = lo + lane; b < hi; b += 32) {
            if (D.type[b] == SPH_TYPE_FIX_GHOST) continue;
            const double2 xb = D.pos[b];
            const double dx = x.x - xb.x, dy = x.y - xb.y;
            const double d = sqrt(dx * dx + dy * dy);
            if (!(d <= P.ghost_r)) continue;
            const double q = d / hg;
            double w;
            if (P.kernel_model == SPH_KERNEL_GAUSSIAN) {
                w = (exp(-(q * q)) - P.gauss_e9) * P.ghost_kf;
            } else {
                const double tq = 1.0 - q / 2.0;
                const double t2 = tq * tq;
                w = P.ghost_kf * (1.0 + 2.0 * q) * (t2 * t2);
            }
            fn(b, dx, dy, q, w);
        }
    }
}

// Sum over the warp, lane 0's association order, broadcast to every lane (so
// that all lanes continue with bit-identical values).
__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return __shfl_sync(0xffffffffu, v, 0);
}
__device__ __forceinline__ int warp_sum(int v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return __shfl_sync(0xffffffffu, v, 0);
}

// Fixed-ghost assignment of the moving-square driver (Moving_Square.../
// Assign_boundary_particles.f90:611-941, with MLS_order_Boundary = 1, i.e.
// Shepard weights Fai_j = W_j V_j / sum W V), at the start of every RHS, from the
// current state of the non-ghost particles within kernel_scale * 1.2 h:
//   p = sum Fai (p_j + rho_j g.(x - x_j)),  u = sum Fai u_j,  m = sum Fai m_j
// (g: gravity, plus the body acceleration for body ghosts), at least 3
// neighbours or nothing.  Body ghosts take the body velocity; wall ghosts, during
// 0 < t <= Shock_wave_release_time, go through the characteristic variables for
// labels -6 / -7 (which return the interpolated values) and keep the zero
// pressure they start from for other labels, as the reference's branch does;
// then the wall velocity is mirrored by label and wall condition.  Finally
// rho = (p - pb)/c0^2 + rho0, or the rest state when m = 0.
// One warp per ghost (ghost_ids: the host ghosts in id order, n_ghost of them),
// the lanes splitting the neighbours; the sums are reduced in a fixed order.
template <typename R>
// gint / gsw (may be null): the interpolated (p, u, v, m) and the weight sum
// sum W V of each ghost slot, kept for the reverse (k_adj_ghost_lambda).
__global__ void k_assign_ghosts(Params P, Sorted<R> D, const int* ghost_ids, int n_ghost, double t, double bvx,
                                double bvy, double bax, double bay, double4* gint = nullptr,
                                double* gsw = nullptr) {
    const int wg = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (wg >= n_ghost) return;                       // whole warps
    const int s = D.slot_of[ghost_ids[wg]];
    const double2 x = D.pos[s];
    const bool body = D.itype[s] == SPH_TYPE_BODY;
    const double gxe = P.grav[0] + (body ? bax : 0.0), gye = P.grav[1] + (body ? bay : 0.0);
    double sw = 0.0, sp = 0.0, su = 0.0, sv = 0.0, sm = 0.0;
    int cnt = 0;
    ghost_visit_warp(P, D, s, [&](int b, double dx, double dy, double, double w) {
        const double4 kb = D.kin[b];
        const double mb = D.mass[b];
        const double W = w * (mb / kb.z);
        sw += W;
        sp += kb.w * W + kb.z * W * (gxe * dx + gye * dy);
        su += kb.x * W;
        sv += kb.y * W;
        sm += mb * W;
        ++cnt;
    });
    sw = warp_sum(sw); sp = warp_sum(sp); su = warp_sum(su); sv = warp_sum(sv); sm = warp_sum(sm);
    cnt = warp_sum(cnt);
    if ((threadIdx.x & 31) != 0) return;
    double uint = 0.0, vint = 0.0, pint = 0.0, m = 0.0;
    if (cnt >= 3) {
        const double inv = 1.0 / sw;
        pint = sp * inv; uint = su * inv; vint = sv * inv; m = sm * inv;
    }
    if (gint) {
        gint[s] = make_double4(pint, uint, vint, m);
        gsw[s] = sw;
    }
    double u, v, p = 0.0;
    if (body) {
        u = bvx; v = bvy; p = pint;
    } else {
        const int lab = D.blabel[s];
        if (0.0 < t && t <= P.shock_t) {
            const double ri = (pint - P.pb) / P.c0sq + P.rho0;
            const double r = ri / P.rho0;
            const double c = P.sqrt_c0 * (r * r * r);
            u = uint; v = vint;
            if (lab == -6 || lab == -7) {
                const double vn = lab == -6 ? vint : uint;
                const double J2 = ri * c * vn + pint, J3 = -ri * c * vn + pint;
                const double vs = (J2 - J3) / (2 * ri * c);
                if (lab == -6) v = vs; else u = vs;
                p = 0.5 * (J2 + J3);
            }
        } else {
            u = uint; v = vint; p = pint;
        }
        if (lab == -6) { if (P.wall_bc == 1) v = -v; else { u = -u; v = -v; } }
        else if (lab == -7) { u = -u; v = -v; }
        else if (lab == -8) { if (P.wall_bc == 1) u = -u; else { u = -u; v = -v; } }
    }
    double rho, c;
    if (m != 0.0) {
        rho = (p - P.pb) / P.c0sq + P.rho0;
        const double r = rho / P.rho0;
        c = P.sqrt_c0 * (r * r * r);
    } else {
        u = 0.0; v = 0.0; p = 0.0; rho = P.rho0; m = 0.0; c = P.sqrt_c0;
    }
    D.mass[s] = m;
    D.smass[s] = m;
    D.vel0[s] = make_double2(u, v);
    D.rho0[s] = rho;
    D.kin[s] = make_double4(u, v, rho, p);
    D.aux[s] = mk4<R>((R)m, (R)(m / rho), (R)c, (R)m);
    store_split(D, s, x, make_double4(u, v, rho, p));
}

// The per-particle arrays k_assign_ghosts writes besides the records (mass,
// SPS mass, step-start velocity and density), set again from the records of a
// state that already holds the assigned ghosts (FP64 records: aux.x = m exactly).
template <typename R>
__global__ void k_ghost_refill(Sorted<R> D, const int* ghost_ids, int n_ghost) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_ghost) return;
    const int s = D.slot_of[ghost_ids[g]];
    const double4 k = D.kin[s];
    const double m = (double)D.aux[s].x;
    D.mass[s] = m;
    D.smass[s] = m;
    D.vel0[s] = make_double2(k.x, k.y);
    D.rho0[s] = k.z;
}

// Kinetic energy and max |v| of the water host particles
// (Sampling_subroutine.f90:346-356): deterministic two-level reduction in FP64.
constexpr int kRedThreads = 256;
template <typename R>
__global__ void k_diag_partial(Params P, Sorted<R> D, double* part_ke, double* part_max) {
    __shared__ double ske[kRedThreads], smx[kRedThreads];
    double ke = 0.0, mx = 0.0;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < P.n_tot; s += gridDim.x * blockDim.x) {
        if (D.type[s] != SPH_TYPE_WATER || D.id[s] >= P.n_host) continue;
        double2 v = D.vel0[s];
        double vv = v.x * v.x + v.y * v.y;
        ke += 0.5 * D.mass[s] * vv;
        mx = fmax(mx, sqrt(vv));
    }
    ske[threadIdx.x] = ke; smx[threadIdx.x] = mx;
    __syncthreads();
    for (int w = kRedThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) { ske[threadIdx.x] += ske[threadIdx.x + w]; smx[threadIdx.x] = fmax(smx[threadIdx.x], smx[threadIdx.x + w]); }
        __syncthreads();
    }
    if (threadIdx.x == 0) { part_ke[blockIdx.x] = ske[0]; part_max[blockIdx.x] = smx[0]; }
}

__global__ void k_diag_final(int nparts, const double* part_ke, const double* part_max, double* out) {
    __shared__ double ske[kRedThreads], smx[kRedThreads];
    double ke = 0.0, mx = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) { ke += part_ke[i]; mx = fmax(mx, part_max[i]); }
    ske[threadIdx.x] = ke; smx[threadIdx.x] = mx;
    __syncthreads();
    for (int w = kRedThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) { ske[threadIdx.x] += ske[threadIdx.x + w]; smx[threadIdx.x] = fmax(smx[threadIdx.x], smx[threadIdx.x + w]); }
        __syncthreads();
    }
    if (threadIdx.x == 0) { out[0] = ske[0]; out[1] = smx[0]; }
}

// Body force of the last RHS (Moving_Square.../Calculate_Body_Force.f90:53-142 and
// Single_step_compute.f90:228-243), FP64: for a particle a with body neighbours b
// (initial type SPH_TYPE_BODY)
//   BFP_a = -sum_b V_b (p_a + p_b) B_a^-1 grad_a W_ab
//   BFV_a =  sum_b rho_a V_b 2 nu ((x_a - x_b).B_a^-1 grad_a W_ab) / r^2 (v_a - v_b)   (Morris)
//       or   sum_b rho_a V_b 2 (dim+2) nu ((v_a-v_b).(x_a-x_b)) / r^2 B_a^-1 grad_a W_ab
// and the forces are sum_a V_a BFP_a, sum_a V_a BFV_a and their sum (no gravity).
// Gathered from the body side: body particle b sums V_a times its terms over its
// pair neighbours a (the pair set is symmetric), so only the body's threads loop.
template <typename R>
__global__ void k_body_force(Params P, Sorted<R> D, double* part) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    double f[6] = {0, 0, 0, 0, 0, 0};
    if (b < P.n_tot && D.itype[b] == SPH_TYPE_BODY) {
        const int nn = D.npairs[b];
        const double2 xb = D.pos[b];
        const double4 kb = D.kin[b];
        const double Vb = D.mass[b] / kb.z;
        for (int e = 0; e < nn; ++e) {
            const int a = (int)(D.pairs[(size_t)e * P.nbr_stride + b] & 0x7fffffffu);
            const double2 xa = D.pos[a];
            const double4 ka = D.kin[a];
            const double4 bi = D.binv64[a];
            const double Va = D.mass[a] / ka.z;
            const double dx = xa.x - xb.x, dy = xa.y - xb.y;
            const double r2 = dx * dx + dy * dy, d = sqrt(r2);
            double w, gx, gy;
            kernel_w_dw<double>(P, d, dx, dy, w, gx, gy);
            const double n0 = bi.x * gx + bi.y * gy, n1 = bi.z * gx + bi.w * gy;
            const double bp0 = -Vb * (ka.w + kb.w) * n0, bp1 = -Vb * (ka.w + kb.w) * n1;
            const double du = ka.x - kb.x, dv = ka.y - kb.y;
            double bv0, bv1;
            if (P.laplacian == 1) {
                const double fv = ka.z * Vb * 2 * P.nu * (dx * n0 + dy * n1) / r2;
                bv0 = fv * du; bv1 = fv * dv;
            } else {
                const double fv = ka.z * Vb * 2 * (2 + 2) * P.nu * (du * dx + dv * dy) / r2;
                bv0 = fv * n0; bv1 = fv * n1;
            }
            f[0] += Va * bp0; f[1] += Va * bp1; f[2] += Va * bv0; f[3] += Va * bv1;
            f[4] += Va * (bp0 + bv0); f[5] += Va * (bp1 + bv1);
        }
    }
    __shared__ double sh[6][kRedThreads];
    for (int c = 0; c < 6; ++c) sh[c][threadIdx.x] = f[c];
    __syncthreads();
    for (int w = kRedThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int c = 0; c < 6; ++c) sh[c][threadIdx.x] += sh[c][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 6; ++c) part[(size_t)c * gridDim.x + blockIdx.x] = sh[c][0];
}

__global__ void k_body_force_final(int nparts, const double* part, double* out) {
    __shared__ double sh[kRedThreads];
    for (int c = 0; c < 6; ++c) {
        double s = 0.0;
        for (int i = threadIdx.x; i < nparts; i += blockDim.x) s += part[(size_t)c * nparts + i];
        sh[threadIdx.x] = s;
        __syncthreads();
        for (int w = kRedThreads / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[c] = sh[0];
        __syncthreads();
    }
}

// Count of flagged surface particles (diagnostics).
template <typename R>
__global__ void k_count_surface(Params P, Sorted<R> D, int* out) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.n_tot) return;
    if (D.flags[s] & 1) atomicAdd(out, 1);
}

// --- find_particle_pair entry point ---------------------------------------
// Pairs are emitted once, by their pair_i (lower id), sorted by (i, j).
template <typename R>
__global__ void k_pair_count(Params P, Sorted<R> D, int* cnt_id) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= P.n_tot) return;
    const int nn = D.nnbr[a];
    const double2 xa = D.pos[a];
    int c = 0;
    for (int e = 0; e < nn; ++e) {
        const unsigned ent = D.nbr[(size_t)e * P.nbr_stride + a];
        if (!(ent >> 31)) continue;
        const double2 xb = D.pos[ent & 0x7fffffffu];
        double d;
        if (in_support(P, xa.x - xb.x, xa.y - xb.y, d)) ++c;
    }
    cnt_id[D.id[a]] = c;
}

template <typename R>
__global__ void k_pair_emit(Params P, Sorted<R> D, const long long* off_id, long long cap, int* pi, int* pj,
                            double* w, double* dwdx) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= P.n_tot) return;
    const int nn = D.nnbr[a];
    const double2 xa = D.pos[a];
    const int ida = D.id[a];
    int bid[256];
    int m = 0;
    for (int e = 0; e < nn && m < 256; ++e) {
        const unsigned ent = D.nbr[(size_t)e * P.nbr_stride + a];
        if (!(ent >> 31)) continue;
        const int b = (int)(ent & 0x7fffffffu);
        const double2 xb = D.pos[b];
        double d;
        if (!in_support(P, xa.x - xb.x, xa.y - xb.y, d)) continue;
        // insertion by neighbour id
        const int idb = D.id[b];
        int k = m++;
        while (k > 0 && D.id[bid[k - 1]] > idb) { bid[k] = bid[k - 1]; --k; }
        bid[k] = b;
    }
    long long o = off_id[ida];
    for (int k = 0; k < m; ++k, ++o) {
        if (o >= cap) return;
        const int b = bid[k];
        const double2 xb = D.pos[b];
        double dx = xa.x - xb.x, dy = xa.y - xb.y, d;
        in_support(P, dx, dy, d);
        double ww, gx, gy;
        kernel_w_dw<double>(P, d, dx, dy, ww, gx, gy);
        pi[o] = ida + 1;
        pj[o] = D.id[b] + 1;
        if (w) w[o] = ww;
        if (dwdx) { dwdx[o] = gx; dwdx[cap + o] = gy; }
    }
}

// --- column-major (n,2) <-> interleaved conversions -----------------------
__global__ void k_interleave(int n, const double* colmaj, double2* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = make_double2(colmaj[i], colmaj[n + i]);
}
__global__ void k_deinterleave(int n, const double2* in, double* colmaj) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { double2 v = in[i]; colmaj[i] = v.x; colmaj[n + i] = v.y; }
}

// Snapshot of the host particles' state (id order, staging arrays) in the
// column-major layout of sph_get_state: [0, 2n) pos, [2n, 4n) vel, [4n, 5n) rho,
// [5n, 6n) pressure from the equation of state.
__global__ void k_snapshot(Params P, int n, const double2* pos, const double2* vel, const double* rho,
                           double* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double2 x = pos[i], v = vel[i];
    const double r = rho[i];
    double p, c;
    eos64(P, r, p, c);
    out[i] = x.x; out[n + i] = x.y;
    out[2 * (size_t)n + i] = v.x; out[3 * (size_t)n + i] = v.y;
    out[4 * (size_t)n + i] = r;
    out[5 * (size_t)n + i] = p;
}

// Per-particle outputs of the last RHS in id order (host particles), as doubles.
// Layout: [0] drho, [1,2] acc, [3,4] avg, [5] fs, [6] near, [7] fra_v,
// [8..11] binv, [12..14] tau, [15..22] grads  (each block n long).
constexpr int kExportFields = 23;
template <typename R>
__global__ void k_export(Params P, Sorted<R> D, double* out) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.n_tot) return;
    int i = D.id[s];
    if (i >= P.n_host) return;
    const size_t n = (size_t)P.n_host;
    out[0 * n + i] = (double)D.drho[s];
    out[1 * n + i] = (double)D.acc[s].x; out[2 * n + i] = (double)D.acc[s].y;
    out[3 * n + i] = (double)D.avg[s].x; out[4 * n + i] = (double)D.avg[s].y;
    out[5 * n + i] = (D.flags[s] & 1) ? 1.0 : 0.0;
    out[6 * n + i] = (D.flags[s] & 2) ? 1.0 : 0.0;
    out[7 * n + i] = (double)D.fra_v[s];
    auto bi = D.binv[s]; auto n1 = D.nb1[s]; auto n2 = D.nb2[s]; auto n3 = D.nb3[s];
    const double gs = grad_scale<R>();
    out[8 * n + i] = (double)bi.x; out[9 * n + i] = (double)bi.y; out[10 * n + i] = (double)bi.z; out[11 * n + i] = (double)bi.w;
    out[12 * n + i] = (double)n1.x; out[13 * n + i] = (double)n1.y; out[14 * n + i] = (double)n1.z;
    out[15 * n + i] = gs * n1.w; out[16 * n + i] = gs * n2.x;
    out[17 * n + i] = gs * n2.y; out[18 * n + i] = gs * n2.z;
    out[19 * n + i] = gs * n2.w; out[20 * n + i] = gs * n3.x;
    out[21 * n + i] = gs * n3.y; out[22 * n + i] = gs * n3.z;
}

}  // namespace sph
