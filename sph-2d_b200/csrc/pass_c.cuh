// pass_c.cuh -- neighbour pass C: the fused force pass.  One thread per
// particle gathers, for every pair neighbour, the linear-Riemann flux (with
// optional MUSCL reconstruction), continuity, pressure force, Monaghan
// artificial viscosity, Morris laplacian, delta-alpha term, SPS force, XSPH,
// delta-SPH density diffusion and (on the last RHS of a step, FP64 and
// moving-square launches) the shifting sum; the mixed Taylor-Green path forms
// the shifting sum in k_shift_gather after this pass.
//
// Reference loops (all in pair order, scattered to pair_i and pair_j):
//   Solver_Normalized_Modified_Linear_Riemann_Delta_SPS.f90:300-502, 552-583, 627-635
//   Solver_Normalized_MUSCL_Linear_Riemann_Delta_SPS.f90:458-682, 690-721
//   Solver_Normalized_Delta_SPH_SPS.f90:324-512, 610-636 (the plain method)
//   MUSCL_Limiter: function_module.f90:34-80
//   Shift_particle_position.f90:78-103
//   assembly: single_step_compute.f90:152-171
//
// Every pair quantity is evaluated in the reference's own orientation
// (pair_i = the particle with the lower id, bit 31 of the list entry), so the
// flux seen by the two particles of a pair is computed by the same sequence
// of operations; each thread then keeps the pair_i or pair_j contribution that
// belongs to its particle.  The physical terms are summed per pair and then
// accumulated (the reference sums each term over all pairs first); the two
// orders agree to round-off.
//
// Precision: R = double is the FP64 path.  R = float is the mixed path: FP32
// pair arithmetic with reciprocal/rsqrt instead of divisions, FP64 sums of
// the FP32 terms for the acceleration and the density rate, and the shifting
// sum in FP64 (its terms are O(h/10) each and cancel to a displacement that
// is orders of magnitude smaller, so FP32 rounding there would inject position
// noise every step into the unstable lattice modes the shifting excites).
#pragma once
#include "pass_a.cuh"

namespace sph {

template <typename R>
__device__ __forceinline__ void muscl_limiter(R di, R dj, R dij, R& li, R& lj) {
    // The reference's two sign branches folded into one: with s = sign(dj)
    // (+1 when dj > 0, else -1) the dj <= 0 branch is the dj > 0 branch applied
    // to (-di, -dj) and negated, since min and max swap under negation:
    //   lim = s max(0, max(min(1.3 s di, s dj), min(s di, 1.3 s dj))),
    //   lim < dij/2 (dj <= 0) <=> s lim > s dij/2,  di < dj <=> s di > s dj.
    // The same values as the branches (zero increments may carry the other
    // sign), one min/max chain, no divergence between the lanes of a warp.
    const R b = R(1.3);
    const R s = dj > R(0) ? R(1) : R(-1);
    const R sdi = s * di, sdj = s * dj;
    const R m = max(R(0), max(min(b * sdi, sdj), min(sdi, b * sdj)));     // s * lim >= 0
    const R half = R(0.5) * dij;
    const bool big = m > s * half && m > R(0);
    const bool first = sdi > sdj;
    const R lim = s * m;
    const R off = dij * R(0);
    li = big ? (first ? half : off) : lim;
    lj = big ? (first ? off : half) : lim;
}

// The FP32 form: multiplying by s = +-1 is a flip of the sign bit (taken from
// dj), and s dj = |dj|.  dj = +0 takes s = +1 instead of -1; both give m = 0,
// big = false and li = lj = 0, so the values are those of the form above
// (a zero increment may carry the other sign).
template <>
__device__ __forceinline__ void muscl_limiter<float>(float di, float dj, float dij, float& li, float& lj) {
    const float b = 1.3f;
    const unsigned sb = __float_as_uint(dj) & 0x80000000u;
    const float sdi = __uint_as_float(__float_as_uint(di) ^ sb), sdj = fabsf(dj);
    const float m = fmaxf(0.f, fmaxf(fminf(b * sdi, sdj), fminf(sdi, b * sdj)));
    const float half = 0.5f * dij;
    const bool big = m > __uint_as_float(__float_as_uint(half) ^ sb) && m > 0.f;
    const bool first = sdi > sdj;
    const float lim = __uint_as_float(__float_as_uint(m) ^ sb);
    li = big ? (first ? half : 0.f) : lim;
    lj = big ? (first ? 0.f : half) : lim;
}

// The same FP32 limiter with its results as a pair term uses them: the sum
// L = li + lj (half when one increment is clamped to dij/2, else 2 lim) and the
// increment of this particle's side (li when it is pair_i, else lj).
__device__ __forceinline__ void muscl_limiter_sum(float di, float dj, float dij, bool a_is_i, float& L, float& own) {
    const float b = 1.3f;
    const unsigned sb = __float_as_uint(dj) & 0x80000000u;
    const float sdi = __uint_as_float(__float_as_uint(di) ^ sb), sdj = fabsf(dj);
    const float m = fmaxf(0.f, fmaxf(fminf(b * sdi, sdj), fminf(sdi, b * sdj)));
    const float half = 0.5f * dij;
    const bool big = m > __uint_as_float(__float_as_uint(half) ^ sb) && m > 0.f;
    const bool first = sdi > sdj;
    const float lim = __uint_as_float(__float_as_uint(m) ^ sb);
    L = big ? half : 2.f * lim;
    own = big ? (first == a_is_i ? half : 0.f) : lim;
}

// Reciprocal and quotient in the pair loop: correctly rounded, except the
// FP32 1/rho-bar and artificial-viscosity quotient (fast_quot: __fdividef,
// about 2 ulp).  Fast forms everywhere made mixed pass C slower (3.46 -> 3.85 ms
// per step at 2048^2: fewer instructions between the neighbour-record loads);
// these two alone took it from 2.80 to 2.75 ms with the velocity L2 against
// FP64 unchanged (2.78e-6 after 100 steps).
__device__ __forceinline__ double rcp(double x) { return 1.0 / x; }
__device__ __forceinline__ float rcp(float x) { return __frcp_rn(x); }
template <typename R>
__device__ __forceinline__ R quot(R a, R b) { return a / b; }
__device__ __forceinline__ double fast_quot(double a, double b) { return a / b; }
__device__ __forceinline__ float fast_quot(float a, float b) { return __fdividef(a, b); }

// Per-particle state a thread needs for one side of a pair.
template <typename R>
struct Side {
    using V4 = typename VT<R>::V4;
    double4 kin;   // u, v, rho, p (FP64)
    float4 kh, kl; // the same, hi + lo (mixed Taylor-Green variants)
    V4 aux;        // m, V, c, smass
    V4 nb1, nb2, nb3;
};

// The pair terms are written with the pair differences du = u_i - u_j,
// dv = v_i - v_j, dp = p_i - p_j, drho = rho_j - rho_i formed in FP64 from the
// kinematic records; in real arithmetic this is the reference's expression,
// e.g. v_i - v* = (v_i - v_j)/2 - (U* - Ubar) e for the modified solver.
// MS: the moving-square solvers (HLLC or modified linear with XSPH in the
// continuity flux, laplacian switch, no SPS); SHIFT: the last RHS of a step with
// shifting on, which also forms the shifting sum.  Both are compile-time so that
// each launch carries only the registers of the terms it evaluates.
#ifndef SPH_PASS_C_SHIFT_BLOCKS
#define SPH_PASS_C_SHIFT_BLOCKS 4
#endif
#ifndef SPH_PASS_C_F32_BLOCKS
#define SPH_PASS_C_F32_BLOCKS 4
#endif
template <typename R, bool MUSCL, bool MS, bool SHIFT>
__global__ void __launch_bounds__(128, sizeof(R) == 4 ? (SHIFT ? SPH_PASS_C_SHIFT_BLOCKS : SPH_PASS_C_F32_BLOCKS) : 3)
    k_pass_c(Params P, Sorted<R> D) {
    using V4 = typename VT<R>::V4;
    using A = typename Acc<R>::T;
    constexpr bool F32 = sizeof(R) == 4;
    // hi/lo records: every mixed variant (the moving-square HLLC state is then
    // formed in FP32 from differences, below)
    constexpr bool HL = F32;
    // the shifting sum needs the FP64 position differences: that launch reads the
    // neighbour's FP64 position (and FP64 volume) instead of its hi/lo position
    // and takes the FP32 difference as the rounding of the FP64 one
    constexpr bool X64 = !HL || SHIFT;
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= P.n_tot) return;
    const int ta = D.type[a];
    const int nn = D.npairs[a];
    const double2 xa = X64 ? D.pos[a] : make_double2(0.0, 0.0);
    float4 xa_hl = make_float4(0.f, 0.f, 0.f, 0.f);
    Side<R> S;
    if (HL) { S.kh = D.kh[a]; S.kl = D.kl[a]; }
    if (!X64) xa_hl = D.xhl[a];
    else S.kin = D.kin[a];
    S.aux = D.aux[a]; S.nb1 = D.nb1[a]; S.nb2 = D.nb2[a];
    if (MUSCL) S.nb3 = D.nb3[a];
    const R rho_a = HL ? (R)S.kh.z : (R)S.kin.z;
    const V4 bi = D.binv[a];
    // Solver_Normalized_Delta_SPH_SPS has no Riemann state: its continuity and
    // pressure terms (:333-374) are the pair-mean (v-bar, P-bar) form the Riemann
    // solvers use near the free surface, so it takes that branch for every pair
    const bool dsph = !MUSCL && !MS && P.dsph;
    const bool near_a = dsph || (D.flags[a] & 2) != 0;
    // delta-SPH and the assembly only apply to integrated particles (Solver :627-635,
    // Moving_Square.../Single_step_compute.f90:273-281)
    const bool water = integrated(P, ta);
    typename VT<R>::V2 avg_a = mk2<R>(R(0), R(0));
    if (MS) avg_a = D.avg[a];

    const R hbar = (R)P.h;
    const R inv_h = (R)(1.0 / P.h);
    const R gk = (R)((P.kernel_model == SPH_KERNEL_GAUSSIAN ? -2.0 : -5.0) * P.kfactor / (P.h * P.h));
    const R inv_sqc0 = (R)(1.0 / P.sqrt_c0);
    const R nu2 = (R)(2.0 * P.nu), alpha = (R)P.alpha, beta = (R)P.beta;
    const R fh2 = (R)((P.fai * P.h) * (P.fai * P.h));
    const R dlt2h = (R)(2.0 * P.delta * P.h);
    const R dla_dh = (R)(P.delta * P.h);
    const R dla_h = (R)(P.delta_alpha * P.h);
    const R eps2 = (R)(2.0 * P.eps);
    // 1/rho: the FP32 MUSCL records carry it (nb3.w, the same rounded reciprocal)
    constexpr bool RREC = F32 && MUSCL;
    const R inv_rho_a = RREC ? (R)S.nb3.w : rcp(rho_a);
    const R rho0_over_rho_a = (R)P.rho0 * inv_rho_a;
    const R dla_rho = dla_h * rho0_over_rho_a;

    A cont, accx, accy;
    cont.init(); accx.init(); accy.init();
    R xsx = R(0), xsy = R(0);
    double shx = 0.0, shy = 0.0;   // shifting sum, FP64 in both paths
    const double inv_h64 = 1.0 / P.h, inv_h2_64 = inv_h64 * inv_h64, inv_wdx = 1.0 / P.w_dx;

    // the pairs pass A found inside the support at this RHS
    unsigned ent_n = nn > 0 ? __ldg(&D.pairs[a]) : 0u;
    // software pipeline: the pair entry two iterations ahead; the neighbour's
    // position and (mixed path) its records one iteration ahead
    constexpr bool PRE = HL;
    unsigned ent_nn = nn > 1 ? __ldg(&D.pairs[(size_t)P.nbr_stride + a]) : 0u;
    double2 xb_n = make_double2(0.0, 0.0);
    float4 xbhl_n = make_float4(0.f, 0.f, 0.f, 0.f);
    double vd_n = 0.0;                 // FP64 volume, mixed SHIFT launch
    constexpr bool VPRE = HL && SHIFT;
    Side<R> T_n;
    auto load_records = [&](int bb, Side<R>& t) {
        if (HL) { t.kh = D.kh[bb]; t.kl = D.kl[bb]; }
        else t.kin = D.kin[bb];
        t.aux = D.aux[bb]; t.nb1 = D.nb1[bb]; t.nb2 = D.nb2[bb];
        if (MUSCL) t.nb3 = D.nb3[bb];
    };
    if (nn > 0) {
        const int b0 = (int)(ent_n & 0x7fffffffu);
        if (X64) xb_n = __ldg(&D.pos[b0]);
        else xbhl_n = __ldg(&D.xhl[b0]);
        if (VPRE) vd_n = __ldg(&D.vol64[b0]);
        if (PRE) load_records(b0, T_n);
    }
    for (int e = 0; e < nn; ++e) {
        const unsigned ent = ent_n;
        const int b = (int)(ent & 0x7fffffffu);
        const bool a_is_i = (ent >> 31) != 0;
        const double2 xb = xb_n;
        const float4 xbhl = xbhl_n;
        const double vd_b = vd_n;
        Side<R> T;
        if (PRE) T = T_n;
        if (e + 1 < nn) {
            ent_n = ent_nn;
            const int b1 = (int)(ent_n & 0x7fffffffu);
            if (X64) xb_n = __ldg(&D.pos[b1]);
            else xbhl_n = __ldg(&D.xhl[b1]);
            if (VPRE) vd_n = __ldg(&D.vol64[b1]);
            if (PRE) load_records(b1, T_n);
            if (e + 2 < nn) ent_nn = __ldg(&D.pairs[(size_t)(e + 2) * P.nbr_stride + a]);
        }
        // x_a - x_b: FP64, or hi/lo in FP32 (the mixed SHIFT launch: the FP32
        // rounding of the FP64 difference, which its shifting sum needs)
        double dxd = 0.0, dyd = 0.0;
        if (X64) { dxd = xa.x - xb.x; dyd = xa.y - xb.y; }
        const float dxf = !HL ? 0.f : X64 ? (float)dxd : (xa_hl.x - xbhl.x) + (xa_hl.z - xbhl.z);
        const float dyf = !HL ? 0.f : X64 ? (float)dyd : (xa_hl.y - xbhl.y) + (xa_hl.w - xbhl.w);
        R d, inv_d;
        if (F32) {
            const R s = HL ? (R)(dxf * dxf + dyf * dyf) : (R)(dxd * dxd + dyd * dyd);
            inv_d = rsqrtf(s);
            d = s * inv_d;
        } else {
            d = (R)sqrt(dxd * dxd + dyd * dyd);
            inv_d = R(1) / d;
        }
        if (!PRE) load_records(b, T);
        // the pair's i and j members (only the moving-square HLLC state reads
        // them; everything else is formed from a's and b's records directly)
        const Side<R>& I = a_is_i ? S : T;
        const Side<R>& J = a_is_i ? T : S;
        const R sgn = a_is_i ? R(1) : R(-1);
        // AB (the mixed MUSCL Taylor-Green launch): the pair terms are formed in a's
        // frame, x_a - x_b and phi_a - phi_b, instead of the pair's i/j frame.
        // Negation is exact, so a term odd in the orientation takes the i/j-frame
        // bits times sgn and the sgn of the final sums cancels it: sgn stays only
        // where the MUSCL limiter needs the i/j frame.
        constexpr bool AB = F32 && MUSCL && !MS;
        // position_difference_ij = x_i - x_j (find_particle_pair.f90:79-107) = sgn (x_a - x_b);
        // xij: that, or x_a - x_b in AB
        R xab0, xab1;
        if (HL) { xab0 = (R)dxf; xab1 = (R)dyf; }
        else { xab0 = (R)dxd; xab1 = (R)dyd; }
        const R xij0 = AB ? xab0 : sgn * xab0, xij1 = AB ? xab1 : sgn * xab1;
        const R fsg = AB ? R(1) : sgn;      // the orientation of the frame's sums
        // pair differences, FP64 or hi/lo in FP32, formed as a - b and oriented
        // by sgn: b - a is exactly -(a - b), so both members of the pair get the
        // same bits, and sums such as rho_i + rho_j are a's plus b's
        R du, dv, dp, drho_ji, rho_a_, rho_b;
        if (HL) {
            du = fsg * (R)((S.kh.x - T.kh.x) + (S.kl.x - T.kl.x));
            dv = fsg * (R)((S.kh.y - T.kh.y) + (S.kl.y - T.kl.y));
            dp = fsg * (R)((S.kh.w - T.kh.w) + (S.kl.w - T.kl.w));
            drho_ji = -(fsg * (R)((S.kh.z - T.kh.z) + (S.kl.z - T.kl.z)));
            rho_a_ = (R)S.kh.z; rho_b = (R)T.kh.z;
        } else {
            du = sgn * (R)(S.kin.x - T.kin.x); dv = sgn * (R)(S.kin.y - T.kin.y);
            dp = sgn * (R)(S.kin.w - T.kin.w);
            drho_ji = -(sgn * (R)(S.kin.z - T.kin.z));
            rho_a_ = (R)S.kin.z; rho_b = (R)T.kin.z;
        }
        // compute_kernel: W and dwdx(k) = g (x_i - x_j).  FP32: g with
        // q/(d h) = 1/h^2 folded into a constant (gk)
        R w, g;
        {
            const R q = d * inv_h;
            const R kf = (R)P.kfactor;
            if (P.kernel_model == SPH_KERNEL_GAUSSIAN) {
                const R ex = exp(-(q * q));
                w = (ex - (R)P.gauss_e9) * kf;
                g = F32 ? ex * gk : ex * (R(-2) * q) * inv_d * inv_h * kf;
            } else {
                const R t = R(1) - R(0.5) * q;
                const R t3 = t * t * t;
                w = kf * (R(1) + R(2) * q) * (t3 * t);
                g = F32 ? t3 * gk : kf * (R(-5) * q * t3) * inv_d * inv_h;
            }
        }
        const R dw0 = g * xij0, dw1 = g * xij1;
        // Normalized_dwdx of this particle's side: B_a^-1 dwdx(k)
        const R nd0 = bi.x * dw0 + bi.y * dw1;
        const R nd1 = bi.z * dw0 + bi.w * dw1;
        const R cbar = R(0.5) * (S.aux.z + T.aux.z);
        const R rbar = R(0.5) * (rho_a_ + rho_b);
        const R inv_rbar = fast_quot(R(1), rbar);
        const R e0 = -xij0 * inv_d, e1 = -xij1 * inv_d;     // x_j - x_i direction (both solvers)
        // Riemann states.  li/lj are the MUSCL reconstruction increments
        // (function_module.f90:34-80); the modified solver has none.
        R lpi = R(0), lpj = R(0), lui = R(0), luj = R(0), lvi = R(0), lvj = R(0);
        if (MUSCL) {
            // DelPhi_i = 0.5 grad phi_i.(x_j - x_i), DelPhi_j = -0.5 grad phi_j.(x_j - x_i):
            // with ga = 0.5 grad phi_a.(x_a - x_b), gb = 0.5 grad phi_b.(x_a - x_b),
            // (DelPhi_i, DelPhi_j) = (-ga, gb) when a is pair_i and (gb, -ga) when it is
            // pair_j.  The products are rounded separately and fused in a fixed order,
            // so both members of the pair form the same bits.
            // nb2 = (grad rho y, grad p x, grad p y, grad u x), nb3 = (grad u y, grad v x, grad v y, 1/rho),
            // the gradients halved in the FP32 records
            // (the FP32 records hold 1/2 grad phi, so the halving is already done, exactly)
            auto half_dot = [&](R g0, R g1) { return (F32 ? R(1) : R(0.5)) * fma(g1, xab1, mul_rn(g0, xab0)); };
            const R gpa = half_dot(S.nb2.y, S.nb2.z), gpb = half_dot(T.nb2.y, T.nb2.z);
            const R gua = half_dot(S.nb2.w, S.nb3.x), gub = half_dot(T.nb2.w, T.nb3.x);
            const R gva = half_dot(S.nb3.y, S.nb3.z), gvb = half_dot(T.nb3.y, T.nb3.z);
            if constexpr (AB) {
                // the limiter in the i/j frame (dij = phi_j - phi_i = -sgn (phi_a - phi_b)),
                // its sum and own-side increment taken back to a's frame by sgn;
                // lpi etc. then hold sgn L and the own increment (lpj, luj, lvj unused)
                float L, own;
                muscl_limiter_sum(a_is_i ? -gpa : gpb, a_is_i ? gpb : -gpa, -(sgn * dp), a_is_i, L, own);
                lpi = sgn * L;
                muscl_limiter_sum(a_is_i ? -gua : gub, a_is_i ? gub : -gua, -(sgn * du), a_is_i, L, own);
                lui = sgn * L; luj = sgn * own;
                muscl_limiter_sum(a_is_i ? -gva : gvb, a_is_i ? gvb : -gva, -(sgn * dv), a_is_i, L, own);
                lvi = sgn * L; lvj = sgn * own;
            } else {
                muscl_limiter<R>(a_is_i ? -gpa : gpb, a_is_i ? gpb : -gpa, -dp, lpi, lpj);
                muscl_limiter<R>(a_is_i ? -gua : gub, a_is_i ? gub : -gua, -du, lui, luj);
                muscl_limiter<R>(a_is_i ? -gva : gvb, a_is_i ? gvb : -gva, -dv, lvi, lvj);
            }
        }
        // U_L - U_R and P_L - P_R from the differences (AB: the frame's e0, e1 and
        // differences; the product is the i/j frame's)
        const R dU = AB ? (du + lui) * e0 + (dv + lvi) * e1 : (du + lui + luj) * e0 + (dv + lvi + lvj) * e1;
        const R Pbar = HL ? R(0.5) * ((R)S.kh.w + (R)T.kh.w) : R(0.5) * ((R)S.kin.w + (R)T.kin.w);
        R PA, wa0, wa1;          // this side's star pressure and velocity minus star velocity
        if (AB) { wa0 = R(0.5) * du + luj; wa1 = R(0.5) * dv + lvj; }
        else if (a_is_i) { wa0 = R(0.5) * du + lui; wa1 = R(0.5) * dv + lvi; }
        else { wa0 = R(-0.5) * du - luj; wa1 = R(-0.5) * dv - lvj; }
        if (!MS || !P.hllc) {
            // AB: dP and U* - Ubar in a's frame; sU e is the i/j frame's product
            const R dP = AB ? dp + lpi : dp + lpi + lpj;
            const R sU = R(0.5) * dP * (inv_rbar * inv_sqc0);               // U* - Ubar
            const R bR = min(R(3) * (max(dU, R(0))), cbar);
            const R Ps = Pbar + R(0.5) * bR * rbar * dU;
            PA = near_a ? Pbar : Ps;
            if (!near_a) { wa0 -= sU * e0; wa1 -= sU * e1; }
        } else if (near_a) {
            PA = Pbar;
        } else if (HL) {
            // The HLLC state of Moving_Square.../Solver_Normalized_HLLC_Riemann_Delta.f90:207-322
            // written in differences, so that FP32 keeps the accuracy of the hi/lo pair
            // differences (rho* and P* = c0^2 (rho_HLLC - rho0) are otherwise differences of
            // O(1) numbers).  Pair frame e (i to j) and t = (-e1, e0); dV = VR0 - VL0 =
            // -(du, dv).e; C_K = rho_K c_K; the reference's contact speed
            // U* = (VR0 C_L + VL0 C_R + P_L - P_R)/(C_L + C_R) gives
            //   sL = U* - VL0 = (C_L dV + dp)/(C_L + C_R),  sR = U* - VR0 = (dp - C_R dV)/(C_L + C_R),
            //   P* - P_L = -C_L (dp + C_R dV)/(C_L + C_R);
            // the state sampled at V0 = (VL0 + VR0)/2, V0 - VL0 = VR0 - V0 = dV/2, gives
            //   rho_HLLC - rho0 = (rho_K - rho0) [+ rho_K (U* - V_K0)/(S_K - U*) in the star regions]
            // and v_K - v* as components along e and t.
            const R rL = a_is_i ? rho_a_ : rho_b, rR = a_is_i ? rho_b : rho_a_;
            const R cL = a_is_i ? (R)S.aux.z : (R)T.aux.z, cR = a_is_i ? (R)T.aux.z : (R)S.aux.z;
            const R rho0f = (R)P.rho0;
            const R dra = (R)((S.kh.z - (float)rho0f) + S.kl.z), drb = (R)((T.kh.z - (float)rho0f) + T.kl.z);
            const R drL = a_is_i ? dra : drb, drR = a_is_i ? drb : dra;   // rho - rho0
            const R CL = rL * cL, CR = rR * cR;
            const R iC = rcp(CL + CR);
            const R dV = -(e0 * du + e1 * dv);
            const R sL = (CL * dV + dp) * iC;
            const R sR = (dp - CR * dV) * iC;
            const R dPL = -(CL * (dp + CR * dV)) * iC;     // P* - P_L
            const R dPR = dPL + dp;                        // P* - P_R
            // shock factor (:243-275): taken when P* > P_K and rho_K > rho*.  With the linear
            // equation of state rho_K - rho* = -(P* - P_K)/c0^2, so the branch is never taken.
            R QL = R(1), QR = R(1);
            if (P.eos != SPH_EOS_LINEAR) {
                const R ic0 = (R)(1.0 / P.c0sq), pbf = (R)P.pb;
                const R pa_ = (R)(S.kh.w + S.kl.w), pbb = (R)(T.kh.w + T.kl.w);
                const R pL = a_is_i ? pa_ : pbb, pR = a_is_i ? pbb : pa_;
                const R gL = drL - (pL - pbf) * ic0 - dPL * ic0;     // rho_L - rho*
                const R gR = drR - (pR - pbf) * ic0 - dPR * ic0;     // rho_R - rho*
                if (dPL > R(0) && gL > R(0)) QL = sqrt(((rL - gL) / rL) * dPL / gL) / cL;
                if (dPR > R(0) && gR > R(0)) QR = sqrt(((rR - gR) / rR) * dPR / gR) / cR;
            }
            const R sLm = -cL * QL, sRm = cR * QR;         // S_L - VL0, S_R - VR0
            const R hdV = R(0.5) * dV;
            const R tdv = e1 * du - e0 * dv;               // VR1 - VL1
            R dH, aI, bI, aJ, bJ;       // rho_HLLC - rho0; v_i - v* = aI e + bI t, v_j - v* = aJ e + bJ t
            if (sLm > hdV) {                                        // S_L > V0: the left state
                dH = drL; aI = R(0); bI = R(0); aJ = dV; bJ = tdv;
            } else if (sL - hdV >= R(0) && hdV >= sLm) {            // U* >= V0 >= S_L
                dH = drL + rL * quot(sL, sLm - sL);
                aI = -sL; bI = R(0); aJ = -sR; bJ = tdv;
            } else if (sRm >= -hdV && sL - hdV <= R(0)) {           // S_R >= V0 >= U*
                dH = drR + rR * quot(sR, sRm - sR);
                aI = -sL; bI = -tdv; aJ = -sR; bJ = R(0);
            } else {                                                // the right state
                dH = drR; aI = -dV; bI = -tdv; aJ = R(0); bJ = R(0);
            }
            PA = (R)P.c0sq * dH + (R)P.pb;
            const R al = a_is_i ? aI : aJ, be = a_is_i ? bI : bJ;
            wa0 = al * e0 - be * e1;
            wa1 = al * e1 + be * e0;
        } else {
            // HLLC in the pair frame (Moving_Square.../Solver_Normalized_HLLC_Riemann_Delta.f90:207-322),
            // FP64 path: the reference's own operations
            const double ed0 = -(a_is_i ? dxd : -dxd) / sqrt(dxd * dxd + dyd * dyd);
            const double ed1 = -(a_is_i ? dyd : -dyd) / sqrt(dxd * dxd + dyd * dyd);
            const double uI = I.kin.x, vI = I.kin.y, uJ = J.kin.x, vJ = J.kin.y;
            const double VL0 = ed0 * uI + ed1 * vI, VL1 = -ed1 * uI + ed0 * vI;
            const double VR0 = ed0 * uJ + ed1 * vJ, VR1 = -ed1 * uJ + ed0 * vJ;
            const double V0 = ed0 * (0.5 * (uI + uJ)) + ed1 * (0.5 * (vI + vJ));
            const double rL = I.kin.z, rR = J.kin.z, cL = (double)I.aux.z, cR = (double)J.aux.z;
            const double PLd = I.kin.w, PRd = J.kin.w;
            const double den = rL * cL + rR * cR;
            const double Us = (VR0 * cL * rL + VL0 * cR * rR + PLd - PRd) / den;
            const double Pst = (PRd * cL * rL + PLd * cR * rR - cL * rL * cR * rR * (VR0 - VL0)) / den;
            const double rst = (Pst - P.pb) / P.c0sq + P.rho0;
            double QL = 1.0, QR = 1.0;
            if (!(Pst <= PLd) && rL > rst) QL = sqrt((rst / rL) * (Pst - PLd) / (rL - rst)) / cL;
            const double SL = VL0 - cL * QL;
            if (!(Pst <= PRd) && rR > rst) QR = sqrt((rst / rR) * (Pst - PRd) / (rR - rst)) / cR;
            const double SR = VR0 + cR * QR;
            double rH, VH0, VH1;
            if (SL > V0) { rH = rL; VH0 = VL0; VH1 = VL1; }
            else if (Us >= V0 && V0 >= SL) {
                const double q = rL * ((SL - VL0) / (SL - Us));
                rH = q; VH0 = (Us * q) / rH; VH1 = (VL1 * q) / rH;
            } else if (SR >= V0 && V0 >= Us) {
                const double q = rR * ((SR - VR0) / (SR - Us));
                rH = q; VH0 = (Us * q) / rH; VH1 = (VR1 * q) / rH;
            } else { rH = rR; VH0 = VR0; VH1 = VR1; }
            const double vs0 = ed0 * VH0 - ed1 * VH1, vs1 = ed1 * VH0 + ed0 * VH1;
            PA = (R)(P.c0sq * (rH - P.rho0) + P.pb);
            const double4& K = S.kin;
            wa0 = (R)(K.x - vs0);
            wa1 = (R)(K.y - vs1);
        }
        if (MS) {        // XSPH velocities inside the continuity flux (MS solvers :199-202)
            const typename VT<R>::V2 avg_b = D.avg[b];
            wa0 += avg_a.x - avg_b.x;
            wa1 += avg_a.y - avg_b.y;
        }
        const R Vb = T.aux.y, mb = T.aux.x;
        // continuity (:360-369)
        R dr = R(2) * rho_a * Vb * (fsg * (wa0 * nd0 + wa1 * nd1));
        // pressure force (:374-388)
        const R rho_ij = inv_rho_a * (RREC ? (R)T.nb3.w : rcp(rho_b));
        const R fp = R(-2) * PA * rho_ij * mb;
        R tx = fp * nd0, ty = fp * nd1;
        // artificial viscosity (:392-417)
        const R inv_r2 = inv_d * inv_d;
        const R vx = du * xij0 + dv * xij1;
        if (vx < R(0)) {
            const R phi1 = fast_quot(hbar * vx, d * d + fh2);
            const R Pi = (-alpha * cbar * phi1 + beta * (phi1 * phi1)) * inv_rbar;
            tx += mb * (-Pi * nd0);
            ty += mb * (-Pi * nd1);
        }
        // (x_i - x_j).B^-1 dwdx / r^2, shared by the laplacian and delta-SPH (FP32)
        const R xnd = (xij0 * nd0 + xij1 * nd1) * inv_r2;
        if (!MS || P.laplacian == 1) {
            // Morris laplacian (:432-436)
            const R lf = F32 ? Vb * nu2 * xnd : Vb * nu2 * (xij0 * nd0 + xij1 * nd1) * inv_r2;
            tx += lf * du;
            ty += lf * dv;
        } else {
            // laplacianTerm 0 (Moving_Square.../Solver_..._Delta.f90:315-318): 2 (dim+2) nu V (v.x)/r^2 grad W
            const R lf = Vb * R(4) * nu2 * vx * inv_r2;
            tx += lf * nd0;
            ty += lf * nd1;
        }
        // delta-alpha artificial internal acceleration (:442-446)
        const R tt = F32 ? dla_rho * cbar * (vx * inv_r2) * Vb : dla_h * cbar * vx * inv_r2 * rho0_over_rho_a * Vb;
        tx += tt * nd0;
        ty += tt * nd1;
        // SPS force, unnormalised dwdx and the neighbour's SPS mass (:450-492);
        // the reference does not reset temp_p between x and y (kept with quirks)
        if (!MS) {
            const R sxx = S.nb1.x + T.nb1.x, sxy = S.nb1.y + T.nb1.y, syy = S.nb1.z + T.nb1.z;
            R tp = (sxx * dw0 + sxy * dw1) * rho_ij;
            const R smb = T.aux.w;
            tx += smb * tp;
            if (!P.quirks) tp = R(0);
            tp = (tp + syy * dw1 + sxy * dw0) * rho_ij;
            ty += smb * tp;
        }
        accx.add(fsg * tx);
        accy.add(fsg * ty);
        // XSPH average velocity (:495-500; modified solver only)
        if (!MUSCL && !MS && P.xsph) {
            const R f = eps2 * mb * rcp(rho_a_ + rho_b) * w;
            xsx -= sgn * (f * du);
            xsy -= sgn * (f * dv);
        }
        // delta-SPH density diffusion (:552-583): psi = (rho_j - rho_i) - 0.5 (grad rho_i + grad rho_j).(x_j - x_i)
        if (water) {
            const R sg0 = S.nb1.w + T.nb1.w, sg1 = S.nb2.x + T.nb2.x;
            if (dsph) {
                // Antuono form (Solver_Normalized_Delta_SPH_SPS.f90:610-636):
                // psi = 2 (rho_j - rho_i) (x_j - x_i)/r^2 - (grad rho_i + grad rho_j), D += delta h c psi.gradW V
                const R f = R(2) * drho_ji * inv_r2;
                const R gsc = F32 ? R(2) : R(1);      // FP32 records: 1/2 grad rho
                const R p0 = -(f * xij0) - gsc * sg0, p1 = -(f * xij1) - gsc * sg1;
                dr += sgn * (dla_dh * cbar * (p0 * nd0 + p1 * nd1) * Vb);
            } else {
                const R psi = drho_ji + (F32 ? R(1) : R(0.5)) * (sg0 * xij0 + sg1 * xij1);
                const R tma = F32 ? -xnd : -(xij0 * nd0 + xij1 * nd1) * inv_r2;
                dr += fsg * (dlt2h * cbar * psi * tma * Vb);
            }
        }
        cont.add(dr);
        // particle shifting sum (Shift_particle_position.f90:97-100), FP64:
        // shift_a = -beta h^2 B_a^-1 sum_b (1 + R (W/W(dx))^n) grad_a W_ab V_b
        if (SHIFT) {
            double gd, wd, Vd;
            if (F32) {
                // FP64 without divisions: q = d/h, grad factor G = g/(d h) = -5 k t^3/h^2
                // (Wendland) or -2 k e^{-q^2}/h^2 (Gaussian), V_b from the FP64 volume record.
                // The distance: one Newton (Heron) step for sqrt(s) from the FP32
                // distance d0 (relative error ~1e-7), d = d0 + (s - d0^2)/(2 d0),
                // leaves a relative error of order 1e-14
                const double d0 = (double)d;
                const double dd2 = fma(fma(-d0, d0, dxd * dxd + dyd * dyd), 0.5 * (double)inv_d, d0);
                const double q = dd2 * inv_h64;
                if (P.kernel_model == SPH_KERNEL_GAUSSIAN) {
                    const double ex = exp(-(q * q));
                    wd = (ex - P.gauss_e9) * P.kfactor;
                    gd = -2.0 * P.kfactor * ex * inv_h2_64;
                } else {
                    const double t = 1.0 - 0.5 * q;
                    const double t2 = t * t;
                    wd = P.kfactor * (1.0 + 2.0 * q) * (t2 * t2);
                    gd = -5.0 * P.kfactor * (t2 * t) * inv_h2_64;
                }
                Vd = VPRE ? vd_b : __ldg(&D.vol64[b]);
            } else {
                wd = (double)w; gd = (double)g; Vd = (double)Vb;
            }
            const double r = wd * inv_wdx;
            const double r2 = r * r;
            const double f = (1 + P.shift_R * (r2 * r2)) * Vd * gd;
            shx += f * dxd;
            shy += f * dyd;
        }
    }
    // assembly (single_step_compute.f90:152-171, Solver :627-635)
    D.drho[a] = cont.val();
    D.acc[a] = water ? mk2<R>(accx.val(), accy.val()) : mk2<R>(R(0), R(0));
    if (!MS) D.avg[a] = mk2<R>(xsx, xsy);
    if (SHIFT) {
        const double4 b64 = D.binv64[a];
        const double c = -P.shift_beta * (P.h * P.h);
        D.shift[a] = make_double2(c * (b64.x * shx + b64.y * shy), c * (b64.z * shx + b64.w * shy));
    }
}

// The particle shifting sum of the mixed Taylor-Green path as a gather of its
// own, launched after pass C on the last RHS of a step (Shift_particle_position.f90:
// 56-100): shift_a = -beta h^2 B_a^-1 sum_b (1 + R (W/W(dx))^4) grad_a W_ab V_b in
// FP64, over the RHS's pair list, with the FP64 positions and volumes.  The same
// sum inside mixed pass C holds its FP64 values at pass C's register bound and
// stalls on their loads; here it runs at full occupancy.  Particles the shift
// does not move (not water, or near the free surface) get 0.  12 blocks of 128
// per SM (40 registers, 24 B spilled): 0.32 -> 0.29 ms per step at 2048^2
// against 44 registers at 11 blocks; at 16 blocks (32 registers, 48 B
// spilled) it was slower.
template <typename R>
__global__ void __launch_bounds__(128, 12) k_shift_gather(Params P, Sorted<R> D) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= P.n_tot) return;
    if (D.type[a] != SPH_TYPE_WATER || (D.flags[a] & 2)) {
        D.shift[a] = make_double2(0.0, 0.0);
        return;
    }
    const int nn = D.npairs[a];
    const double2 xa = D.pos[a];
    const double inv_h64 = 1.0 / P.h, inv_h2_64 = inv_h64 * inv_h64, inv_wdx = 1.0 / P.w_dx;
    double shx = 0.0, shy = 0.0;
    // the pair entry two iterations ahead, the neighbour's position and volume one ahead
    unsigned ent_n = nn > 0 ? __ldg(&D.pairs[a]) : 0u;
    unsigned ent_nn = nn > 1 ? __ldg(&D.pairs[(size_t)P.nbr_stride + a]) : 0u;
    double2 xb_n = make_double2(0.0, 0.0);
    double vd_n = 0.0;
    if (nn > 0) {
        const int b0 = (int)(ent_n & 0x7fffffffu);
        xb_n = __ldg(&D.pos[b0]);
        vd_n = __ldg(&D.vol64[b0]);
    }
    for (int e = 0; e < nn; ++e) {
        const double2 xb = xb_n;
        const double Vd = vd_n;
        if (e + 1 < nn) {
            ent_n = ent_nn;
            const int b1 = (int)(ent_n & 0x7fffffffu);
            xb_n = __ldg(&D.pos[b1]);
            vd_n = __ldg(&D.vol64[b1]);
            if (e + 2 < nn) ent_nn = __ldg(&D.pairs[(size_t)(e + 2) * P.nbr_stride + a]);
        }
        const double dxd = xa.x - xb.x, dyd = xa.y - xb.y;
        const double s2 = dxd * dxd + dyd * dyd;
        // distance: FP32 estimate, then one Newton (Heron) step for sqrt(s2),
        // d = d0 + (s2 - d0^2)/(2 d0): relative error of order 1e-14
        const float sf = (float)s2;
        const float yf = rsqrtf(sf);
        const double d0 = (double)(sf * yf);
        const double dd = fma(fma(-d0, d0, s2), 0.5 * (double)yf, d0);
        const double q = dd * inv_h64;
        // grad factor G = g/(d h) and W (compute_kernel), FP64 without divisions
        double wd, gd;
        if (P.kernel_model == SPH_KERNEL_GAUSSIAN) {
            const double ex = exp(-(q * q));
            wd = (ex - P.gauss_e9) * P.kfactor;
            gd = -2.0 * P.kfactor * ex * inv_h2_64;
        } else {
            const double t = 1.0 - 0.5 * q;
            const double t2 = t * t;
            wd = P.kfactor * (1.0 + 2.0 * q) * (t2 * t2);
            gd = -5.0 * P.kfactor * (t2 * t) * inv_h2_64;
        }
        const double r = wd * inv_wdx;
        const double r2 = r * r;
        const double f = (1 + P.shift_R * (r2 * r2)) * Vd * gd;
        shx += f * dxd;
        shy += f * dyd;
    }
    const double4 b64 = D.binv64[a];
    const double c = -P.shift_beta * (P.h * P.h);
    D.shift[a] = make_double2(c * (b64.x * shx + b64.y * shy), c * (b64.z * shx + b64.w * shy));
}

}  // namespace sph
