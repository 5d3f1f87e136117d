// pass_a.cuh -- neighbour pass A (one thread per particle, gather form):
// volume fraction, renormalisation tensor and its inverse, normalised
// gradients of rho / p / u / v, SPS strain and stress.
//
// Reference: Define_freesurface_and_Normailized_derivates.f90:79-188 (fra_v,
// Tensor_dyadic_matrix, inverse), Solver_Normalized_Modified_Linear_Riemann_Delta_SPS.f90:
// 126-139 (normalised dW), :144-182 and :256-296 (SPS), :508-526 (grad rho),
// Solver_Normalized_MUSCL_Linear_Riemann_Delta_SPS.f90:151-185 (grad p, u, v).
//
// Gather form of the reference's pair scatter: for particle a and pair
// neighbour b, grad_a W_ab = f(d) (x_a - x_b) is the reference's dwdx(k) when a
// is pair_i and -dwdx(k) when a is pair_j, so every scatter term becomes
// "sum over b of (phi_b - phi_a) V_b B_a^-1 grad_a W_ab".  Since B_a^-1 is the
// same matrix for all b, the raw sums are accumulated first and multiplied by
// B_a^-1 once (exact in real arithmetic).
#pragma once
#include "setup.cuh"

namespace sph {

// HLREC: in the mixed path, read the hi/lo float records (position, u, v, rho, p)
// instead of the FP64 ones and form the pair differences in FP32 from them
// (see store_split); the adjoint, which runs this pass on stored stage states
// that carry only the FP64 records, uses HLREC = false.  The Taylor-Green
// launch forms the differences of u, v, rho and p from the hi parts alone (the
// position difference keeps hi + lo: the kernel and B need it to the FP32
// rounding of the FP64 difference): each gradient term is an FP32 product
// summed in FP32, and at 2048^2 dropping the lo record took this pass from
// 2.07 to 1.87 ms per step (1.80 at 8 blocks per SM) while the velocity L2
// against FP64 after 100 steps went from 2.78e-6 to 2.83e-6 and the density
// error (relative to its variation) from 2.46e-5 to 2.70e-5.  MS: the
// moving-square solvers (P.ms), whose XSPH sum is formed here and which keep
// the hi + lo differences; compile-time so that the Taylor-Green launches carry
// none of its registers.
#ifndef SPH_PASS_A_F32_BLOCKS
#define SPH_PASS_A_F32_BLOCKS 8
#endif
#ifndef SPH_PASS_A_F32_MS_BLOCKS
#define SPH_PASS_A_F32_MS_BLOCKS 7
#endif
template <typename R, bool HLREC, bool MS>
__global__ void __launch_bounds__(128, sizeof(R) == 4 ? (MS ? SPH_PASS_A_F32_MS_BLOCKS : SPH_PASS_A_F32_BLOCKS) : 4)
    k_pass_a(Params P, Sorted<R> D) {
    using V4 = typename VT<R>::V4;
    constexpr bool F32 = sizeof(R) == 4;
    constexpr bool HL = HLREC && F32;
    constexpr bool LO = HL && MS;        // the lo parts of u, v, rho, p
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= P.n_tot) return;
    const int ta = D.type[a];
    const int nn = D.nnbr[a];
    const double2 xa = HL ? make_double2(0.0, 0.0) : D.pos[a];
    const double4 ka = HL ? make_double4(0.0, 0.0, __ldg(&D.kin[a].z), 0.0) : D.kin[a];
    const float4 xa_hl = HL ? D.xhl[a] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 kah = HL ? D.kh[a] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 kal = LO ? D.kl[a] : make_float4(0.f, 0.f, 0.f, 0.f);
    const double rho_a = ka.z;
    // the sums of this pass have no large cancellation (differences of smooth
    // fields, or B ~ I), so FP32 accumulates them directly in the mixed path
    R fra = R(0), b00 = R(0), b01 = R(0), b10 = R(0), b11 = R(0);
    R g[8];
    for (int c = 0; c < 8; ++c) g[c] = R(0);
    // moving-square solvers: XSPH average velocity, computed before their main
    // loop (Solver_Normalized_..._Delta.f90:114-121):
    //   avg_a = -epsilon sum_b m_b (v_a - v_b) / (rho_a + rho_b) W_ab
    R xs0 = R(0), xs1 = R(0);
    const R inv_h = (R)(1.0 / P.h);
    const R r2cut = (R)(P.r_cut * P.r_cut), r2min = (R)(P.cut_min * P.cut_min);
    int np = 0;
    // two-deep software pipeline: the list entry two iterations ahead, the
    // neighbour's position and records (kin, volume) one iteration ahead, so the
    // loads of the next neighbour are in flight while this one is evaluated
    unsigned ent_n = nn > 0 ? __ldg(&D.nbr[a]) : 0u;
    unsigned ent_nn = nn > 1 ? __ldg(&D.nbr[(size_t)P.nbr_stride + a]) : 0u;
    double2 xb_n = make_double2(0.0, 0.0);
    double4 kb_n = make_double4(0.0, 0.0, 0.0, 0.0);
    float4 xbhl_n = make_float4(0.f, 0.f, 0.f, 0.f), kbh_n = xbhl_n, kbl_n = xbhl_n;
    R vb_n = R(0);
    auto fetch = [&](int bb) {
        if (HL) { xbhl_n = __ldg(&D.xhl[bb]); kbh_n = __ldg(&D.kh[bb]); if (LO) kbl_n = __ldg(&D.kl[bb]); }
        else { xb_n = __ldg(&D.pos[bb]); kb_n = D.kin[bb]; }
        vb_n = D.aux[bb].y;
    };
    if (nn > 0) fetch((int)(ent_n & 0x7fffffffu));
    for (int e = 0; e < nn; ++e) {
        const unsigned ent = ent_n;
        const int b = (int)(ent & 0x7fffffffu);
        const double2 xb = xb_n;
        const double4 kb = kb_n;
        const float4 xbhl = xbhl_n, kbh = kbh_n, kbl = kbl_n;
        const R Vb = vb_n;
        if (e + 1 < nn) {
            ent_n = ent_nn;
            fetch((int)(ent_n & 0x7fffffffu));
            if (e + 2 < nn) ent_nn = __ldg(&D.nbr[(size_t)(e + 2) * P.nbr_stride + a]);
        }
        const double dxd = HL ? 0.0 : xa.x - xb.x, dyd = HL ? 0.0 : xa.y - xb.y;
        const float dxf = HL ? (xa_hl.x - xbhl.x) + (xa_hl.z - xbhl.z) : 0.f;
        const float dyf = HL ? (xa_hl.y - xbhl.y) + (xa_hl.w - xbhl.w) : 0.f;
        R d, inv_d;
        if (F32) {
            const R s = HL ? (R)(dxf * dxf + dyf * dyf) : (R)(dxd * dxd + dyd * dyd);
            if (!(s <= r2cut) || s < r2min) continue;
            inv_d = rsqrtf(s);
            d = s * inv_d;
        } else {
            double dd;
            if (!in_support(P, dxd, dyd, dd)) continue;
            d = (R)dd;
            inv_d = R(1) / d;
        }
        D.pairs[(size_t)np * P.nbr_stride + a] = ent;
        ++np;
        const R dx = HL ? (R)dxf : (R)dxd, dy = HL ? (R)dyf : (R)dyd;
        // grad_a W = g(d) (x_a - x_b)  (compute_kernel)
        R gs, wk;
        {
            const R q = d * inv_h;
            const R kf = (R)P.kfactor;
            if (P.kernel_model == SPH_KERNEL_GAUSSIAN) {
                const R ex = exp(-(q * q));
                wk = (ex - (R)P.gauss_e9) * kf;
                gs = ex * (R(-2) * q) * inv_d * inv_h * kf;
            } else {
                const R t = R(1) - R(0.5) * q;
                const R t3 = t * t * t;
                wk = kf * (R(1) + R(2) * q) * (t3 * t);
                gs = kf * (R(-5) * q * t3) * inv_d * inv_h;
            }
        }
        // differences of the records (b minus a): FP64, or hi/lo in FP32
        R drho, du, dv, dp;
        if (LO) {
            drho = (R)((kbh.z - kah.z) + (kbl.z - kal.z));
            du = (R)((kbh.x - kah.x) + (kbl.x - kal.x));
            dv = (R)((kbh.y - kah.y) + (kbl.y - kal.y));
            dp = (R)((kbh.w - kah.w) + (kbl.w - kal.w));
        } else if (HL) {
            drho = (R)(kbh.z - kah.z);
            du = (R)(kbh.x - kah.x);
            dv = (R)(kbh.y - kah.y);
            dp = (R)(kbh.w - kah.w);
        } else {
            drho = (R)(kb.z - ka.z);
            du = (R)(kb.x - ka.x); dv = (R)(kb.y - ka.y);
            dp = (R)(kb.w - ka.w);
        }
        if (MS) {
            const R rsum = HL ? (R)(kah.z + kbh.z) : (R)(ka.z + kb.z);
            const R f = (R)P.eps * D.aux[b].x / rsum * wk;
            xs0 += f * du;
            xs1 += f * dv;
        }
        const R gx = gs * dx * Vb, gy = gs * dy * Vb;    // V_b grad_a W
        // volume fraction (Define_freesurface...f90:84-85)
        fra += Vb;
        // B(l,o) += (x_b - x_a)_l grad_a W_o V_b (:151-152)
        b00 -= dx * gx; b01 -= dx * gy;
        b10 -= dy * gx; b11 -= dy * gy;
        // raw gradient sums (phi_b - phi_a) V_b grad_a W
        g[0] += drho * gx; g[1] += drho * gy;
        g[4] += du * gx; g[5] += du * gy;
        g[6] += dv * gx; g[7] += dv * gy;
        if (P.muscl) { g[2] += dp * gx; g[3] += dp * gy; }
    }
    D.npairs[a] = np;
    fra = fra * (R)(1.0 / P.sv);
    // inverse of the 2x2 tensor in FP64 (matrix_inversion_less_three,
    // function_module.f90:190-204); the reference keeps the identity on success
    // (Define_freesurface...f90:180-186) unless renormalisation is switched on.
    double i00 = 1.0, i01 = 0.0, i10 = 0.0, i11 = 1.0;
    // the moving-square variant also inverts for outlet particles (MS Define_freesurface...f90:131)
    if ((ta == SPH_TYPE_WATER || (MS && ta == -202)) && P.renorm) {
        double a1 = (double)b00, bb1 = (double)b01, a2 = (double)b10, bb2 = (double)b11;
        double det = (a1 * bb2 - bb1 * a2);
        if (det != 0) { i00 = bb2 / det; i01 = -bb1 / det; i10 = -a2 / det; i11 = a1 / det; }
    }
    const R m00 = (R)i00, m01 = (R)i01, m10 = (R)i10, m11 = (R)i11;
    D.binv[a] = mk4<R>(m00, m01, m10, m11);
    D.binv64[a] = make_double4(i00, i01, i10, i11);
    R gr[8];
    for (int f = 0; f < 4; ++f) {
        R x = g[2 * f], y = g[2 * f + 1];
        gr[2 * f] = m00 * x + m01 * y;
        gr[2 * f + 1] = m10 * x + m11 * y;
    }
    // SPS stress for water particles (:256-296)
    R txx = R(0), txy = R(0), tyy = R(0);
    if (ta == SPH_TYPE_WATER && !MS) {
        const double sxx = (double)gr[4], sxy = (double)gr[5] + (double)gr[6], syy = (double)gr[7];
        const double abs2 = 2 * (sxx * sxx + syy * syy) + sxy * sxy;
        const double DL = P.sps_dl;               // SPS_Delta_L = sqrt(2.0)/2.0*interior_dx (host-side product)
        const double t = P.sps_c012 * DL;
        const double nut = (t * t) * sqrt(abs2);
        const double kk = P.sps_23 * nut * (sxx + syy);
        const double blin = P.sps_blin * (DL * DL) * abs2;
        const double rho = (double)rho_a;
        txx = (R)((2 * nut * sxx - kk - blin) * rho);
        txy = (R)((nut * sxy) * rho);
        tyy = (R)((2 * nut * syy - kk - blin) * rho);
    }
    // FP32 records: the gradients halved (exact), since pass C uses only
    // 1/2 grad phi, and w = 1/rho (rounded FP32 reciprocal of the FP32 density),
    // which pass C reads instead of forming it for every pair
    if (F32)
        for (int c = 0; c < 8; ++c) gr[c] *= R(0.5);
    D.nb1[a] = mk4<R>(txx, txy, tyy, gr[0]);
    D.nb2[a] = mk4<R>(gr[1], gr[2], gr[3], gr[4]);
    D.nb3[a] = mk4<R>(gr[5], gr[6], gr[7], F32 ? (R)__frcp_rn((float)rho_a) : R(0));
    const R fv = fra;
    D.fra_v[a] = fv;
    uint8_t fl = 0;
    if (P.free_surface && ta == SPH_TYPE_WATER && (double)fv <= P.fs_thr) fl = 4;   // surface candidate (:123)
    D.flags[a] = fl;
    if (MS) D.avg[a] = mk2<R>(xs0, xs1);
}

template <typename R, bool HLREC>
void launch_pass_a(const Params& P, const Sorted<R>& D, int nb, cudaStream_t st) {
    if (P.ms) k_pass_a<R, HLREC, true><<<nb, 128, 0, st>>>(P, D);
    else k_pass_a<R, HLREC, false><<<nb, 128, 0, st>>>(P, D);
}

// Geometric free-surface test of the candidates (Define_freesurface...f90:295-376):
// normal n = -B^-1 sum(grad W V)/|.|; the candidate is interior as soon as one
// water neighbour j satisfies  |x_j-x_i| >= 1.414h and |x_j - (x_i + h n)| < h,
// or |x_j-x_i| < 1.414h and acos(n.(x_j-x_i)/|x_j-x_i|) <= pi/4.
// Both criteria only accept j within 2h <= support, so the list covers them.
template <typename R>
// Grid-stride over the particles: candidates are rare, so most threads only
// read a flag byte, and a grid of 148 x 8 blocks does that with little block
// scheduling.
__global__ void k_surface(Params P, Sorted<R> D) {
    using V4 = typename VT<R>::V4;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < P.n_tot; a += gridDim.x * blockDim.x) {
    uint8_t fl = D.flags[a];
    if (!(fl & 4)) continue;
    const int nn = D.npairs[a];
    const double2 xa = D.pos[a];
    // sum_dwdx (:155-156) recomputed here (candidates are rare)
    double s0 = 0.0, s1 = 0.0;
    for (int e = 0; e < nn; ++e) {
        const int b = (int)(D.pairs[(size_t)e * P.nbr_stride + a] & 0x7fffffffu);
        const double2 xb = D.pos[b];
        double dx = xa.x - xb.x, dy = xa.y - xb.y, d;
        if (!in_support(P, dx, dy, d)) continue;
        double w, gx, gy;
        kernel_w_dw<double>(P, d, dx, dy, w, gx, gy);
        const double Vb = (double)D.aux[b].y;
        s0 += gx * Vb; s1 += gy * Vb;
    }
    const V4 bi = D.binv[a];
    double n0 = (double)bi.x * s0 + (double)bi.y * s1;
    double n1 = (double)bi.z * s0 + (double)bi.w * s1;
    double len = sqrt(n0 * n0 + n1 * n1);
    bool surface = true;
    if (isnan(len) || len == 0.0) surface = false;
    else {
        n0 = -n0 / len; n1 = -n1 / len;
        const double h = P.h;
        const double vx = xa.x + h * n0, vy = xa.y + h * n1;
        for (int e = 0; e < nn && surface; ++e) {
            const int b = (int)(D.pairs[(size_t)e * P.nbr_stride + a] & 0x7fffffffu);
            if (D.type[b] != SPH_TYPE_WATER) continue;
            const double2 xb = D.pos[b];
            double p0 = xb.x - xa.x, p1 = xb.y - xa.y;
            double ji = sqrt(p0 * p0 + p1 * p1);
            double nd = n0 * p0 + n1 * p1;
            double q0 = xb.x - vx, q1 = xb.y - vy;
            double jt = sqrt(q0 * q0 + q1 * q1);
            if (ji >= P.c1414 * h && jt < h) surface = false;
            else if (ji < P.c1414 * h && acos(nd / ji) <= (P.pi / 4.0)) surface = false;
        }
    }
    D.flags[a] = surface ? (uint8_t)(fl | 1) : (uint8_t)(fl & ~1);
    }
}

// Near-free-surface flags (Define_freesurface...f90:418-440): every pair
// neighbour of a surface particle.  Idempotent byte stores, no atomics needed.
template <typename R>
__global__ void k_near(Params P, Sorted<R> D) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < P.n_tot; a += gridDim.x * blockDim.x) {
        if (!(D.flags[a] & 1)) continue;
        const int nn = D.npairs[a];
        for (int e = 0; e < nn; ++e) {
            const int b = (int)(D.pairs[(size_t)e * P.nbr_stride + a] & 0x7fffffffu);
            D.flags[b] |= 2;
        }
    }
}

// The free-surface test and the near-surface flags of one RHS.
template <typename R>
void launch_surface(const Params& P, const Sorted<R>& D, cudaStream_t st) {
    // without free-surface detection pass A marks no candidate, so both kernels
    // would only read flags
    if (!P.free_surface) return;
    int nb = (P.n_tot + 127) / 128;
    if (nb > 148 * 8) nb = 148 * 8;
    if (nb == 0) return;
    k_surface<R><<<nb, 128, 0, st>>>(P, D);
    k_near<R><<<nb, 128, 0, st>>>(P, D);
}

}  // namespace sph
