// pass_c_tile.cuh -- pass C of the Taylor-Green MUSCL linear-Riemann solver
// (Solver_Normalized_MUSCL_Linear_Riemann_Delta_SPS.f90:458-721, with the
// delta-SPH term of :690-721 and the assembly of single_step_compute.f90:152-171)
// in which every pair whose two particles lie in the same block is evaluated
// once.
//
// A block is a tile of kTileThreads consecutive cell-sorted slots (a patch
// two cell rows high, see cell_key).  Each of a particle's pairs is one of:
//   owned    both particles in the tile, this particle the pair's owner: it
//            evaluates the pair once, forms both members' terms, keeps its own
//            and leaves the partner's in shared memory;
//   received both in the tile, the partner owns the pair: the particle adds
//            the partner's stored terms after the block barrier;
//   cross    the partner lies outside the tile: the particle forms its own
//            terms only (the partner's block forms the other side), as the
//            gather pass k_pass_c does for every pair.
// The owner of an in-tile pair (a, b) is min(a, b) when a + b is odd and
// max(a, b) when it is even, which splits each particle's in-tile pairs about
// evenly.  Threads take their particles in order of decreasing work (owned
// plus cross pairs; a counting sort per block), so that the lanes of a warp
// run loops of similar length: tile-edge particles have many cross pairs,
// interior ones many owned pairs.
//
// Every pair is still evaluated in the reference's orientation (pair_i = the
// lower id), so both members see the flux of the same operations.  Each
// particle's sums run in a fixed order -- its owned and cross pairs in list
// order, then its received pairs in list order -- so the results are
// deterministic.  A block in which a particle has more than kTileCap pairs or
// more than kOwnCap owned pairs runs the gather pass instead (a block-uniform
// decision, so the two members of every pair agree on who forms what).
#pragma once
#include "pass_c.cuh"

namespace sph {

constexpr int kTileThreads = 128;   // slots per tile = threads per block
constexpr int kTileCap = 32;        // pair entries per particle held in shared memory
constexpr int kOwnCap = 16;         // owned pairs per particle held in shared memory

template <typename R>
struct TileShared {
    unsigned work[kTileCap][kTileThreads];   // owned entries from row 0 up, cross entries from the last row down
    R cdr[kOwnCap][kTileThreads];            // the partner's terms of owned pair k of local particle p
    R ctx[kOwnCap][kTileThreads];
    R cty[kOwnCap][kTileThreads];
    uint8_t skip[kTileCap][kTileThreads];    // local index of the owner of each received pair, in list order
    uint8_t no[kTileThreads], nc[kTileThreads], ns[kTileThreads], perm[kTileThreads];
    int hist[kTileCap + 1];
};

template <typename R>
__global__ void __launch_bounds__(kTileThreads, sizeof(R) == 4 ? 4 : 3) k_pass_c_tile(Params P, Sorted<R> D) {
    using V4 = typename VT<R>::V4;
    using A = typename Acc<R>::T;
    constexpr bool F32 = sizeof(R) == 4;
    extern __shared__ __align__(16) unsigned char tile_smem[];
    TileShared<R>& T = *reinterpret_cast<TileShared<R>*>(tile_smem);
    const int tid = threadIdx.x;
    const int t0 = blockIdx.x * kTileThreads;

    // ---- the pairs of particle t0 + tid, sorted into owned / cross / received
    {
        const int a = t0 + tid;
        const int nn = a < P.n_tot ? D.npairs[a] : 0;
        int no = 0, nc = 0, ns = 0;
        bool ovf = nn > kTileCap;
        if (!ovf) {
            for (int e = 0; e < nn; ++e) {
                const unsigned ent = __ldg(&D.pairs[(size_t)e * P.nbr_stride + a]);
                const int b = (int)(ent & 0x7fffffffu);
                const unsigned lb = (unsigned)(b - t0);
                if (lb < (unsigned)kTileThreads) {
                    if (((a ^ b) & 1) ? (a < b) : (a > b)) T.work[no++][tid] = ent;
                    else T.skip[ns++][tid] = (uint8_t)lb;
                } else {
                    T.work[kTileCap - 1 - nc++][tid] = ent;
                }
            }
            ovf = no > kOwnCap;
        }
        if (__syncthreads_or(ovf)) {
            if (a < P.n_tot) pass_c_gather<R, true, false, false>(P, D, a);
            return;
        }
        T.no[tid] = (uint8_t)no;
        T.nc[tid] = (uint8_t)nc;
        T.ns[tid] = (uint8_t)ns;
        if (tid <= kTileCap) T.hist[tid] = 0;
        __syncthreads();
        // counting sort by work, most work first: bucket kTileCap - (no + nc)
        const int bucket = kTileCap - (no + nc);
        atomicAdd(&T.hist[bucket], 1);
        __syncthreads();
        if (tid < 32) {
            const int v = T.hist[tid];
            int incl = v;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (tid >= o) incl += y;
            }
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            T.hist[tid] = incl - v;
            if (tid == 0) T.hist[kTileCap] = total;    // the last bucket starts after buckets 0..31
        }
        __syncthreads();
        T.perm[atomicAdd(&T.hist[bucket], 1)] = (uint8_t)tid;
        __syncthreads();
    }

    // ---- owned and cross pairs of particle a = t0 + p -------------------------
    const int p = T.perm[tid];
    const int a = t0 + p;
    const bool live = a < P.n_tot;
    const int no = T.no[p], nwork = no + T.nc[p];

    Side<R> S;
    double2 xa = make_double2(0.0, 0.0);
    float4 xa_hl = make_float4(0.f, 0.f, 0.f, 0.f);
    V4 bi = mk4<R>(R(0), R(0), R(0), R(0));
    bool near_a = false, water_a = false;
    auto load_side = [&](int bb, Side<R>& t) {
        if (F32) { t.kh = D.kh[bb]; t.kl = D.kl[bb]; }
        else t.kin = D.kin[bb];
        t.aux = D.aux[bb]; t.nb1 = D.nb1[bb]; t.nb2 = D.nb2[bb]; t.nb3 = D.nb3[bb];
    };
    if (live) {
        load_side(a, S);
        if (F32) xa_hl = D.xhl[a];
        else xa = D.pos[a];
        bi = D.binv[a];
        const uint8_t fa = D.flags[a];
        near_a = (fa & 2) != 0;
        water_a = (fa & 8) != 0;
    }
    const R rho_a = F32 ? (R)S.kh.z : (R)S.kin.z;
    const R hbar = (R)P.h;
    const R inv_h = (R)(1.0 / P.h);
    const R inv_sqc0 = (R)(1.0 / P.sqrt_c0);
    const R nu2 = (R)(2.0 * P.nu), alpha = (R)P.alpha, beta = (R)P.beta;
    const R fh2 = (R)((P.fai * P.h) * (P.fai * P.h));
    const R dlt2h = (R)(2.0 * P.delta * P.h);
    const R dla_h = (R)(P.delta_alpha * P.h);
    const R rho0 = (R)P.rho0;
    const R inv_rho_a = live ? rcp(rho_a) : R(0);
    const R rho0_over_rho_a = rho0 * inv_rho_a;

    A cont, accx, accy;
    cont.init(); accx.init(); accy.init();

    auto entry = [&](int k) { return T.work[k < no ? k : kTileCap - 1 - (k - no)][p]; };
    // the neighbour's records one iteration ahead (and, for an owned pair, its
    // B^-1 and flags, which its terms need)
    Side<R> Nn;
    double2 xb_n = make_double2(0.0, 0.0);
    float4 xbhl_n = make_float4(0.f, 0.f, 0.f, 0.f);
    V4 bib_n = mk4<R>(R(0), R(0), R(0), R(0));
    uint8_t flb_n = 0;
    auto fetch = [&](int k) {
        const int b = (int)(entry(k) & 0x7fffffffu);
        if (F32) xbhl_n = __ldg(&D.xhl[b]);
        else xb_n = __ldg(&D.pos[b]);
        load_side(b, Nn);
        if (k < no) { bib_n = D.binv[b]; flb_n = D.flags[b]; }
    };
    if (nwork > 0) fetch(0);
    for (int k = 0; k < nwork; ++k) {
        const unsigned ent = entry(k);
        const bool a_is_i = (ent >> 31) != 0;
        const bool own = k < no;
        const Side<R> N = Nn;
        const double2 xb = xb_n;
        const float4 xbhl = xbhl_n;
        const V4 bib = bib_n;
        const uint8_t flb = flb_n;
        if (k + 1 < nwork) fetch(k + 1);
        // x_a - x_b: hi/lo in FP32 (the rounding of the FP64 difference), or FP64
        double dxd = 0.0, dyd = 0.0;
        float dxf = 0.f, dyf = 0.f;
        R d, inv_d;
        if (F32) {
            dxf = (xa_hl.x - xbhl.x) + (xa_hl.z - xbhl.z);
            dyf = (xa_hl.y - xbhl.y) + (xa_hl.w - xbhl.w);
            const R s = (R)(dxf * dxf + dyf * dyf);
            inv_d = rsqrtf(s);
            d = s * inv_d;
        } else {
            dxd = xa.x - xb.x;
            dyd = xa.y - xb.y;
            d = (R)sqrt(dxd * dxd + dyd * dyd);
            inv_d = R(1) / d;
        }
        const Side<R>& I = a_is_i ? S : N;
        const Side<R>& J = a_is_i ? N : S;
        // position_difference_ij = x_i - x_j (find_particle_pair.f90:79-107)
        R xij0, xij1;
        if (F32) { xij0 = (R)(a_is_i ? dxf : -dxf); xij1 = (R)(a_is_i ? dyf : -dyf); }
        else { xij0 = (R)(a_is_i ? dxd : -dxd); xij1 = (R)(a_is_i ? dyd : -dyd); }
        R du, dv, dp, drho_ji, rho_i, rho_j, rho_b;
        if (F32) {
            du = (R)((I.kh.x - J.kh.x) + (I.kl.x - J.kl.x));
            dv = (R)((I.kh.y - J.kh.y) + (I.kl.y - J.kl.y));
            dp = (R)((I.kh.w - J.kh.w) + (I.kl.w - J.kl.w));
            drho_ji = (R)((J.kh.z - I.kh.z) + (J.kl.z - I.kl.z));
            rho_i = (R)I.kh.z; rho_j = (R)J.kh.z; rho_b = (R)N.kh.z;
        } else {
            du = (R)(I.kin.x - J.kin.x); dv = (R)(I.kin.y - J.kin.y);
            dp = (R)(I.kin.w - J.kin.w);
            drho_ji = (R)(J.kin.z - I.kin.z);
            rho_i = (R)I.kin.z; rho_j = (R)J.kin.z; rho_b = (R)N.kin.z;
        }
        // compute_kernel: dwdx(k) = g (x_i - x_j)
        R g;
        {
            const R q = d * inv_h;
            const R kf = (R)P.kfactor;
            if (P.kernel_model == SPH_KERNEL_GAUSSIAN) {
                const R ex = exp(-(q * q));
                g = ex * (R(-2) * q) * inv_d * inv_h * kf;
            } else {
                const R t = R(1) - R(0.5) * q;
                const R t3 = t * t * t;
                g = kf * (R(-5) * q * t3) * inv_d * inv_h;
            }
        }
        const R dw0 = g * xij0, dw1 = g * xij1;
        const R cbar = R(0.5) * (I.aux.z + J.aux.z);
        const R rbar = R(0.5) * (rho_i + rho_j);
        const R inv_rbar = rcp(rbar);
        const R e0 = -xij0 * inv_d, e1 = -xij1 * inv_d;
        // MUSCL reconstruction increments (:470-502, function_module.f90:34-80)
        R lpi, lpj, lui, luj, lvi, lvj;
        {
            const R x0 = -xij0, x1 = -xij1;          // j - i
            muscl_limiter<R>(R(0.5) * (I.nb2.y * x0 + I.nb2.z * x1), R(-0.5) * (J.nb2.y * x0 + J.nb2.z * x1), -dp,
                             lpi, lpj);
            muscl_limiter<R>(R(0.5) * (I.nb2.w * x0 + I.nb3.x * x1), R(-0.5) * (J.nb2.w * x0 + J.nb3.x * x1), -du,
                             lui, luj);
            muscl_limiter<R>(R(0.5) * (I.nb3.y * x0 + I.nb3.z * x1), R(-0.5) * (J.nb3.y * x0 + J.nb3.z * x1), -dv,
                             lvi, lvj);
        }
        // linear Riemann state (:503-520): U_L - U_R, P*, U* - Ubar
        const R dU = (du + lui + luj) * e0 + (dv + lvi + lvj) * e1;
        const R Pbar = F32 ? R(0.5) * ((R)I.kh.w + (R)J.kh.w) : R(0.5) * ((R)I.kin.w + (R)J.kin.w);
        const R dP = dp + lpi + lpj;
        const R sU = R(0.5) * dP * (inv_rbar * inv_sqc0);
        const R bR = min(R(3) * (max(dU, R(0))), cbar);
        const R Ps = Pbar + R(0.5) * bR * rbar * dU;
        // reconstructed velocity minus the pair mean, of the i and j members
        const R wi0 = R(0.5) * du + lui, wi1 = R(0.5) * dv + lvi;
        const R wj0 = R(-0.5) * du - luj, wj1 = R(-0.5) * dv - lvj;
        const R inv_r2 = inv_d * inv_d;
        const R vx = du * xij0 + dv * xij1;
        const R rcp_b = rcp(rho_b);
        const R rho_ij = inv_rho_a * rcp_b;
        // artificial viscosity coefficient (:392-417), 0 unless the pair approaches
        R Pi = R(0);
        if (vx < R(0)) {
            const R phi1 = hbar * vx / (d * d + fh2);
            Pi = (-alpha * cbar * phi1 + beta * (phi1 * phi1)) * inv_rbar;
        }
        // SPS (:450-492, unnormalised dwdx; temp_p carried from x to y with quirks)
        const R sxx = I.nb1.x + J.nb1.x, sxy = I.nb1.y + J.nb1.y, syy = I.nb1.z + J.nb1.z;
        const R tp = (sxx * dw0 + sxy * dw1) * rho_ij;
        const R tp2 = ((P.quirks ? tp : R(0)) + syy * dw1 + sxy * dw0) * rho_ij;
        // delta-alpha (:442-446) and delta-SPH (:690-721) factors common to both members
        const R cav = dla_h * cbar * vx * inv_r2;
        const R sg0 = I.nb1.w + J.nb1.w, sg1 = I.nb2.x + J.nb2.x;
        const R dps = dlt2h * cbar * (drho_ji + R(0.5) * (sg0 * xij0 + sg1 * xij1));
        // The terms of pair member X (the other member Y): continuity, pressure
        // force, artificial viscosity, Morris laplacian, delta-alpha, SPS and
        // delta-SPH, with X's normalised gradient B_X^-1 dwdx and star state.
        auto side = [&](const V4& bX, bool nearX, bool waterX, bool X_is_i, R rhoX, R rho0_over_rhoX, R VY, R mY,
                        R smY, R& dr, R& tx, R& ty) {
            const R nd0 = bX.x * dw0 + bX.y * dw1;
            const R nd1 = bX.z * dw0 + bX.w * dw1;
            R w0 = X_is_i ? wi0 : wj0, w1 = X_is_i ? wi1 : wj1;
            if (!nearX) { w0 -= sU * e0; w1 -= sU * e1; }
            const R PX = nearX ? Pbar : Ps;
            const R sg = X_is_i ? R(1) : R(-1);
            dr = R(2) * rhoX * VY * (sg * (w0 * nd0 + w1 * nd1));
            const R fp = R(-2) * PX * rho_ij * mY;
            R x = fp * nd0, y = fp * nd1;
            x += mY * (-Pi * nd0);
            y += mY * (-Pi * nd1);
            const R rnd = xij0 * nd0 + xij1 * nd1;
            const R lf = VY * nu2 * rnd * inv_r2;
            x += lf * du;
            y += lf * dv;
            const R tt = cav * rho0_over_rhoX * VY;
            x += tt * nd0;
            y += tt * nd1;
            x += smY * tp;
            y += smY * tp2;
            tx = sg * x;
            ty = sg * y;
            if (waterX) dr += sg * (dps * (-rnd * inv_r2) * VY);
        };
        R dra, txa, tya;
        side(bi, near_a, water_a, a_is_i, rho_a, rho0_over_rho_a, N.aux.y, N.aux.x, N.aux.w, dra, txa, tya);
        cont.add(dra);
        accx.add(txa);
        accy.add(tya);
        if (own) {
            R drb, txb, tyb;
            side(bib, (flb & 2) != 0, (flb & 8) != 0, !a_is_i, rho_b, rho0 * rcp_b, S.aux.y, S.aux.x, S.aux.w, drb,
                 txb, tyb);
            T.cdr[k][p] = drb;
            T.ctx[k][p] = txb;
            T.cty[k][p] = tyb;
        }
    }
    __syncthreads();

    // ---- received pairs: the owners' stored terms, in list order ---------------
    if (!live) return;
    const int ns = T.ns[p];
    for (int s = 0; s < ns; ++s) {
        const int la = T.skip[s][p];
        const int nol = T.no[la];
        int k = 0;
        while (k < nol && (T.work[k][la] & 0x7fffffffu) != (unsigned)a) ++k;
        if (k < nol) {
            cont.add(T.cdr[k][la]);
            accx.add(T.ctx[k][la]);
            accy.add(T.cty[k][la]);
        }
    }
    // assembly (single_step_compute.f90:152-171, Solver :627-635); no XSPH in this solver
    D.drho[a] = cont.val();
    D.acc[a] = water_a ? mk2<R>(accx.val(), accy.val()) : mk2<R>(R(0), R(0));
    D.avg[a] = mk2<R>(R(0), R(0));
}

// Dynamic shared memory of one k_pass_c_tile block.
template <typename R>
constexpr size_t pass_c_tile_smem() {
    return sizeof(TileShared<R>);
}

}  // namespace sph
