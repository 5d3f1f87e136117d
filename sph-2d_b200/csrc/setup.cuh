// setup.cuh -- per-step set-up kernels: periodic wrap and images, the
// background-cell sort, cell ranges and the per-particle neighbour lists.
#pragma once
#include "common.cuh"

namespace sph {

// Particle arrays in id order ("staging"): the host particles 0..n_host-1
// followed by the periodic images of this step, numbered as the reference
// appends them (Distribute_Period_Boundary_Particle.f90:95-206).
struct Staging {
    double2* pos;     // x, y
    double2* vel;     // u, v
    double* rho;
    double* mass;
    double* smass;    // mass the SPS force multiplies with (quirk A.6), default = mass
    int* type;
    int* itype;       // initial type (body force), images get SPH_TYPE_PERIODIC
    int* blabel;      // wall label of the ghost assignment (host particles)
    // rates of the last RHS of the previous step (the reused K1), host particles only
    double* r_drho;
    double2* r_acc;
    double2* r_avg;
    int* cnt;         // scratch pair that sizes the image scan's temporary storage
    int* off;
    // image counts and offsets of this step, kept for routing image adjoints:
    // left/right images of host i sit at n_host + lr_off[i] + k (k < lr_cnt[i]),
    // bottom/top images of source s at n_host + n_lr + tb_off[s] + k (k < tb_cnt[s])
    int* lr_cnt;
    int* lr_off;
    int* tb_cnt;
    int* tb_off;
};

// --- 1. periodic wrap (Distribute_Period_Boundary_Particle.f90:56-90), done by
// the first image count below: a host particle outside the box re-enters on the
// opposite side before its images are counted.
__device__ __forceinline__ double2 wrap_position(const Params& P, double2 x) {
    const double Lx = P.box_hi[0] - P.box_lo[0], Ly = P.box_hi[1] - P.box_lo[1];
    if (x.x > P.box_hi[0]) x.x = x.x - Lx;
    else if (x.x < P.box_lo[0]) x.x = x.x + Lx;
    if (x.y > P.box_hi[1]) x.y = x.y - Ly;
    else if (x.y < P.box_lo[1]) x.y = x.y + Ly;
    return x;
}

// --- 2. images: count per source, then emit at scanned offsets -------------
// axis 0: left/right images of the host particles (:98-148),
// axis 1: bottom/top images of host particles and left/right images (:156-206).
// cnt: the routing counts of this axis (lr_cnt / tb_cnt), scanned in place into
// the routing offsets (lr_off / tb_off) that k_img_emit reads
// axis 0 (sources = the host particles) wraps the positions first.
__global__ void k_img_count(Params P, Staging S, int n_src, int axis, int* cnt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_src) return;
    int c = 0;
    if (S.type[i] != SPH_TYPE_ILL) {
        double2 xy = S.pos[i];
        if (axis == 0) {
            const double2 w = wrap_position(P, xy);
            if (w.x != xy.x || w.y != xy.y) S.pos[i] = w;
            xy = w;
        }
        double x = axis == 0 ? xy.x : xy.y;
        double lo = P.box_lo[axis], hi = P.box_hi[axis];
        if (x <= (lo + P.band) && x >= lo) c++;
        if (x >= (hi - P.band) && x <= hi) c++;
    }
    cnt[i] = c;
}

__global__ void k_img_emit(Params P, Staging S, int n_src, int axis, int base, const int* off) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_src || S.type[i] == SPH_TYPE_ILL) return;
    double2 x = S.pos[i];
    double v = axis == 0 ? x.x : x.y;
    double lo = P.box_lo[axis], hi = P.box_hi[axis], L = hi - lo;
    int o = base + off[i];
    for (int side = 0; side < 2; ++side) {
        bool in = side == 0 ? (v <= (lo + P.band) && v >= lo) : (v >= (hi - P.band) && v <= hi);
        if (!in) continue;
        double2 y = x;
        double sh = side == 0 ? L : -L;
        if (axis == 0) y.x = x.x + sh; else y.y = x.y + sh;
        S.pos[o] = y;
        S.vel[o] = S.vel[i];
        S.rho[o] = S.rho[i];
        S.mass[o] = S.mass[i];
        S.smass[o] = S.smass[i];
        S.type[o] = SPH_TYPE_PERIODIC;
        S.itype[o] = SPH_TYPE_PERIODIC;
        ++o;
    }
}

// --- 3. cell keys (row-major cells of edge >= list radius) -----------------
__global__ void k_cell_keys(Params P, const double2* pos, const int* type, unsigned* keys, unsigned* vals,
                            unsigned* status, unsigned dead_key) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n_tot) return;
    vals[i] = (unsigned)i;
    int t = type[i];
    if (t == SPH_TYPE_ILL || t == 0) { keys[i] = dead_key; return; }   // not binned (Assign_boundary_particles.f90:82)
    double2 x = pos[i];
    double fx = floor((x.x - P.gx0) / P.cs), fy = floor((x.y - P.gy0) / P.cs);
    int cx = (int)fx, cy = (int)fy;
    if (!(fx >= 0.0 && fy >= 0.0 && cx < P.gnx && cy < P.gny)) {
        atomicOr(status, ST_DOMAIN);
        keys[i] = dead_key;
        return;
    }
    keys[i] = (unsigned)(cy * P.gnx + cx);
}

// Device-side arrays in cell-sorted order (templated on the pair precision).
template <typename R>
struct Sorted {
    using V2 = typename VT<R>::V2;
    using V4 = typename VT<R>::V4;
    int* id;          // id-order index (host index, or n_host + image number)
    int* slot_of;     // inverse: the sorted slot of id i
    uint8_t* nflag;   // reverse sweep: bit 0 near a ghost (within its interpolation radius),
                      // bit 1 a pair neighbour of a body particle
    int* type;
    int* itype;       // initial type (SPH_TYPE_BODY marks the body)
    int* blabel;      // wall label of the ghost assignment (0 for images)
    double2* pos;     // current stage position (FP64)
    double2* pos0;    // step-start (master) position, also the list-build position
    double2* vel0;    // step-start velocity (FP64 master)
    double* rho0;     // step-start density (FP64 master)
    double* mass;
    double* smass;
    double4* kin;     // u, v, rho, p (FP64 in both paths: pair differences are  -- neighbour record 1
                      // formed from it in FP64 before the FP32 arithmetic)
    V4* aux;          // m, V = m/rho, c, smass                      -- neighbour record 2
    V4* nb1;          // tau_xx, tau_xy, tau_yy, grad rho x          -- neighbour record 3
    V4* nb2;          // grad rho y, grad p x, grad p y, grad u x     -- neighbour record 4
    V4* nb3;          // grad u y, grad v x, grad v y, 1/rho (FP32) or 0 -- neighbour record 5 (MUSCL)
                      // (the FP32 records hold the gradients halved: grad_scale<R>())
    V4* binv;         // B^-1 (11, 12, 21, 22) in the pair precision
    double4* binv64;  // B^-1 in FP64 (applied to the FP64 shifting sum)
    R* fra_v;
    uint8_t* flags;   // bit0 surface, bit1 near surface, bit2 surface candidate
    // rates of the current RHS
    R* drho;
    V2* acc;
    V2* avg;
    double2* shift;   // shifting displacement (last RHS of a step), FP64
    // Runge-Kutta sums K1 + 2 K2 + 2 K3 (time_iteration.f90:1040-1045)
    R* ks_r;
    V2* ks_a;
    double2* ks_v;    // velocity sums in FP64 (they move the FP64 positions)
    // rates carried to the next step (K1 reuse)
    R* c_drho;
    V2* c_acc;
    V2* c_avg;
    // neighbour lists: slot-major [max_nbr][stride], bit 31 = "this particle has the lower id"
    unsigned* nbr;
    int* nnbr;
    // the pairs of the current RHS (list entries inside the support), same layout,
    // written by pass A and read by the passes that follow it
    unsigned* pairs;
    int* npairs;
    // cell ranges
    int* cell_start;
    int* cell_end;
    // mixed path only: the kinematic record and the position split into float
    // hi + lo parts (v = hi + lo, hi = (float)v), so pass C forms pair
    // differences (hi_i - hi_j) + (lo_i - lo_j) in FP32 with the accuracy of the
    // FP64 difference rounded to FP32, without FP64 arithmetic or conversions
    double* vol64;    // m / rho in FP64 (the mixed path's FP64 shifting sum)
    float4* kh;       // u, v, rho, p  (hi)
    float4* kl;       //               (lo)
    float4* xhl;      // x hi, y hi, x lo, y lo
};

// Factor from the stored gradient records (nb1.w, nb2, nb3.xyz) to the
// gradients: the FP32 records hold 1/2 grad phi (pass C uses only that).
template <typename R>
__host__ __device__ constexpr double grad_scale() { return sizeof(R) == 4 ? 2.0 : 1.0; }

// Hi/lo split of the records a particle's pass-C neighbours read (mixed path).
template <typename R>
__device__ __forceinline__ void store_split(Sorted<R>& D, int s, double2 x, double4 k) {
    if (sizeof(R) != 4) return;
    D.vol64[s] = D.mass[s] / k.z;
    const float uh = (float)k.x, vh = (float)k.y, rh = (float)k.z, ph = (float)k.w;
    D.kh[s] = make_float4(uh, vh, rh, ph);
    D.kl[s] = make_float4((float)(k.x - (double)uh), (float)(k.y - (double)vh), (float)(k.z - (double)rh),
                          (float)(k.w - (double)ph));
    const float xh = (float)x.x, yh = (float)x.y;
    D.xhl[s] = make_float4(xh, yh, (float)(x.x - (double)xh), (float)(x.y - (double)yh));
}

// --- 4. gather the id-ordered arrays into cell order -----------------------
template <typename R>
__global__ void k_gather_sorted(Params P, Staging S, Sorted<R> D, const unsigned* perm) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.n_tot) return;
    int i = (int)perm[s];
    D.id[s] = i;
    D.slot_of[i] = s;
    D.type[s] = S.type[i];
    D.itype[s] = S.itype[i];
    D.blabel[s] = i < P.n_host ? S.blabel[i] : 0;
    double2 x = S.pos[i];
    D.pos[s] = x;
    D.pos0[s] = x;
    const double2 v = S.vel[i];
    const double rho = S.rho[i], m = S.mass[i], sm = S.smass[i];
    D.vel0[s] = v;
    D.rho0[s] = rho;
    D.mass[s] = m;
    D.smass[s] = sm;
    // neighbour records of the step-start state (formed here from the values
    // just gathered, instead of a second pass over the sorted arrays)
    double p, c;
    eos64(P, rho, p, c);
    D.kin[s] = make_double4(v.x, v.y, rho, p);
    D.aux[s] = mk4<R>((R)m, (R)(m / rho), (R)c, (R)sm);
    store_split(D, s, x, make_double4(v.x, v.y, rho, p));
    if (i < P.n_host) {
        D.c_drho[s] = (R)S.r_drho[i];
        D.c_acc[s] = mk2<R>((R)S.r_acc[i].x, (R)S.r_acc[i].y);
        D.c_avg[s] = mk2<R>((R)S.r_avg[i].x, (R)S.r_avg[i].y);
    } else {
        D.c_drho[s] = R(0);
        D.c_acc[s] = mk2<R>(R(0), R(0));
        D.c_avg[s] = mk2<R>(R(0), R(0));
    }
}

// sorted master state -> id order (host particles only; images are dropped)
template <typename R>
__global__ void k_unsort(Params P, Staging S, Sorted<R> D) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.n_tot) return;
    int i = D.id[s];
    if (i >= P.n_host) return;
    S.pos[i] = D.pos0[s];
    S.vel[i] = D.vel0[s];
    S.rho[i] = D.rho0[s];
    S.mass[i] = D.mass[s];
    S.smass[i] = D.smass[s];
    S.type[i] = D.type[s];
    S.itype[i] = D.itype[s];
    S.r_drho[i] = (double)D.c_drho[s];
    S.r_acc[i] = make_double2((double)D.c_acc[s].x, (double)D.c_acc[s].y);
    S.r_avg[i] = make_double2((double)D.c_avg[s].x, (double)D.c_avg[s].y);
}

// --- 5. cell ranges from the sorted keys ----------------------------------
__global__ void k_cell_ranges(int n, const unsigned* keys, int* start, int* end, unsigned dead_key) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    unsigned k = keys[s];
    if (k == dead_key) return;
    if (s == 0 || keys[s - 1] != k) start[k] = s;
    if (s == n - 1 || keys[s + 1] != k) end[k] = s + 1;
}

// Pair-rule of find_particle_pair (TGV :76, MS :73-75).
__device__ __forceinline__ bool pair_allowed(int rule, int ti, int tj) {
    if (rule == SPH_PAIRS_ONE_FLUID) return ti == SPH_TYPE_WATER || tj == SPH_TYPE_WATER;
    if (ti == -2 && tj == -2) return false;
    if (ti == -3 && tj == -3) return false;
    if (ti == -201 && tj == -201) return false;
    return true;
}

// --- 6. neighbour lists ----------------------------------------------------
// Every particle b != a in the 3x3 cells with |x_a - x_b|^2 <= (support*(1+skin))^2
// and an allowed type pair.  The exact support test is repeated at every RHS on
// the current positions, so the list only has to be a superset of the pairs of
// the whole step; k_stage checks the displacement bound that guarantees it.
// The first kListStage entries of each list are staged in shared memory
// ([entry][thread], conflict-free) and written out row by row after the scan, so
// the stores of a warp are coalesced; longer lists write the rest directly.
constexpr int kListStage = 32;
template <typename R>
__global__ void __launch_bounds__(128) k_build_lists(Params P, Sorted<R> D, unsigned* status) {
    __shared__ unsigned stage[kListStage][128];
    const int tid = threadIdx.x;
    int a = blockIdx.x * blockDim.x + tid;
    if (a >= P.n_tot) return;
    int ta = D.type[a];
    int cnt = 0;
    // one list entry: staged, or (past the stage) straight to global memory
    auto put = [&](int b, unsigned lower) {
        const unsigned v = (unsigned)b | lower;
        if (cnt < kListStage) stage[cnt][tid] = v;
        else if (cnt < P.max_nbr) D.nbr[(size_t)cnt * P.nbr_stride + a] = v;
        ++cnt;
    };
    // the mixed path tests the FP32 hi positions against the widened radius
    // r2_list32 (a superset of the FP64 list, see derive_params)
    constexpr bool F32 = sizeof(R) == 4;
    const float2* xh = reinterpret_cast<const float2*>(D.xhl);     // (x hi, y hi) at 2 s
    if (ta != SPH_TYPE_ILL && ta != 0) {
        double2 xa = D.pos[a];
        const float2 xa_h = F32 ? xh[2 * (size_t)a] : make_float2(0.f, 0.f);
        int ida = D.id[a];
        int cx = (int)floor((xa.x - P.gx0) / P.cs), cy = (int)floor((xa.y - P.gy0) / P.cs);
        int x0 = max(cx - 1, 0), x1 = min(cx + 1, P.gnx - 1);
        // with the one-fluid rule every pair of a water particle is allowed
        const bool check_type = !(P.pair_rule == SPH_PAIRS_ONE_FLUID && ta == SPH_TYPE_WATER);
        for (int gy = max(cy - 1, 0); gy <= min(cy + 1, P.gny - 1); ++gy) {
            // the cells x0..x1 of a row are consecutive keys, so their particles
            // form one contiguous range of the sorted order
            const int row = gy * P.gnx;
            int b0 = -1, b1 = -1;
            for (int gx = x0; gx <= x1; ++gx) {
                const int st = D.cell_start[row + gx];
                if (st < 0) continue;
                if (b0 < 0) b0 = st;
                b1 = D.cell_end[row + gx];
            }
            // candidates four at a time: their loads are issued together, then
            // tested in order (the list is the same as a one-by-one scan)
            int b = b0;
            for (; b + 4 <= b1; b += 4) {
                double2 xb[4];
                float2 xbh[4];
                int tb[4], ib[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (F32) xbh[k] = __ldg(&xh[2 * (size_t)(b + k)]);
                    else xb[k] = __ldg(&D.pos[b + k]);
                    ib[k] = __ldg(&D.id[b + k]);
                    tb[k] = check_type ? __ldg(&D.type[b + k]) : 0;
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (b + k == a) continue;
                    if (check_type && !pair_allowed(P.pair_rule, ta, tb[k])) continue;
                    if (F32) {
                        const float dx = xa_h.x - xbh[k].x, dy = xa_h.y - xbh[k].y;
                        if (dx * dx + dy * dy > P.r2_list32) continue;
                    } else {
                        const double dx = xa.x - xb[k].x, dy = xa.y - xb[k].y;
                        if (dx * dx + dy * dy > P.r2_list) continue;
                    }
                    put(b + k, ida < ib[k] ? 0x80000000u : 0u);
                }
            }
            for (; b < b1; ++b) {
                if (b == a) continue;
                if (check_type && !pair_allowed(P.pair_rule, ta, D.type[b])) continue;
                if (F32) {
                    const float2 xbh = xh[2 * (size_t)b];
                    const float dx = xa_h.x - xbh.x, dy = xa_h.y - xbh.y;
                    if (dx * dx + dy * dy > P.r2_list32) continue;
                } else {
                    const double2 xb = D.pos[b];
                    const double dx = xa.x - xb.x, dy = xa.y - xb.y;
                    if (dx * dx + dy * dy > P.r2_list) continue;
                }
                put(b, ida < D.id[b] ? 0x80000000u : 0u);
            }
        }
        if (cnt > P.max_nbr) { atomicOr(status, ST_NBR_OVERFLOW); cnt = P.max_nbr; }
    }
    const int ns = min(cnt, kListStage);
    for (int e = 0; e < ns; ++e) D.nbr[(size_t)e * P.nbr_stride + a] = stage[e][tid];
    D.nnbr[a] = cnt;
}

}  // namespace sph
