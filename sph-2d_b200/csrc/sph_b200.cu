// sph_b200.cu -- libsph_b200: host orchestration and the C-ABI of
// include/sph_b200.h.  Build: see sph-2d_b200/build_lib.py (nvcc, sm_100a).
//
// One handle = the device-resident particle state of one Fortran subdomain
// (now the whole domain: the MPI decomposition of Devide_block_and_send_tasks
// and the halo exchanges of exchange_buffer_domain_information are gone).
//
// Per time step (time_iteration.f90:781-1073):
//   prepare: periodic wrap + images (id order), cell keys, radix sort,
//            cell ranges, neighbour lists with a skin, neighbour records
//   RHS    : pass A (renormalisation, gradients, SPS) -> surface test ->
//            near-surface flags -> pass C (fused forces)
//   stages : k_stage 0..3, shifting fused into the last stage
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <new>
#include <vector>

#include "adjoint.cuh"

using namespace sph;

namespace {

const char* kMessages[] = {
    "ok", "invalid argument", "capacity exceeded", "non-finite value in the state", "(unused)",
    "CUDA runtime error", "device wait timed out", "unsupported configuration",
    "a particle left the cell grid", "a particle moved further than the neighbour-list skin",
    "no usable CUDA device",
};

#define CK(call)                                                                 \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess) {                                                 \
            fprintf(stderr, "libsph_b200: %s failed: %s (%s:%d)\n", #call,     \
                    cudaGetErrorString(e_), __FILE__, __LINE__);                 \
            return SPH_E_CUDA;                                                   \
        }                                                                        \
    } while (0)

inline int blocks(long long n, int t) { return (int)((n + t - 1) / t); }

enum Phase { PH_SORT, PH_A, PH_SURF, PH_C, PH_UPDATE, PH_IMAGES, PH_ADJ, PH_COUNT };

template <typename T>
cudaError_t dalloc(T** p, size_t count) {
    return cudaMalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T));
}

}  // namespace

// ---------------------------------------------------------------------------
struct sph_handle {
    sph_config cfg;
    Params P;
    int device = 0;
    int cap_host = 0, cap_img = 0, cap_tot = 0;
    int n_host = 0, n_img = 0, n_lr = 0;
    bool staging_valid = false;
    bool sorted_valid = false;
    bool have_rhs = false;
    long long step_count = 0;
    long long last_pairs = 0;
    cudaStream_t stream = nullptr;
    Staging S{};
    Sorted<double> D64{};
    Sorted<float> D32{};
    bool mixed = false;
    // sort
    unsigned *keys_in = nullptr, *keys_out = nullptr, *vals_in = nullptr, *vals_out = nullptr;
    void* cub_tmp = nullptr;
    size_t cub_bytes = 0;
    int key_bits = 0;
    unsigned dead_key = 0;
    int ncells = 0;
    // misc device buffers
    unsigned* d_status = nullptr;
    int* d_int = nullptr;           // small int scratch
    double* d_part = nullptr;       // reduction partials
    double* d_diag = nullptr;
    double* d_xfer = nullptr;       // column-major transfer scratch [cap_host * 6]
    double* d_export = nullptr;     // k_export output (lazy)
    long long* d_off64 = nullptr;   // pair offsets (lazy)
    int* d_cnt_id = nullptr;
    // timing
    bool timing = true;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::vector<int> ev_phase;
    double t_ms[PH_COUNT] = {0};
    double t_total = 0;
    long long n_rhs = 0, n_steps = 0;
    long long launches = 0;
    double bf[6] = {0, 0, 0, 0, 0, 0};   // body force of the last RHS
    double* d_bf = nullptr;               // [6 * blocks(cap_tot) partials + 6]
    bool bf_every_rhs = false;            // sph_rhs also reports it
    bool bf_pending = false;              // the device copy is newer than bf (read on demand)
    struct AdjCtx* adj = nullptr;         // saved context of sph_adjoint_forward
    double* d_mls = nullptr;              // re-initialised densities [cap_tot]
    double t_phys = 0.0;                  // Real_physical_time (ghost assignment)
    double body_vel[2] = {0.0, 0.0};      // Custom_velocity
    double body_acc[2] = {0.0, 0.0};      // Custom_accleration
    // per-step body motion of an adjoint run: step (step_count - sched_step0)
    // takes sched[4k .. 4k+3] (velocity, acceleration) when 0 <= k < sched_n
    const double* sched = nullptr;
    long long sched_step0 = 0;
    int sched_n = 0;
    double* drag_acc = nullptr;           // adjoint forward: += drag_w * F_x at each step's last RHS
    double drag_w = 0.0;
    // fixed-ghost host particles (type SPH_TYPE_FIX_GHOST) in id order, from sph_set_state
    int* d_ghost_ids = nullptr;           // [cap_host]
    int n_ghost = 0;
    // snapshot streaming: the id-order copy is made in the step stream, the
    // device-to-host transfer runs on copy_stream
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t snap_ready = nullptr, snap_done = nullptr;
    double* d_snap = nullptr;             // [6 * cap_host]
    bool snap_pending = false;
};

namespace {

// --- configuration -> kernel parameters (mirrors the oracle's constants) ---
int derive_params(const sph_config& c, Params& P) {
    if (c.kernel_model != SPH_KERNEL_GAUSSIAN && c.kernel_model != SPH_KERNEL_WENDLAND2) return SPH_E_CONFIG;
    if (c.solver < SPH_SOLVER_MODLR_DELTA_SPS || c.solver > SPH_SOLVER_DELTA_SPS) return SPH_E_CONFIG;
    if (c.laplacian != 0 && c.laplacian != 1) return SPH_E_CONFIG;
    if (c.eos != SPH_EOS_TAIT && c.eos != SPH_EOS_LINEAR) return SPH_E_CONFIG;
    if (c.precision != SPH_PREC_FP64 && c.precision != SPH_PREC_MIXED) return SPH_E_CONFIG;
    if (c.integrator != SPH_INTEGRATOR_RK4_REUSE && c.integrator != SPH_INTEGRATOR_EULER_PC) return SPH_E_CONFIG;
    if (!(c.h > 0) || !(c.kernel_scale >= 2.0) || !(c.dx > 0) || !(c.rho0 > 0) || !(c.c0sq > 0)) return SPH_E_CONFIG;
    if (c.cell_skin < 0 || c.cell_skin > 2) return SPH_E_CONFIG;
    if (c.shift_n != 4) return SPH_E_CONFIG;
    if (c.mls_order != 0 && c.mls_order != 1 && c.mls_order != 3 && c.mls_order != 6) return SPH_E_CONFIG;
    if (c.mls_order != 0 && (c.mls_every < 1 || !(c.mls_alpha >= 0))) return SPH_E_CONFIG;
    if (c.ghost_assign != 0 && c.ghost_assign != 1) return SPH_E_CONFIG;
    if (c.ghost_assign && (!(c.ghost_h_factor > 0) || (c.wall_bc != 0 && c.wall_bc != 1))) return SPH_E_CONFIG;
    memset(&P, 0, sizeof(P));
    const bool q = c.reference_literals != 0;
    P.kernel_model = c.kernel_model;
    P.solver = c.solver;
    P.muscl = c.solver == SPH_SOLVER_MUSCL_DELTA_SPS;
    P.dsph = c.solver == SPH_SOLVER_DELTA_SPS ? 1 : 0;
    // XSPH: the modified linear Riemann solvers only (Solver_Normalized_Delta_SPH_SPS.f90:286-322
    // has it commented out)
    P.xsph = (c.xsph_eps != 0.0 && !P.muscl && !P.dsph) ? 1 : 0;
    P.ms = (c.solver == SPH_SOLVER_MS_MODLR_DELTA || c.solver == SPH_SOLVER_MS_HLLC_DELTA) ? 1 : 0;
    P.hllc = c.solver == SPH_SOLVER_MS_HLLC_DELTA ? 1 : 0;
    P.laplacian = c.laplacian;
    P.free_surface = c.free_surface ? 1 : 0;
    P.integrator = c.integrator;
    P.mls_order = c.mls_order;
    P.mls_every = c.mls_order ? c.mls_every : 1;
    P.mls_alpha3 = c.mls_alpha * c.mls_alpha * c.mls_alpha;
    P.has_body = 0;
    P.renorm = c.renormalize ? 1 : 0;
    P.quirks = q ? 1 : 0;
    P.pair_rule = c.pair_rule;
    P.shifting = c.shifting;
    P.eos = c.eos;
    const double pi = 3.14159265358979324;
    const double pi_k = q ? (double)3.14159265358f : pi;
    P.pi = pi;
    P.h = c.h;
    const double hbar = (c.h + c.h) / 2.0;
    P.r_cut = c.kernel_scale * hbar;
    if (q) {
        float e9 = expf(-9.0f);
        P.gauss_e9 = (double)e9;
        double den = (double)(1.0f - 10.0f * e9);
        P.kfactor = c.kernel_model == SPH_KERNEL_GAUSSIAN ? 1.0 / (pi_k * (c.h * c.h) * den) : 7.0 / (4 * pi_k * (c.h * c.h));
        P.cut_min = (double)1.0e-7f;
        P.fs_thr = (double)(float)c.fs_threshold;
        P.c1414 = (double)1.414f;
        P.sps_dl = (double)(sqrtf(2.0f) / 2.0f) * c.dx;
        P.sps_c012 = (double)0.12f;
        P.sps_23 = (double)(2.0f / 3.0f);
        P.sps_blin = (double)((2.0f / 3.0f) * 0.0066f);
        P.q_zero = (double)1.0e-8f;
    } else {
        P.gauss_e9 = exp(-9.0);
        double den = 1.0 - 10.0 * P.gauss_e9;
        P.kfactor = c.kernel_model == SPH_KERNEL_GAUSSIAN ? 1.0 / (pi_k * (c.h * c.h) * den) : 7.0 / (4 * pi_k * (c.h * c.h));
        P.cut_min = 1.0e-7;
        P.fs_thr = c.fs_threshold;
        P.c1414 = 1.414;
        P.sps_dl = sqrt(2.0) / 2.0 * c.dx;
        P.sps_c012 = 0.12;
        P.sps_23 = 2.0 / 3.0;
        P.sps_blin = 2.0 / 3.0 * 0.0066;
        P.q_zero = 1.0e-8;
    }
    P.rho0 = c.rho0; P.c0sq = c.c0sq; P.sqrt_c0 = sqrt(c.c0sq); P.eos_b = c.c0sq * c.rho0 / 7.0; P.pb = c.background_p;
    P.nu = c.nu; P.alpha = c.alpha; P.beta = c.beta; P.fai = c.fai;
    P.delta = c.delta; P.delta_alpha = c.delta_alpha; P.eps = c.xsph_eps;
    const double sr = c.kernel_scale * c.h;
    P.sv = pi * (sr * sr);
    P.shift_beta = c.shift_beta; P.shift_R = c.shift_R; P.shift_max = c.shift_max; P.shift_n = c.shift_n;
    // W(dx) (Shift_particle_position.f90:56-68)
    {
        double qd = c.dx / c.h;
        if (c.kernel_model == SPH_KERNEL_GAUSSIAN) P.w_dx = (exp(-(qd * qd)) - P.gauss_e9) * P.kfactor;
        else { double t = 1 - qd / 2.0; double t2 = t * t; P.w_dx = P.kfactor * (1 + 2 * qd) * (t2 * t2); }
    }
    for (int k = 0; k < 2; ++k) { P.box_lo[k] = c.box_lo[k]; P.box_hi[k] = c.box_hi[k]; }
    P.band = c.kernel_scale * c.h;
    // cell grid: edge = list radius, one spare cell on every side
    const double rl = P.r_cut * (1.0 + c.cell_skin);
    P.r2_list = rl * rl;
    const double skin = P.r_cut * c.cell_skin;
    P.skin_half2 = (0.5 * skin) * (0.5 * skin);
    P.cs = rl;
    P.gx0 = c.grid_lo[0] - rl;
    P.gy0 = c.grid_lo[1] - rl;
    P.gnx = (int)ceil((c.grid_hi[0] - c.grid_lo[0]) / rl) + 3;
    P.gny = (int)ceil((c.grid_hi[1] - c.grid_lo[1]) / rl) + 3;
    // The mixed list build tests |x_a - x_b| on the FP32 hi positions: each is
    // within 2^-24 |x| of the FP64 one and the FP32 difference within 2^-24 of
    // its magnitude, so each computed component is within 2^-22 X of the FP64
    // one (X = the largest coordinate on the grid) and the distance within
    // 2^-21 X; the radius widened by that and the square by (1 + 2^-19) keeps
    // every FP64 list member (the extra candidates fail the exact support tests
    // of the passes that read the list).
    {
        const double X = fmax(fmax(fabs(P.gx0), fabs(P.gx0 + P.gnx * P.cs)),
                              fmax(fabs(P.gy0), fabs(P.gy0 + P.gny * P.cs)));
        const double r32 = rl + X * 0x1p-21;
        P.r2_list32 = (float)(r32 * r32 * (1.0 + 0x1p-19));
    }
    if (!(c.grid_hi[0] > c.grid_lo[0]) || !(c.grid_hi[1] > c.grid_lo[1])) return SPH_E_CONFIG;
    if ((long long)P.gnx * P.gny > (1LL << 30)) return SPH_E_CONFIG;
    // neighbour-list capacity: twice the lattice count inside the list radius
    const double lat = pi * (rl / c.dx) * (rl / c.dx);
    int mn = (int)ceil(2.0 * lat) + 16;
    mn = (mn + 3) & ~3;
    P.max_nbr = std::min(mn, 256);
    // ghost assignment: average_smooth_length = 1.2*smooth_length (a default-real
    // literal under reference_literals), support kernel_scale times that, cells
    // covering it plus the half skin the neighbours may move within a step
    P.ghost_assign = c.ghost_assign;
    P.wall_bc = c.wall_bc;
    P.ghost_h = (q ? (double)(float)c.ghost_h_factor : c.ghost_h_factor) * c.h;
    P.ghost_r = c.kernel_scale * P.ghost_h;
    P.ghost_kf = c.kernel_model == SPH_KERNEL_GAUSSIAN
                     ? 1.0 / (pi_k * (P.ghost_h * P.ghost_h) * (q ? (double)(1.0f - 10.0f * expf(-9.0f))
                                                                  : 1.0 - 10.0 * exp(-9.0)))
                     : 7.0 / (4 * pi_k * (P.ghost_h * P.ghost_h));
    P.ghost_cells = c.ghost_assign ? (int)ceil((P.ghost_r + 0.5 * skin) / P.cs) : 1;
    P.shock_t = c.shock_release_time;
    P.grav[0] = c.gravity[0];
    P.grav[1] = c.gravity[1];
    return SPH_OK;
}

int status_to_code(unsigned st) {
    if (st & ST_DOMAIN) return SPH_E_DOMAIN;
    if (st & (ST_NBR_OVERFLOW | ST_PAIR_OVERFLOW)) return SPH_E_CAPACITY;
    if (st & ST_NONFINITE) return SPH_E_NONFINITE;
    if (st & ST_SKIN) return SPH_E_SKIN;
    return SPH_OK;
}

// --- timing helpers ---------------------------------------------------------
void tic(sph_handle* h, int phase) {
    if (!h->timing) return;
    if (h->ev_used >= h->ev_pool.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        h->ev_pool.push_back(e);
    }
    cudaEventRecord(h->ev_pool[h->ev_used], h->stream);
    h->ev_phase.push_back(phase);
    h->ev_used++;
}

void timing_flush(sph_handle* h) {
    if (!h->timing || h->ev_used == 0) return;
    cudaEventSynchronize(h->ev_pool[h->ev_used - 1]);
    for (size_t k = 0; k + 1 < h->ev_used; ++k) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, h->ev_pool[k], h->ev_pool[k + 1]);
        int ph = h->ev_phase[k];
        if (ph >= 0 && ph < PH_COUNT) h->t_ms[ph] += ms;
        h->t_total += ms;
    }
    h->ev_used = 0;
    h->ev_phase.clear();
}

template <typename R> Sorted<R>& sorted(sph_handle* h);
template <> Sorted<double>& sorted<double>(sph_handle* h) { return h->D64; }
template <> Sorted<float>& sorted<float>(sph_handle* h) { return h->D32; }

template <typename R>
int alloc_sorted(Sorted<R>& D, int cap, int max_nbr, int ncells) {
    CK(dalloc(&D.id, cap)); CK(dalloc(&D.type, cap)); CK(dalloc(&D.itype, cap)); CK(dalloc(&D.blabel, cap));
    CK(dalloc(&D.slot_of, cap)); CK(dalloc(&D.nflag, cap));
    CK(dalloc(&D.pos, cap)); CK(dalloc(&D.pos0, cap)); CK(dalloc(&D.vel0, cap)); CK(dalloc(&D.rho0, cap));
    CK(dalloc(&D.mass, cap)); CK(dalloc(&D.smass, cap));
    CK(dalloc(&D.kin, cap)); CK(dalloc(&D.aux, cap));
    CK(dalloc(&D.nb1, cap)); CK(dalloc(&D.nb2, cap)); CK(dalloc(&D.nb3, cap)); CK(dalloc(&D.binv, cap));
    CK(dalloc(&D.binv64, cap));
    CK(dalloc(&D.fra_v, cap)); CK(dalloc(&D.flags, cap));
    CK(dalloc(&D.drho, cap)); CK(dalloc(&D.acc, cap)); CK(dalloc(&D.avg, cap)); CK(dalloc(&D.shift, cap));
    CK(dalloc(&D.ks_r, cap)); CK(dalloc(&D.ks_a, cap)); CK(dalloc(&D.ks_v, cap));
    CK(dalloc(&D.c_drho, cap)); CK(dalloc(&D.c_acc, cap)); CK(dalloc(&D.c_avg, cap));
    CK(dalloc(&D.nbr, (size_t)cap * max_nbr)); CK(dalloc(&D.nnbr, cap));
    CK(dalloc(&D.pairs, (size_t)cap * max_nbr)); CK(dalloc(&D.npairs, cap));
    CK(dalloc(&D.cell_start, ncells)); CK(dalloc(&D.cell_end, ncells));
    if (sizeof(R) == 4) {
        CK(dalloc(&D.kh, cap)); CK(dalloc(&D.kl, cap)); CK(dalloc(&D.xhl, cap)); CK(dalloc(&D.vol64, cap));
    }
    CK(cudaMemset(D.nb3, 0, sizeof(*D.nb3) * (size_t)cap));
    CK(cudaMemset(D.flags, 0, (size_t)cap));
    return SPH_OK;
}

template <typename R>
void free_sorted(Sorted<R>& D) {
    void* ptrs[] = {D.id, D.type, D.itype, D.blabel, D.pos, D.pos0, D.vel0, D.rho0, D.mass, D.smass, D.kin, D.aux, D.nb1, D.nb2, D.nb3,
                    D.binv, D.binv64, D.fra_v, D.flags, D.drho, D.acc, D.avg, D.shift, D.ks_r, D.ks_a, D.ks_v, D.c_drho,
                    D.c_acc, D.c_avg, D.nbr, D.nnbr, D.pairs, D.npairs, D.cell_start, D.cell_end, D.kh, D.kl,
                    D.xhl, D.vol64, D.slot_of, D.nflag};
    for (void* p : ptrs) if (p) cudaFree(p);
    D = Sorted<R>{};
}

// sorted master state -> staging (id order)
template <typename R>
int unsort(sph_handle* h) {
    if (h->staging_valid) return SPH_OK;
    if (!h->sorted_valid) return SPH_E_ARG;
    Params P = h->P;
    k_unsort<R><<<blocks(P.n_tot, 256), 256, 0, h->stream>>>(P, h->S, sorted<R>(h));
    CK(cudaGetLastError());
    h->launches += 1;
    h->staging_valid = true;
    return SPH_OK;
}

// One exclusive scan of cnt[0..n) into off, returning the total on the host.
int scan_total(sph_handle* h, const int* cnt, int* off, int n, int* total) {
    if (n <= 0) { *total = 0; return SPH_OK; }
    size_t bytes = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, cnt, off, n, h->stream));
    if (bytes > h->cub_bytes) return SPH_E_CAPACITY;
    CK(cub::DeviceScan::ExclusiveSum(h->cub_tmp, bytes, cnt, off, n, h->stream));
    int last[2];
    CK(cudaMemcpyAsync(&last[0], off + n - 1, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(&last[1], cnt + n - 1, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    *total = last[0] + last[1];
    return SPH_OK;
}

// Step-start set-up: wrap + periodic images, sort, cell ranges, lists, records.
template <typename R>
int prepare(sph_handle* h) {
    int rc = unsort<R>(h);
    if (rc) return rc;
    Params& P = h->P;
    P.n_host = h->n_host;
    tic(h, PH_IMAGES);
    int n_img = 0;
    if (h->cfg.periodic) {
        // left/right images of the host particles; the counts and offsets are
        // kept for routing image adjoints back to their sources
        k_img_count<<<blocks(h->n_host, 256), 256, 0, h->stream>>>(P, h->S, h->n_host, 0, h->S.lr_cnt);
        int n_lr = 0;
        rc = scan_total(h, h->S.lr_cnt, h->S.lr_off, h->n_host, &n_lr);
        if (rc) return rc;
        if (h->n_host + n_lr > h->cap_tot) return SPH_E_CAPACITY;
        k_img_emit<<<blocks(h->n_host, 256), 256, 0, h->stream>>>(P, h->S, h->n_host, 0, h->n_host, h->S.lr_off);
        // bottom/top images of host particles and left/right images
        const int n_src = h->n_host + n_lr;
        k_img_count<<<blocks(n_src, 256), 256, 0, h->stream>>>(P, h->S, n_src, 1, h->S.tb_cnt);
        int n_tb = 0;
        rc = scan_total(h, h->S.tb_cnt, h->S.tb_off, n_src, &n_tb);
        if (rc) return rc;
        if (n_src + n_tb > h->cap_tot) return SPH_E_CAPACITY;
        k_img_emit<<<blocks(n_src, 256), 256, 0, h->stream>>>(P, h->S, n_src, 1, n_src, h->S.tb_off);
        h->n_lr = n_lr;
        n_img = n_lr + n_tb;
        CK(cudaGetLastError());
    }
    h->n_img = n_img;
    h->launches += h->cfg.periodic ? 4 : 0;
    P.n_tot = h->n_host + n_img;
    tic(h, PH_SORT);
    Sorted<R>& D = sorted<R>(h);
    k_cell_keys<<<blocks(P.n_tot, 256), 256, 0, h->stream>>>(P, h->S.pos, h->S.type, h->keys_in, h->vals_in,
                                                              h->d_status, h->dead_key);
    size_t bytes = h->cub_bytes;
    CK(cub::DeviceRadixSort::SortPairs(h->cub_tmp, bytes, h->keys_in, h->keys_out, h->vals_in, h->vals_out,
                                       P.n_tot, 0, h->key_bits, h->stream));
    k_gather_sorted<R><<<blocks(P.n_tot, 256), 256, 0, h->stream>>>(P, h->S, D, h->vals_out);
    CK(cudaMemsetAsync(D.cell_start, 0xff, sizeof(int) * (size_t)h->ncells, h->stream));
    CK(cudaMemsetAsync(D.cell_end, 0xff, sizeof(int) * (size_t)h->ncells, h->stream));
    k_cell_ranges<<<blocks(P.n_tot, 256), 256, 0, h->stream>>>(P.n_tot, h->keys_out, D.cell_start, D.cell_end,
                                                                h->dead_key);
    k_build_lists<R><<<blocks(P.n_tot, 128), 128, 0, h->stream>>>(P, D, h->d_status);
    CK(cudaGetLastError());
    h->launches += 4;
    h->sorted_valid = true;
    h->staging_valid = false;   // the master state now lives in the sorted arrays
    return SPH_OK;
}

template <typename R>
int keep_stage(sph_handle* h, int j, int k);

// One RHS evaluation on the current stage state.  keep_j >= 0 (the adjoint's
// segment re-run): the ghost interpolation sums go to gint / gsw and the state
// after the ghost assignment to stage slot keep_j.
template <typename R>
int rhs(sph_handle* h, int last, int keep_j = -1, double4* gint = nullptr, double* gsw = nullptr) {
    const Params& P = h->P;
    Sorted<R>& D = sorted<R>(h);
    const int nb = blocks(P.n_tot, 128);
    if (P.ghost_assign) {
        // Assign_boundary_particles at the start of single_step_compute (MS Single_step_compute.f90:73)
        tic(h, PH_UPDATE);
        if (h->n_ghost > 0) {
            k_assign_ghosts<R><<<blocks((long long)h->n_ghost * 32, 128), 128, 0, h->stream>>>(
                P, D, h->d_ghost_ids, h->n_ghost, h->t_phys, h->body_vel[0], h->body_vel[1], h->body_acc[0],
                h->body_acc[1], gint, gsw);
            h->launches += 1;
        }
    }
    if (keep_j >= 0) {
        int rc = keep_stage<R>(h, keep_j, 0);
        if (rc) return rc;
    }
    tic(h, PH_A);
    launch_pass_a<R, true>(P, D, nb, h->stream);
    tic(h, PH_SURF);
    launch_surface<R>(P, D, h->stream);
    tic(h, PH_C);
    // the mixed Taylor-Green path forms the shifting sum in k_shift_gather after
    // pass C; the FP64 and moving-square launches form it inside pass C
    const bool sep = sizeof(R) == 4 && !P.ms;
    const bool sh = last && h->cfg.shifting;
    const bool shc = sh && !sep;
    if (P.ms) {
        if (shc) k_pass_c<R, false, true, true><<<nb, 128, 0, h->stream>>>(P, D);
        else k_pass_c<R, false, true, false><<<nb, 128, 0, h->stream>>>(P, D);
    } else if (P.muscl) {
        if constexpr (sizeof(R) == 8) {       // the mixed launches never carry the sum
            if (shc) k_pass_c<R, true, false, true><<<nb, 128, 0, h->stream>>>(P, D);
            else k_pass_c<R, true, false, false><<<nb, 128, 0, h->stream>>>(P, D);
        } else {
            k_pass_c<R, true, false, false><<<nb, 128, 0, h->stream>>>(P, D);
        }
    } else {
        if constexpr (sizeof(R) == 8) {
            if (shc) k_pass_c<R, false, false, true><<<nb, 128, 0, h->stream>>>(P, D);
            else k_pass_c<R, false, false, false><<<nb, 128, 0, h->stream>>>(P, D);
        } else {
            k_pass_c<R, false, false, false><<<nb, 128, 0, h->stream>>>(P, D);
        }
    }
    if constexpr (sizeof(R) == 4) if (sh && sep) {
        // timed with the update: shifting is part of the step's second pass
        tic(h, PH_UPDATE);
        k_shift_gather<R><<<nb, 128, 0, h->stream>>>(P, D);
        h->launches += 1;
    }
    CK(cudaGetLastError());
    h->launches += P.free_surface ? 4 : 2;
    if (P.has_body && (last || h->bf_every_rhs)) {
        const int nbf = blocks(P.n_tot, kRedThreads);      // <= blocks(cap_tot), the partial buffer size
        double* fin = h->d_bf + (size_t)6 * blocks(h->cap_tot, kRedThreads);
        k_body_force<R><<<nbf, kRedThreads, 0, h->stream>>>(P, D, h->d_bf);
        k_body_force_final<<<1, kRedThreads, 0, h->stream>>>(nbf, h->d_bf, fin);
        h->bf_pending = true;
        h->launches += 2;
        if (h->drag_acc && last) {
            k_drag_acc<<<1, 32, 0, h->stream>>>(fin, h->drag_w, h->drag_acc);
            h->launches += 1;
        }
    }
    h->n_rhs++;
    h->have_rhs = true;
    return SPH_OK;
}

template <typename R>
int stage(sph_handle* h, int st, double dt, int use_carried, int do_shift, int to_staging = 0) {
    const Params& P = h->P;
    tic(h, PH_UPDATE);
    k_stage<R><<<blocks(P.n_tot, 256), 256, 0, h->stream>>>(P, sorted<R>(h), st, dt, use_carried, do_shift,
                                                             h->d_status, h->S, to_staging);
    CK(cudaGetLastError());
    h->launches += 1;
    return SPH_OK;
}

int read_status(sph_handle* h) {
    unsigned st = 0;
    CK(cudaMemcpyAsync(&st, h->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (st) CK(cudaMemsetAsync(h->d_status, 0, sizeof(unsigned), h->stream));
    return status_to_code(st);
}

// Reinitialize_particle_density on the state after the integrator update of a
// step, then the step's shift (time_iteration.f90:673-682).
template <typename R>
int reinit_density(sph_handle* h, int do_shift) {
    const Params& P = h->P;
    Sorted<R>& D = sorted<R>(h);
    const int nb = blocks(P.n_tot, 128);
    tic(h, PH_UPDATE);
    // (order 1 formed its densities on the step's last RHS: mls1_on_last_rhs)
    if (P.mls_order == 6) k_mls<R, 6><<<nb, 128, 0, h->stream>>>(P, D, h->d_mls);
    else if (P.mls_order == 3) k_mls<R, 3><<<nb, 128, 0, h->stream>>>(P, D, h->d_mls);
    k_finish_mls<R><<<blocks(P.n_tot, 256), 256, 0, h->stream>>>(P, D, h->d_mls, do_shift, h->d_status);
    CK(cudaGetLastError());
    h->launches += P.mls_order == 1 ? 1 : 2;
    return SPH_OK;
}

// MLS order 1 reads the pair list and state of the step's last RHS: formed right
// after it, before the stage that ends the step moves the particles.
template <typename R>
int mls1_on_last_rhs(sph_handle* h) {
    const Params& P = h->P;
    tic(h, PH_UPDATE);
    k_mls1<R><<<blocks(P.n_tot, 128), 128, 0, h->stream>>>(P, sorted<R>(h), h->d_mls);
    CK(cudaGetLastError());
    h->launches += 1;
    return SPH_OK;
}

// Start of a step: Real_time = Real_time + dt, then Body_Motion_Solver (MS
// SPH_Time_Iteration.f90:71-114): the body motion of the step (an adjoint run's
// schedule, else the handle's), and the body moved by its velocity times dt.
template <typename R>
int step_begin(sph_handle* h, double dt) {
    h->t_phys += dt;
    if (h->sched) {
        const long long k = h->step_count - h->sched_step0;
        if (k >= 0 && k < h->sched_n) {
            const double* m = h->sched + 4 * k;
            h->body_vel[0] = m[0]; h->body_vel[1] = m[1]; h->body_acc[0] = m[2]; h->body_acc[1] = m[3];
        }
    }
    if (h->P.ghost_assign && (h->body_vel[0] != 0.0 || h->body_vel[1] != 0.0)) {
        int rc = unsort<R>(h);
        if (rc) return rc;
        k_translate_body<<<blocks(h->n_host, 256), 256, 0, h->stream>>>(h->n_host, h->S.itype, h->S.pos,
                                                                          h->body_vel[0] * dt, h->body_vel[1] * dt);
        CK(cudaGetLastError());
        h->launches += 1;
        h->sorted_valid = false;
    }
    return SPH_OK;
}

template <typename R>
int run_steps(sph_handle* h, int nsteps, double dt) {
    for (int s = 0; s < nsteps; ++s) {
        int rc = step_begin<R>(h, dt);
        if (rc) return rc;
        rc = prepare<R>(h);
        if (rc) return rc;
        const int first = h->step_count == 0;
        // density re-initialisation after every mls_every-th step (1-based step number)
        const bool mls = h->P.mls_order != 0 && (h->step_count + 1) % h->P.mls_every == 0;
        const int shift_now = mls ? 0 : h->cfg.shifting;
        // the Taylor-Green driver's final stage keeps the id-order staging current
        // (the moving-square ghost assignment and MLS change the sorted state
        // after or outside it)
        const int to_staging = (!h->P.ms && !h->P.ghost_assign && !mls) ? 1 : 0;
        if (first) { rc = rhs<R>(h, 0); if (rc) return rc; }
        const bool mls1 = mls && h->P.mls_order == 1;
        if (h->cfg.integrator == SPH_INTEGRATOR_EULER_PC) {
            rc = stage<R>(h, 10, dt, first ? 0 : 1, 0); if (rc) return rc;
            rc = rhs<R>(h, 1); if (rc) return rc;
            if (mls1 && (rc = mls1_on_last_rhs<R>(h))) return rc;
            rc = stage<R>(h, 11, dt, 0, shift_now); if (rc) return rc;
        } else {
            rc = stage<R>(h, 0, dt, first ? 0 : 1, 0); if (rc) return rc;
            rc = rhs<R>(h, 0); if (rc) return rc;
            rc = stage<R>(h, 1, dt, 0, 0); if (rc) return rc;
            rc = rhs<R>(h, 0); if (rc) return rc;
            rc = stage<R>(h, 2, dt, 0, 0); if (rc) return rc;
            rc = rhs<R>(h, 1); if (rc) return rc;
            if (mls1 && (rc = mls1_on_last_rhs<R>(h))) return rc;
            rc = stage<R>(h, 3, dt, 0, shift_now, to_staging); if (rc) return rc;
            if (to_staging) h->staging_valid = true;
        }
        if (mls && (rc = reinit_density<R>(h, h->cfg.shifting))) return rc;
        tic(h, -1);
        h->step_count++;
        h->n_steps++;
        if (h->ev_used > 4096) timing_flush(h);
    }
    timing_flush(h);
    return read_status(h);
}

template <typename R>
int diagnostics(sph_handle* h, sph_diag* out) {
    memset(out, 0, sizeof(*out));
    if (!h->sorted_valid) {
        // state only in staging: sort it once to reduce over the same arrays
        int rc = prepare<R>(h);
        if (rc) return rc;
    }
    const Params& P = h->P;
    const int nparts = 148 * 4;
    k_diag_partial<R><<<nparts, kRedThreads, 0, h->stream>>>(P, sorted<R>(h), h->d_part, h->d_part + nparts);
    k_diag_final<<<1, kRedThreads, 0, h->stream>>>(nparts, h->d_part, h->d_part + nparts, h->d_diag);
    CK(cudaMemsetAsync(h->d_int, 0, sizeof(int), h->stream));
    k_count_surface<R><<<blocks(P.n_tot, 256), 256, 0, h->stream>>>(P, sorted<R>(h), h->d_int);
    h->launches += 3;
    double v[2];
    int nsurf = 0;
    CK(cudaMemcpyAsync(v, h->d_diag, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(&nsurf, h->d_int, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    if (h->bf_pending) {
        const double* fin = h->d_bf + (size_t)6 * blocks(h->cap_tot, kRedThreads);
        CK(cudaMemcpyAsync(h->bf, fin, 6 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    h->bf_pending = false;
    out->kinetic_energy = v[0];
    out->max_speed = v[1];
    out->n_images = h->n_img;
    out->n_surface = h->have_rhs ? nsurf : 0;
    out->pair_count = h->last_pairs;
    for (int c = 0; c < 6; ++c) out->body_force[c] = h->bf[c];
    return SPH_OK;
}

__global__ void k_to_ll(int n, const int* in, long long* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[i];
}

// find_particle_pair on the current (prepared) state.
template <typename R>
int find_pairs(sph_handle* h, long long pair_cap, int* pi, int* pj, double* w, double* dwdx, long long* total) {
    const Params& P = h->P;
    const int n = P.n_tot;
    if (!h->d_cnt_id) CK(dalloc(&h->d_cnt_id, h->cap_tot));
    if (!h->d_off64) CK(dalloc(&h->d_off64, 2 * ((size_t)h->cap_tot + 1)));
    long long* cnt64 = h->d_off64 + (h->cap_tot + 1);
    k_pair_count<R><<<blocks(n, 128), 128, 0, h->stream>>>(P, sorted<R>(h), h->d_cnt_id);
    k_to_ll<<<blocks(n, 256), 256, 0, h->stream>>>(n, h->d_cnt_id, cnt64);
    size_t bytes = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, cnt64, h->d_off64, n, h->stream));
    if (bytes > h->cub_bytes) return SPH_E_CAPACITY;
    CK(cub::DeviceScan::ExclusiveSum(h->cub_tmp, bytes, cnt64, h->d_off64, n, h->stream));
    long long last[2];
    CK(cudaMemcpyAsync(&last[0], h->d_off64 + n - 1, sizeof(long long), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(&last[1], cnt64 + n - 1, sizeof(long long), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    *total = last[0] + last[1];
    h->last_pairs = *total;
    if (pi == nullptr || pair_cap <= 0) return SPH_OK;
    const long long m = std::min(*total, pair_cap);
    int *dpi = nullptr, *dpj = nullptr;
    double *dw = nullptr, *ddw = nullptr;
    CK(dalloc(&dpi, m)); CK(dalloc(&dpj, m));
    if (w) CK(dalloc(&dw, m));
    if (dwdx) CK(dalloc(&ddw, 2 * m));
    k_pair_emit<R><<<blocks(n, 128), 128, 0, h->stream>>>(P, sorted<R>(h), h->d_off64, m, dpi, dpj, dw, ddw);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(pi, dpi, sizeof(int) * m, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(pj, dpj, sizeof(int) * m, cudaMemcpyDeviceToHost, h->stream));
    if (w) CK(cudaMemcpyAsync(w, dw, sizeof(double) * m, cudaMemcpyDeviceToHost, h->stream));
    if (dwdx) {
        CK(cudaMemcpyAsync(dwdx, ddw, sizeof(double) * m, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(dwdx + pair_cap, ddw + m, sizeof(double) * m, cudaMemcpyDeviceToHost, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    cudaFree(dpi); cudaFree(dpj);
    if (dw) cudaFree(dw);
    if (ddw) cudaFree(ddw);
    return *total > pair_cap ? SPH_E_CAPACITY : SPH_OK;
}

template <typename R>
int export_fields(sph_handle* h) {
    if (!h->have_rhs || !h->sorted_valid) return SPH_E_ARG;
    if (!h->d_export) CK(dalloc(&h->d_export, (size_t)kExportFields * h->cap_host));
    const Params& P = h->P;
    k_export<R><<<blocks(P.n_tot, 256), 256, 0, h->stream>>>(P, sorted<R>(h), h->d_export);
    CK(cudaGetLastError());
    return SPH_OK;
}

// ---------------------------------------------------------------------------
// Discrete adjoint: checkpointed forward run and the reverse sweep.
// ---------------------------------------------------------------------------

// Host-particle state in id order: what a step starts from.
struct Snap {
    double2 *pos = nullptr, *vel = nullptr, *r_acc = nullptr, *r_avg = nullptr;
    double *rho = nullptr, *r_drho = nullptr;
};

}  // namespace

struct AdjCtx {
    bool valid = false;
    int nsteps = 0, every = 0, loss = 0, nseg = 0;
    double dt = 0.0;
    long long step0 = 0;       // handle step count when the forward started
    int n_host = 0;
    int cap_ck = 0, cap_seg = 0, cap_host = 0, cap_tot = 0;
    Snap ck;                   // checkpoints [nseg + 1] (the last: the final state)
    Snap seg;                  // step-start states of the segment being reversed
    // stage states S1..S3 in sorted order (and, with density re-initialisation,
    // the state the step's last stage produced before it), [stage_slots][nst][cap_tot]: one slot per
    // step of the segment when memory allows (kept while the segment is re-run),
    // else one slot that each reversed step recomputes
    int stage_slots = 0;
    int nst = 3;                // states per stage slot
    // reverse of the density re-initialisation (moving least squares, orders 3 and 6)
    double2* mls_x = nullptr;   // adjoint of the positions it read, per slot
    double* mls_r = nullptr;    //   and of the densities
    double* mls_lam = nullptr;  // adjoint of the densities it produced
    double* mls_cy = nullptr;   // per owner: c = A^-1 e_1, y = A^-1 (lam r), (mode, sum W, out, own) [16]
    double2* mls_xe = nullptr;  // the step end's position adjoint (after the shift's reverse)
    double2* mls_xo = nullptr;  // an owner's position adjoint through its own sum
    double2* mls_gm = nullptr;  // moving square: the ghosts' density and mass adjoints through it
    double2* st_pos = nullptr;
    double4* st_kin = nullptr;
    double4* st_aux = nullptr;  // V4 of the pair precision (float4 uses the first half)
    std::vector<int> seg_ntot;  // particles + images of each step of the segment
    // sorted step-start state of each step of the segment (PrepDesc), kept with
    // the stage states when memory allows: [stage_slots][prep_words]
    unsigned* prep = nullptr;
    long long prep_words = 0;
    PrepDesc* d_prep = nullptr;    // descriptor table (rebuilt by each forward call)
    int n_prep = 0, cap_prep = 0;
    long long prep_nnbr_off = 0;   // slot offset of the saved list lengths
    std::vector<int> seg_nimg, seg_nlr;
    // moving square: what the corrector RHS of each step of the segment computed
    // before pass C (the ghost interpolation sums, pass A's pair list, B^-1,
    // gradient records, flags and XSPH velocity), written there by the segment
    // re-run and read by the reverse step instead of re-running the ghost
    // assignment, pass A and the surface tests (allocated with the sorted-state
    // slots when they also leave 1 GiB free).  Per slot: pairs [max_nbr][cap_tot],
    // the rest [cap_tot]; the pair-precision arrays as bytes.
    bool pa = false;
    int pa_per_step = 0;         // pass-A slots per step: 1 (Euler PC corrector) or 3 (RK4 RHS 2-4)
    unsigned* pa_pairs = nullptr;
    int* pa_npairs = nullptr;
    unsigned char* pa_binv = nullptr;
    unsigned char* pa_nb1 = nullptr;
    unsigned char* pa_nb2 = nullptr;
    unsigned char* pa_nb3 = nullptr;   // Taylor-Green only (MUSCL gradients, 1/rho)
    unsigned char* pa_fra = nullptr;
    unsigned char* pa_avg = nullptr;
    uint8_t* pa_flags = nullptr;
    double4* pa_binv64 = nullptr;
    double4* pa_gint = nullptr;
    double* pa_gsw = nullptr;
    std::vector<char> seg_kept;  // the corrector RHS of step j ran in the re-run into slot j
    double2* target = nullptr;
    double* loss_part = nullptr;
    Adj A{};
    std::vector<void*> owned;
    // moving-square runs
    int cap_steps = 0;          // capacity of A.g_motion in steps
    double t0 = 0.0;            // physical time the forward started from
    double dloss = 0.0;
    bool have_grad = false;     // A.g_motion holds the last backward pass's result
    std::vector<double> motion; // [4 nsteps] body motion schedule (empty: the handle's)
    double* drag_acc = nullptr; // [1] drag loss of the forward run
};

namespace {

template <typename T>
int adj_alloc(AdjCtx* X, T** p, size_t count) {
    CK(dalloc(p, count));
    X->owned.push_back((void*)*p);
    return SPH_OK;
}

void adj_free_all(AdjCtx* X) {
    for (void* p : X->owned) cudaFree(p);
    X->owned.clear();
}

int snap_alloc(AdjCtx* X, Snap& s, size_t n) {
    int rc;
    if ((rc = adj_alloc(X, &s.pos, n)) || (rc = adj_alloc(X, &s.vel, n)) || (rc = adj_alloc(X, &s.r_acc, n)) ||
        (rc = adj_alloc(X, &s.r_avg, n)) || (rc = adj_alloc(X, &s.rho, n)) || (rc = adj_alloc(X, &s.r_drho, n)))
        return rc;
    return SPH_OK;
}

// staging (id order) <-> snapshot slot k
int snap_io(sph_handle* h, const Snap& s, int k, int n, bool save) {
    const size_t o = (size_t)k * n;
    const SnapPtrs slot{s.pos + o, s.vel + o, s.r_acc + o, s.r_avg + o, s.rho + o, s.r_drho + o};
    const SnapPtrs stg{h->S.pos, h->S.vel, h->S.r_acc, h->S.r_avg, h->S.rho, h->S.r_drho};
    k_snap_copy<<<blocks(n, 256), 256, 0, h->stream>>>(n, save ? slot : stg, save ? stg : slot);
    CK(cudaGetLastError());
    h->launches += 1;
    if (!save) {
        h->staging_valid = true;
        h->sorted_valid = false;
    }
    return SPH_OK;
}

int adj_config_ok(const sph_handle* h, int loss) {
    const Params& P = h->P;
    if (P.ms) {
        // moving-square modified linear or HLLC solver, Morris laplacian, Euler
        // predictor-corrector, with or without shifting
        if ((h->cfg.solver != SPH_SOLVER_MS_MODLR_DELTA && h->cfg.solver != SPH_SOLVER_MS_HLLC_DELTA) ||
            P.laplacian != 1)
            return SPH_E_CONFIG;
        if (h->cfg.integrator != SPH_INTEGRATOR_EULER_PC || h->cfg.periodic) return SPH_E_CONFIG;
    } else {
        if ((h->cfg.solver != SPH_SOLVER_MODLR_DELTA_SPS && h->cfg.solver != SPH_SOLVER_MUSCL_DELTA_SPS &&
             h->cfg.solver != SPH_SOLVER_DELTA_SPS) ||
            P.xsph)
            return SPH_E_CONFIG;
        if (h->cfg.integrator != SPH_INTEGRATOR_RK4_REUSE) return SPH_E_CONFIG;
    }
    if (loss == SPH_LOSS_DRAG && !P.has_body) return SPH_E_CONFIG;
    return SPH_OK;
}

// Clears the per-step schedule and the drag accumulation of the handle on exit.
struct SchedGuard {
    sph_handle* h;
    ~SchedGuard() { h->sched = nullptr; h->sched_n = 0; h->drag_acc = nullptr; }
};

// The arrays prepare writes for one step (see PrepDesc): per-particle fields of
// the sorted state, one descriptor per neighbour-list row, the cell ranges and
// the id-order image routing; slot offsets from the capacities, 256-byte aligned.
template <typename R>
std::vector<PrepDesc> prep_table(sph_handle* h, long long* words, long long* nnbr_off = nullptr) {
    Sorted<R>& D = sorted<R>(h);
    std::vector<PrepDesc> v;
    long long off = 0;
    const long long cap = h->cap_tot;
    auto add = [&](void* f, int per_particle, long long w, long long pitch = 0) {
        v.push_back(PrepDesc{(unsigned*)f, off, per_particle, (int)w, pitch});
        const long long nw = pitch > 0 ? pitch * w : per_particle ? cap * w : w;
        off += (nw + 63) & ~63LL;
    };
    auto pp = [&](void* f, size_t bytes) { add(f, 1, (long long)(bytes / 4)); };
    pp(D.id, 4); pp(D.slot_of, 4); pp(D.type, 4); pp(D.itype, 4); pp(D.blabel, 4);
    pp(D.pos, sizeof(*D.pos)); pp(D.pos0, sizeof(*D.pos0)); pp(D.vel0, sizeof(*D.vel0));
    pp(D.rho0, sizeof(*D.rho0)); pp(D.mass, sizeof(*D.mass)); pp(D.smass, sizeof(*D.smass));
    pp(D.kin, sizeof(*D.kin)); pp(D.aux, sizeof(*D.aux));
    pp(D.c_drho, sizeof(*D.c_drho)); pp(D.c_acc, sizeof(*D.c_acc)); pp(D.c_avg, sizeof(*D.c_avg));
    if (nnbr_off) *nnbr_off = off;
    pp(D.nnbr, 4);
    if (sizeof(R) == 4) {
        pp(D.vol64, sizeof(*D.vol64)); pp(D.kh, sizeof(*D.kh)); pp(D.kl, sizeof(*D.kl)); pp(D.xhl, sizeof(*D.xhl));
    }
    add(D.cell_start, 0, h->ncells);
    add(D.cell_end, 0, h->ncells);
    pp(h->S.lr_cnt, 4); pp(h->S.lr_off, 4); pp(h->S.tb_cnt, 4); pp(h->S.tb_off, 4);
    // the lists, last (a reverse step that does not re-run pass A skips them):
    // max_nbr rows at the lists' own pitch (nbr_stride = cap_tot)
    add(D.nbr, 1, h->P.max_nbr, h->P.nbr_stride);
    *words = off;
    return v;
}

long long prep_slot_words(sph_handle* h) {
    long long w = 0;
    if (h->mixed) prep_table<float>(h, &w);
    else prep_table<double>(h, &w);
    return w;
}

// Upload the descriptor table of the handle's current arrays (the per-call part).
template <typename R>
int prep_upload(sph_handle* h) {
    AdjCtx* X = h->adj;
    if (!X->prep) return SPH_OK;
    long long w = 0;
    std::vector<PrepDesc> v = prep_table<R>(h, &w, &X->prep_nnbr_off);
    if (w != X->prep_words) return SPH_E_ARG;
    if (X->cap_prep < (int)v.size()) {
        int rc = adj_alloc(X, &X->d_prep, v.size());
        if (rc) return rc;
        X->cap_prep = (int)v.size();
    }
    CK(cudaMemcpyAsync(X->d_prep, v.data(), sizeof(PrepDesc) * v.size(), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    X->n_prep = (int)v.size();
    return SPH_OK;
}

// After prepare in the segment re-run: keep what it wrote in slot j (lists =
// false: without the neighbour lists, the last descriptor).
int prep_save(sph_handle* h, int j, bool lists = true) {
    AdjCtx* X = h->adj;
    if (!X->prep) return SPH_OK;
    const int nt = h->P.n_tot;
    const int* cnt = h->mixed ? h->D32.nnbr : h->D64.nnbr;
    k_prep_copy<<<dim3(blocks(nt, 256), X->n_prep - (lists ? 0 : 1)), 256, 0, h->stream>>>(
        X->d_prep, nt, X->prep + (size_t)j * X->prep_words, 1, cnt);
    CK(cudaGetLastError());
    h->launches += 1;
    X->seg_nimg[j] = h->n_img;
    X->seg_nlr[j] = h->n_lr;
    return SPH_OK;
}

// In place of prepare in a reversed step: the sorted step-start state of slot j
// (the same as a re-sort of the restored step-start state gives, the sort being
// deterministic); lists = false: without the neighbour lists.
int prep_restore(sph_handle* h, int j, bool lists = true) {
    AdjCtx* X = h->adj;
    Params& P = h->P;
    P.n_host = h->n_host;
    h->n_img = X->seg_nimg[j];
    h->n_lr = X->seg_nlr[j];
    P.n_tot = h->n_host + h->n_img;
    tic(h, PH_SORT);
    unsigned* slot = X->prep + (size_t)j * X->prep_words;
    k_prep_copy<<<dim3(blocks(P.n_tot, 256), X->n_prep - (lists ? 0 : 1)), 256, 0, h->stream>>>(
        X->d_prep, P.n_tot, slot, 0, (const int*)(slot + X->prep_nnbr_off));
    CK(cudaGetLastError());
    h->launches += 1;
    h->sorted_valid = true;
    h->staging_valid = false;
    return SPH_OK;
}

int adj_prepare_ctx(sph_handle* h, const sph_adj_config* ac) {
    AdjCtx* X = h->adj;
    const int nseg = (ac->nsteps + ac->checkpoint_every - 1) / ac->checkpoint_every;
    const int every = std::min(ac->checkpoint_every, ac->nsteps);
    if (X && (X->cap_ck < nseg + 1 || X->cap_seg < every || X->cap_host < h->n_host || X->cap_tot < h->cap_tot)) {
        adj_free_all(X);
        delete X;
        X = h->adj = nullptr;
    }
    if (!X) {
        X = new (std::nothrow) AdjCtx();
        if (!X) return SPH_E_CAPACITY;
        h->adj = X;
        const size_t nh = (size_t)h->cap_host, nt = (size_t)h->cap_tot;
        X->cap_ck = nseg + 1; X->cap_seg = every; X->cap_host = h->cap_host; X->cap_tot = h->cap_tot;
        int rc;
        if ((rc = snap_alloc(X, X->ck, nh * (nseg + 1))) || (rc = snap_alloc(X, X->seg, nh * every))) return rc;
        if ((rc = adj_alloc(X, &X->target, nh)) || (rc = adj_alloc(X, &X->loss_part, 148 * 4))) return rc;
        Adj& A = X->A;
        for (int k = 0; k < 4; ++k)
            if ((rc = adj_alloc(X, &A.lr[k], nt)) || (rc = adj_alloc(X, &A.la[k], nt))) return rc;
        if ((rc = adj_alloc(X, &A.lxe, nt)) || (rc = adj_alloc(X, &A.ax0, nt)) || (rc = adj_alloc(X, &A.av0, nt)) ||
            (rc = adj_alloc(X, &A.ar0, nt)) || (rc = adj_alloc(X, &A.sx, nt)) || (rc = adj_alloc(X, &A.su, nt)) ||
            (rc = adj_alloc(X, &A.sr, nt)) || (rc = adj_alloc(X, &A.gbinv, nt)) || (rc = adj_alloc(X, &A.ggr, nt)) ||
            (rc = adj_alloc(X, &A.gtau, nt)) || (rc = adj_alloc(X, &A.mu1, nt)) || (rc = adj_alloc(X, &A.mu2, nt)) ||
            (rc = adj_alloc(X, &A.mu3, nt)) ||
            (rc = adj_alloc(X, &A.nu_part, (size_t)5 * blocks((long long)nt * kAdjLanes, kAdjThreads))) ||
            (rc = adj_alloc(X, &A.nu_acc, 1)) || (rc = adj_alloc(X, &A.irho, nt)) || (rc = adj_alloc(X, &A.ssum, nt)) || (rc = adj_alloc(X, &A.ggp, nt)) ||
            (rc = adj_alloc(X, &A.ggu, nt)) || (rc = adj_alloc(X, &A.ggv, nt)) || (rc = adj_alloc(X, &A.mu4, nt)) ||
            (rc = adj_alloc(X, &A.smu, nt)) || (rc = adj_alloc(X, &A.shgr, nt)) || (rc = adj_alloc(X, &A.shbi, nt)) || (rc = adj_alloc(X, &A.lx, nt)) || (rc = adj_alloc(X, &A.lv, nt)) ||
            (rc = adj_alloc(X, &A.lrho, nt)) || (rc = adj_alloc(X, &A.lk_r, nh)) || (rc = adj_alloc(X, &A.lk_a, nh)))
            return rc;
        // stage states: every step of a segment if that leaves 1 GiB free, else one
        X->nst = h->P.mls_order ? 4 : 3;
        const size_t per_slot = (size_t)X->nst * nt * (sizeof(double2) + 2 * sizeof(double4));
        size_t free_b = 0, total_b = 0;
        CK(cudaMemGetInfo(&free_b, &total_b));
        X->stage_slots = (per_slot * every + (size_t(1) << 30) <= free_b) ? every : 1;
        const size_t ns = (size_t)X->stage_slots * X->nst * nt;
        if ((rc = adj_alloc(X, &X->st_pos, ns)) || (rc = adj_alloc(X, &X->st_kin, ns)) ||
            (rc = adj_alloc(X, &X->st_aux, ns)))
            return rc;
        // the sorted step-start states, when every step has a stage slot and they
        // also leave 1 GiB free (else the reverse step re-sorts)
        const long long pw = prep_slot_words(h);
        CK(cudaMemGetInfo(&free_b, &total_b));
        if (X->stage_slots == every && (size_t)pw * 4 * every + (size_t(1) << 30) <= free_b) {
            if ((rc = adj_alloc(X, &X->prep, (size_t)pw * every))) return rc;
            X->prep_words = pw;
        }
        // (FP64 forward only: the mixed forward's pass A reads the hi/lo records,
        // the reverse step's re-run the FP64 state)
        // (the moving square: FP64 forward only)
        if (X->prep && (!h->P.ms || !h->mixed)) {
            const bool ms = h->P.ms != 0;
            const int per = ms ? 1 : 3;
            const size_t rs = h->mixed ? sizeof(float) : sizeof(double);
            const size_t per_pa = nt * ((size_t)h->P.max_nbr * 4 + 4 + (ms ? 3 : 4) * 4 * rs + rs + 2 * rs + 1 +
                                        sizeof(double4) + (ms ? sizeof(double4) + sizeof(double) : 0));
            CK(cudaMemGetInfo(&free_b, &total_b));
            if (per_pa * every * per + (size_t(1) << 30) <= free_b) {
                const size_t ne = nt * every * per;
                if ((rc = adj_alloc(X, &X->pa_pairs, ne * h->P.max_nbr)) || (rc = adj_alloc(X, &X->pa_npairs, ne)) ||
                    (rc = adj_alloc(X, &X->pa_binv, ne * 4 * rs)) || (rc = adj_alloc(X, &X->pa_nb1, ne * 4 * rs)) ||
                    (rc = adj_alloc(X, &X->pa_nb2, ne * 4 * rs)) || (rc = adj_alloc(X, &X->pa_fra, ne * rs)) ||
                    (rc = adj_alloc(X, &X->pa_avg, ne * 2 * rs)) || (rc = adj_alloc(X, &X->pa_flags, ne)) ||
                    (rc = adj_alloc(X, &X->pa_binv64, ne)))
                    return rc;
                if (ms && ((rc = adj_alloc(X, &X->pa_gint, ne)) || (rc = adj_alloc(X, &X->pa_gsw, ne)))) return rc;
                if (!ms && (rc = adj_alloc(X, &X->pa_nb3, ne * 4 * rs))) return rc;
                X->pa = true;
                X->pa_per_step = per;
            }
        }
    }
    if (h->P.mls_order && !X->mls_x) {
        const size_t nt = (size_t)X->cap_tot;
        int rc;
        if ((rc = adj_alloc(X, &X->mls_x, nt)) || (rc = adj_alloc(X, &X->mls_r, nt)) ||
            (rc = adj_alloc(X, &X->mls_lam, nt)) || (rc = adj_alloc(X, &X->mls_cy, nt * 16)) ||
            (rc = adj_alloc(X, &X->mls_xe, nt)) || (rc = adj_alloc(X, &X->mls_xo, nt)) ||
            (rc = adj_alloc(X, &X->mls_gm, nt)))
            return rc;
    }
    if (h->P.ms && !X->A.gavg) {
        Adj& A = X->A;
        const size_t nh = (size_t)X->cap_host, nt = (size_t)X->cap_tot;
        int rc;
        if ((rc = adj_alloc(X, &A.lg[0], nt)) || (rc = adj_alloc(X, &A.lg[1], nt)) ||
            (rc = adj_alloc(X, &A.lk_g, nh)) || (rc = adj_alloc(X, &A.gavg, nt)) || (rc = adj_alloc(X, &A.sm, nt)) ||
            (rc = adj_alloc(X, &A.glam, nt)) || (rc = adj_alloc(X, &A.glamw, nt)) ||
            (rc = adj_alloc(X, &A.gint, nt)) || (rc = adj_alloc(X, &A.gsw, nt)) ||
            // per-block partials: k_adj_ghost_lambda (4 per block of 4 ghosts), k_adj_body_pos (2 per block of 256)
            (rc = adj_alloc(X, &A.mo_part, std::max((size_t)4 * blocks((long long)nh * 32, kAdjThreads),
                                                    (size_t)2 * blocks((long long)nt, 256)))) ||
            (rc = adj_alloc(X, &X->drag_acc, 1)))
            return rc;
    }
    if (X->cap_steps < ac->nsteps) {
        int rc = adj_alloc(X, &X->A.g_motion, (size_t)4 * ac->nsteps);
        if (rc) return rc;
        X->cap_steps = ac->nsteps;
    }
    X->valid = false;
    X->have_grad = false;
    X->nsteps = ac->nsteps; X->every = every; X->nseg = nseg; X->loss = ac->loss; X->dt = ac->dt;
    X->n_host = h->n_host;
    X->seg_ntot.assign(every, 0);
    X->seg_nimg.assign(every, 0);
    X->seg_nlr.assign(every, 0);
    X->seg_kept.assign(every, 0);
    return SPH_OK;
}

template <typename R>
int adjoint_forward(sph_handle* h, const sph_adj_config* ac, double* loss) {
    int rc = adj_prepare_ctx(h, ac);
    if (rc || (rc = prep_upload<R>(h))) return rc;
    AdjCtx* X = h->adj;
    // with density re-initialisation every step of a segment keeps its states
    // (the reverse of a re-initialised step reads the state before it)
    if (h->P.mls_order && X->stage_slots < X->every) return SPH_E_CAPACITY;
    const int n = h->n_host;
    if (ac->loss == SPH_LOSS_VELOCITY_MISFIT) {
        CK(cudaMemcpyAsync(h->d_xfer, ac->target_vel, sizeof(double) * 2 * n, cudaMemcpyHostToDevice, h->stream));
        k_interleave<<<blocks(n, 256), 256, 0, h->stream>>>(n, h->d_xfer, X->target);
        h->launches += 1;
    }
    X->step0 = h->step_count;
    X->t0 = h->t_phys;
    X->motion.clear();
    if (ac->body_motion) X->motion.assign(ac->body_motion, ac->body_motion + 4 * (size_t)ac->nsteps);
    SchedGuard guard{h};
    if (!X->motion.empty()) {
        h->sched = X->motion.data(); h->sched_step0 = X->step0; h->sched_n = X->nsteps;
    }
    if (ac->loss == SPH_LOSS_DRAG) {
        CK(cudaMemsetAsync(X->drag_acc, 0, sizeof(double), h->stream));
        h->drag_acc = X->drag_acc;
        h->drag_w = ac->dt;
    }
    for (int c = 0; c < X->nseg; ++c) {
        if ((rc = unsort<R>(h)) || (rc = snap_io(h, X->ck, c, n, true))) return rc;
        const int ns = std::min(X->every, X->nsteps - c * X->every);
        if ((rc = run_steps<R>(h, ns, X->dt))) return rc;
    }
    if ((rc = unsort<R>(h)) || (rc = snap_io(h, X->ck, X->nseg, n, true))) return rc;
    double v = 0.0;
    if (ac->loss == SPH_LOSS_DRAG) {
        CK(cudaMemcpyAsync(&v, X->drag_acc, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    } else {
        const int nparts = 148 * 4;
        k_adj_loss<<<nparts, 256, 0, h->stream>>>(n, X->loss, h->S.type, h->S.vel, h->S.mass, X->target,
                                                 X->loss_part);
        h->launches += 2;
        CK(cudaMemsetAsync(h->d_diag, 0, sizeof(double), h->stream));
        k_adj_nu_sum<<<1, 1024, 0, h->stream>>>(nparts, X->loss_part, h->d_diag);
        CK(cudaMemcpyAsync(&v, h->d_diag, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    if (loss) *loss = v;
    X->valid = true;
    return SPH_OK;
}

// The sorted arrays with the positions and records of stage state k of stage slot j.
template <typename R>
Sorted<R> stage_view(sph_handle* h, int j, int k) {
    AdjCtx* X = h->adj;
    Sorted<R> V = sorted<R>(h);
    const size_t o = ((size_t)j * X->nst + k) * (size_t)X->cap_tot;
    V.pos = X->st_pos + o;
    V.kin = X->st_kin + o;
    V.aux = reinterpret_cast<typename VT<R>::V4*>(X->st_aux + o);
    return V;
}

// The sorted arrays V with what pass A writes (and the surface tests update)
// taken from pass-A slot j.
template <typename R>
Sorted<R> pa_view(sph_handle* h, Sorted<R> V, int j) {
    using V4 = typename VT<R>::V4;
    using V2 = typename VT<R>::V2;
    AdjCtx* X = h->adj;
    const size_t o = (size_t)j * X->cap_tot;
    V.pairs = X->pa_pairs + o * h->P.max_nbr;
    V.npairs = X->pa_npairs + o;
    V.binv = reinterpret_cast<V4*>(X->pa_binv) + o;
    V.nb1 = reinterpret_cast<V4*>(X->pa_nb1) + o;
    V.nb2 = reinterpret_cast<V4*>(X->pa_nb2) + o;
    V.fra_v = reinterpret_cast<R*>(X->pa_fra) + o;
    V.avg = reinterpret_cast<V2*>(X->pa_avg) + o;
    V.flags = X->pa_flags + o;
    V.binv64 = X->pa_binv64 + o;
    if (X->pa_nb3) V.nb3 = reinterpret_cast<V4*>(X->pa_nb3) + o;
    return V;
}

// While a kept corrector RHS and its stage run in the segment re-run, the
// handle's sorted arrays point at pass-A slot j; the destructor points them back.
template <typename R>
struct PaSwap {
    Sorted<R>& D;
    Sorted<R> saved;
    PaSwap(sph_handle* h, int j, bool on = true) : D(sorted<R>(h)), saved(D) {
        if (on) D = pa_view<R>(h, D, j);
    }
    ~PaSwap() { D = saved; }
};

// Copy the current stage state into stage slot j, state k.
template <typename R>
int keep_stage(sph_handle* h, int j, int k) {
    Sorted<R> V = stage_view<R>(h, j, k);
    const int nt = h->P.n_tot;
    k_keep_stage<R><<<blocks(nt, 256), 256, 0, h->stream>>>(nt, sorted<R>(h), V.pos, V.kin, V.aux);
    CK(cudaGetLastError());
    h->launches += 1;
    return SPH_OK;
}

// One step exactly as run_steps takes it, keeping the stage states in stage
// slot j (RK4: S1..S3; Euler predictor-corrector: the predicted state); with
// full = false the step stops after the last kept state (all the reverse needs).
template <typename R>
int step_keep(sph_handle* h, double dt, int j, bool full) {
    const int first = h->step_count == 0;
    // density re-initialisation after this step (1-based step number): the step
    // runs in full, and its reverse reads the state the last stage produced
    // (stage slot state 3) and the neighbour lists
    const bool mls = h->P.mls_order != 0 && (h->step_count + 1) % h->P.mls_every == 0;
    const bool mls1 = mls && h->P.mls_order == 1;   // formed on the last RHS, before the final stage
    if (mls) full = true;
    // the RHS evaluations of a step that runs here in full (the moving square's
    // corrector; the Runge-Kutta RHS 2-4) fill its pass-A slots, and its reverse
    // step re-runs no pass A, so it needs no neighbour lists
    const bool keep_pa = h->adj->pa && full && !first && !mls;
    int rc = step_begin<R>(h, dt);
    if (rc || (rc = prepare<R>(h)) || (rc = prep_save(h, j, !keep_pa))) return rc;
    h->adj->seg_ntot[j] = h->P.n_tot;
    if (first && (rc = rhs<R>(h, 0))) return rc;
    if (h->cfg.integrator == SPH_INTEGRATOR_EULER_PC) {
        AdjCtx* X = h->adj;
        X->seg_kept[j] = 0;
        if ((rc = stage<R>(h, 10, dt, first ? 0 : 1, 0))) return rc;
        if (keep_pa) {
            // the corrector RHS writes what pass A computes into pass-A slot j,
            // for the reverse step to read
            const size_t o = (size_t)j * X->cap_tot;
            {
                PaSwap<R> sw(h, j);
                if ((rc = rhs<R>(h, 1, j, X->pa_gint + o, X->pa_gsw + o)) ||
                    (rc = stage<R>(h, 11, dt, 0, h->cfg.shifting)))
                    return rc;
            }
            X->seg_kept[j] = 1;
            h->step_count++;
            h->n_steps++;
        } else {
            if ((rc = keep_stage<R>(h, j, 0))) return rc;
            if (full) {
                if ((rc = rhs<R>(h, 1)) || (mls1 && (rc = mls1_on_last_rhs<R>(h))) ||
                    (rc = stage<R>(h, 11, dt, 0, mls ? 0 : h->cfg.shifting)))
                    return rc;
                // the re-initialisation reads the corrected state (stage slot state 3)
                if (mls && ((rc = keep_stage<R>(h, j, 3)) || (rc = reinit_density<R>(h, h->cfg.shifting))))
                    return rc;
                h->step_count++;
                h->n_steps++;
            }
        }
        tic(h, -1);
        if (h->ev_used > 4096) timing_flush(h);
        return SPH_OK;
    }
    // RK4: RHS k + 1 (k = 0, 1, 2) on stage state S(k+1) and the stage it feeds
    // write pass A's outputs into pass-A slot 3 j + k when the step is kept
    h->adj->seg_kept[j] = keep_pa ? 1 : 0;
    if ((rc = stage<R>(h, 0, dt, first ? 0 : 1, 0)) || (rc = keep_stage<R>(h, j, 0))) return rc;
    {
        PaSwap<R> sw(h, 3 * j, keep_pa);
        if ((rc = rhs<R>(h, 0)) || (rc = stage<R>(h, 1, dt, 0, 0))) return rc;
    }
    if ((rc = keep_stage<R>(h, j, 1))) return rc;
    {
        PaSwap<R> sw(h, 3 * j + 1, keep_pa);
        if ((rc = rhs<R>(h, 0)) || (rc = stage<R>(h, 2, dt, 0, 0))) return rc;
    }
    if ((rc = keep_stage<R>(h, j, 2))) return rc;
    if (full) {
        {
            PaSwap<R> sw(h, 3 * j + 2, keep_pa);
            if ((rc = rhs<R>(h, 1)) || (mls1 && (rc = mls1_on_last_rhs<R>(h))) ||
                (rc = stage<R>(h, 3, dt, 0, mls ? 0 : h->cfg.shifting)))
                return rc;
        }
        if (mls && ((rc = keep_stage<R>(h, j, 3)) || (rc = reinit_density<R>(h, h->cfg.shifting)))) return rc;
        h->step_count++;
        h->n_steps++;
    }
    tic(h, -1);
    if (h->ev_used > 4096) timing_flush(h);
    return SPH_OK;
}

// Pass A and the surface tests re-run on a kept stage state V, as the forward
// ran them: the mixed forward reads the hi/lo records, which are formed here
// from V's FP64 state first (the same records the forward's stage wrote).
template <typename R>
void adj_pass_a(sph_handle* h, const Sorted<R>& V) {
    const Params& P = h->P;
    const int nb = blocks(P.n_tot, 128);
    if constexpr (sizeof(R) == 4) {
        k_resplit<R><<<blocks(P.n_tot, 256), 256, 0, h->stream>>>(P.n_tot, V);
        launch_pass_a<R, true>(P, V, nb, h->stream);
        h->launches += 1;
    } else {
        launch_pass_a<R, false>(P, V, nb, h->stream);
    }
    launch_surface<R>(P, V, h->stream);
    h->launches += P.free_surface ? 3 : 1;
}

// Reverse of one RHS evaluation on the stage state V, with the rate adjoints
// of RHS k of the step; stage = the stage that produced V (-1: the step start).
// shift: the last RHS of a step with particle shifting (pass A already re-run by
// adj_step, the step-end reverse left smu / shgr / shbi).
// mls1: the last RHS of a step that ended with the order-1 re-initialisation,
// formed on this RHS's state and pairs (its reverse follows k_adj_c).
template <typename R>
int adj_rhs(sph_handle* h, const Sorted<R>& V, int k, int stage, bool shift = false, bool kept = false,
            bool mls1 = false) {
    const Params& P = h->P;
    AdjCtx* X = h->adj;
    Adj& A = X->A;
    const int nb = blocks(P.n_tot, kAdjThreads);
    const int nbc = blocks((long long)P.n_tot * kAdjLanes, kAdjThreads);
    if (!shift && !kept) {
        tic(h, PH_A);
        adj_pass_a<R>(h, V);
    }
    tic(h, PH_ADJ);
    if (P.muscl)
        k_adj_c<R, false, true><<<nbc, kAdjThreads, 0, h->stream>>>(P, V, A, A.lr[k], A.la[k],
                                                                     A.nu_part + (size_t)k * nbc);
    else
        k_adj_c<R><<<nbc, kAdjThreads, 0, h->stream>>>(P, V, A, A.lr[k], A.la[k], A.nu_part + (size_t)k * nbc);
    if (shift) {
        k_adj_shift<R><<<nb, kAdjThreads, 0, h->stream>>>(P, V, A);
        h->launches += 1;
    }
    if (mls1) {
        k_adj_mls1_own<R><<<blocks(P.n_tot, 128), 128, 0, h->stream>>>(P, V, X->mls_cy);
        k_adj_mls1_nbr<R><<<blocks(P.n_tot, 128), 128, 0, h->stream>>>(P, V, A, X->mls_lam, X->mls_cy);
        h->launches += 2;
    }
    k_adj_point<R><<<blocks(P.n_tot, 256), 256, 0, h->stream>>>(P, V, A, shift ? 1 : 0);
    if (P.muscl) k_adj_a<R, false, true><<<nbc, kAdjThreads, 0, h->stream>>>(P, V, A, stage, X->dt, nullptr);
    else k_adj_a<R><<<nbc, kAdjThreads, 0, h->stream>>>(P, V, A, stage, X->dt, nullptr);
    CK(cudaGetLastError());
    h->launches += 3;
    return SPH_OK;
}

// Reverse of one time step from the staged step-start state: rebuild the
// images, the sort and the lists (the same permutation as in the forward
// run), take S1..S3 from stage slot j (or recompute them into slot 0 when
// j < 0), then run the reverse kernels from the step end to its start.
template <typename R>
int adj_step(sph_handle* h, bool first, int j) {
    AdjCtx* X = h->adj;
    Adj& A = X->A;
    const double dt = X->dt;
    int rc;
    if (j < 0) {
        if ((rc = step_keep<R>(h, dt, 0, false))) return rc;
        j = 0;
    } else {
        if ((rc = X->prep ? prep_restore(h, j, !(X->pa && X->seg_kept[j])) : prepare<R>(h))) return rc;
        if (h->P.n_tot != X->seg_ntot[j]) return SPH_E_ARG;
    }
    const Params& P = h->P;
    Sorted<R>& D = sorted<R>(h);
    const int nb = blocks(P.n_tot, 256);
    const bool shift = h->cfg.shifting != 0;
    // kept: the segment re-run left the pass-A outputs of RHS k + 1 in pass-A slot 3 j + k
    const bool kept = X->pa && X->seg_kept[j];
    auto view = [&](int k) {
        return kept ? pa_view<R>(h, stage_view<R>(h, j, k), 3 * j + k) : stage_view<R>(h, j, k);
    };
    if (shift) {
        // the step end's shift reads the last RHS's pass A (B^-1, grad rho, flags)
        // and its shifting sum: re-form them on the kept state S3 first
        const Sorted<R> V = view(2);
        if (!kept) {
            tic(h, PH_A);
            adj_pass_a<R>(h, V);
        }
        tic(h, PH_ADJ);
        k_shift_sum<R><<<nb, 256, 0, h->stream>>>(P, V, A);
        h->launches += 1;
    }
    tic(h, PH_ADJ);
    // a step that ended with the density re-initialisation (never a kept one)
    const bool mls = P.mls_order != 0 && (h->step_count + 1) % P.mls_every == 0;
    const bool mls1 = mls && P.mls_order == 1;
    if (mls1) {
        // the shift's reverse; the positions pass through to the last stage, the
        // re-initialised densities' adjoint waits for the last RHS's reverse
        k_adj_mls_end<R><<<nb, 256, 0, h->stream>>>(P, D, A, shift ? 1 : 0, X->mls_xe, X->mls_lam);
        k_adj_mls1_end<R><<<nb, 256, 0, h->stream>>>(P, D, X->mls_xe, X->mls_lam, X->mls_x, X->mls_r);
        k_adj_stage3<R><<<nb, 256, 0, h->stream>>>(P, D, A, dt, 0, X->mls_x, X->mls_r);
        h->launches += 3;
    } else if (mls) {
        // the shift's reverse, then that of the re-initialisation on the state the
        // last stage produced (stage slot state 3) over the step's lists
        const Sorted<R> V3 = stage_view<R>(h, j, 3);
        const int nbo = blocks(P.n_tot, 128);
        k_adj_mls_end<R><<<nb, 256, 0, h->stream>>>(P, D, A, shift ? 1 : 0, X->mls_xe, X->mls_lam);
        if (P.mls_order == 6) {
            k_adj_mls_own<R, 6><<<nbo, 128, 0, h->stream>>>(P, V3, X->mls_lam, X->mls_cy, X->mls_xo);
            k_adj_mls_nbr<R, 6><<<nbo, 128, 0, h->stream>>>(P, V3, X->mls_lam, X->mls_cy, X->mls_xo, X->mls_xe,
                                                             X->mls_x, X->mls_r, nullptr);
        } else {
            k_adj_mls_own<R, 3><<<nbo, 128, 0, h->stream>>>(P, V3, X->mls_lam, X->mls_cy, X->mls_xo);
            k_adj_mls_nbr<R, 3><<<nbo, 128, 0, h->stream>>>(P, V3, X->mls_lam, X->mls_cy, X->mls_xo, X->mls_xe,
                                                             X->mls_x, X->mls_r, nullptr);
        }
        k_adj_stage3<R><<<nb, 256, 0, h->stream>>>(P, D, A, dt, 0, X->mls_x, X->mls_r);
        h->launches += 4;
    } else {
        // the step end's shift reads the last RHS's flags, B^-1 and grad rho (kept:
        // from pass-A slot 3 j + 2; else the re-run above left them in the arrays)
        k_adj_stage3<R><<<nb, 256, 0, h->stream>>>(P, kept ? pa_view<R>(h, D, 3 * j + 2) : D, A, dt,
                                                     shift ? 1 : 0);
        h->launches += 1;
    }
    for (int k = 2; k >= 0; --k)
        if ((rc = adj_rhs<R>(h, view(k), k + 1, k, shift && k == 2, kept, mls1 && k == 2))) return rc;
    if (first) {
        // the fresh K1 of the first step was evaluated on the step-start state
        k_adj_load<R><<<nb, 256, 0, h->stream>>>(P, D, nullptr, nullptr);
        h->launches += 1;
        if ((rc = adj_rhs<R>(h, D, 0, -1))) return rc;
    }
    tic(h, PH_ADJ);
    const int nba = blocks((long long)P.n_tot * kAdjLanes, kAdjThreads);
    k_adj_nu_sum<<<1, 1024, 0, h->stream>>>((first ? 4 : 3) * nba, A.nu_part + (first ? 0 : nba), A.nu_acc);
    k_adj_scatter<R><<<nb, 256, 0, h->stream>>>(P, D, A, first ? 1 : 0);
    h->launches += 2;
    if (h->cfg.periodic) {
        const int n_src = h->n_host + h->n_lr;
        k_adj_route<<<blocks(n_src, 256), 256, 0, h->stream>>>(n_src, n_src, h->S.tb_cnt, h->S.tb_off, A);
        k_adj_route<<<blocks(h->n_host, 256), 256, 0, h->stream>>>(h->n_host, h->n_host, h->S.lr_cnt, h->S.lr_off,
                                                                     A);
        h->launches += 2;
    }
    CK(cudaGetLastError());
    tic(h, -1);
    if (h->ev_used > 4096) timing_flush(h);
    return SPH_OK;
}

// The forward values a moving-square RHS's reverse reads, on the state V: the
// ghost assignment and pass A re-run (the same values as in the forward run),
// or, for a kept corrector RHS (kept_j >= 0), the ghosts' mass and step-start
// arrays refilled from what the segment re-run left.
template <typename R>
void adj_rhs_ms_values(sph_handle* h, const Sorted<R>& V, int kept_j) {
    const Params& P = h->P;
    AdjCtx* X = h->adj;
    const bool ghosts = P.ghost_assign && h->n_ghost > 0;
    if (kept_j >= 0) {
        if (ghosts) {
            k_ghost_refill<R><<<blocks(h->n_ghost, 256), 256, 0, h->stream>>>(V, h->d_ghost_ids, h->n_ghost);
            h->launches += 1;
        }
        return;
    }
    tic(h, PH_A);
    if (ghosts) {
        k_assign_ghosts<R><<<blocks((long long)h->n_ghost * 32, 128), 128, 0, h->stream>>>(
            P, V, h->d_ghost_ids, h->n_ghost, h->t_phys, h->body_vel[0], h->body_vel[1], h->body_acc[0],
            h->body_acc[1], X->A.gint, X->A.gsw);
        h->launches += 1;
    }
    launch_pass_a<R, false>(P, V, blocks(P.n_tot, kAdjThreads), h->stream);
    launch_surface<R>(P, V, h->stream);
}

// Reverse of one moving-square RHS evaluation on the state V with the rate
// adjoints of RHS k of the step (0: the predictor's K1, 1: the corrector's):
// the forward values first (adj_rhs_ms_values, unless pre: adj_step_ms formed
// them before the step end's reverse), then the reverse of pass C (and of the
// step's drag term), of the shifting sums (shift: the corrector RHS of a step
// with particle shifting, whose step-end reverse left smu / shgr / shbi), the
// ghosts' density and mass adjoints through the step's density
// re-initialisation (gm, when it ran), the reverse of the per-particle end of
// pass A, of its pair sums and XSPH velocity, of the ghost assignment, and of
// the predictor (pred = 1) or the step-start accumulation.  The body-motion
// adjoints of the RHS go to g_motion[4 jstep ..].
template <typename R>
int adj_rhs_ms(sph_handle* h, const Sorted<R>& V, int k, int pred, bool drag, int jstep, int kept_j = -1,
               bool pre = false, bool shift = false, const double2* gm = nullptr, bool mls1 = false) {
    const Params& P = h->P;
    AdjCtx* X = h->adj;
    Adj A = X->A;
    const int nb = blocks(P.n_tot, kAdjThreads);
    const int nbc = blocks((long long)P.n_tot * kAdjLanes, kAdjThreads);
    const bool ghosts = P.ghost_assign && h->n_ghost > 0;
    if (kept_j >= 0) {
        // the segment re-run left this RHS's assigned ghosts in the stage slot and
        // its interpolation sums and pass-A outputs in pass-A slot kept_j (V)
        const size_t o = (size_t)kept_j * X->cap_tot;
        A.gint = X->pa_gint + o;
        A.gsw = X->pa_gsw + o;
    }
    if (!pre) adj_rhs_ms_values<R>(h, V, kept_j);
    tic(h, PH_ADJ);
    CK(cudaMemsetAsync(V.nflag, 0, (size_t)P.n_tot, h->stream));
    if (P.hllc)
        k_adj_c<R, true, false, true><<<nbc, kAdjThreads, 0, h->stream>>>(P, V, A, A.lr[k], A.la[k],
                                                                          A.nu_part + (size_t)k * nbc);
    else
        k_adj_c<R, true><<<nbc, kAdjThreads, 0, h->stream>>>(P, V, A, A.lr[k], A.la[k], A.nu_part + (size_t)k * nbc);
    if (shift) {
        k_adj_shift<R><<<nb, kAdjThreads, 0, h->stream>>>(P, V, A);
        h->launches += 1;
    }
    if (gm) {
        k_adj_add_ghost_rm<R><<<blocks(P.n_tot, 256), 256, 0, h->stream>>>(P, V, A, gm);
        h->launches += 1;
    }
    if (mls1) {
        k_adj_mls1_own<R><<<blocks(P.n_tot, 128), 128, 0, h->stream>>>(P, V, X->mls_cy);
        k_adj_mls1_nbr<R><<<blocks(P.n_tot, 128), 128, 0, h->stream>>>(P, V, A, X->mls_lam, X->mls_cy);
        h->launches += 2;
    }
    if (drag) {
        double* part = A.nu_part + (size_t)4 * nbc;
        k_mark_body_nbrs<R><<<blocks(P.n_tot, 256), 256, 0, h->stream>>>(P, V);
        k_adj_drag<R><<<nb, kAdjThreads, 0, h->stream>>>(P, V, A, X->dloss * X->dt, part);
        k_adj_nu_sum<<<1, 1024, 0, h->stream>>>(nb, part, A.nu_acc);
        h->launches += 3;
    }
    k_adj_point<R><<<blocks(P.n_tot, 256), 256, 0, h->stream>>>(P, V, A, shift ? 1 : 0);
    k_adj_a<R, true><<<nbc, kAdjThreads, 0, h->stream>>>(P, V, A, 0, X->dt, A.lg[k]);
    if (ghosts) {
        const int ngb = blocks((long long)h->n_ghost * 32, kAdjThreads);
        k_adj_ghost_lambda<R><<<ngb, kAdjThreads, 0, h->stream>>>(P, V, A, h->d_ghost_ids, h->n_ghost, h->t_phys,
                                                                  h->body_acc[0], h->body_acc[1], A.mo_part);
        k_adj_motion_sum<<<1, 1024, 0, h->stream>>>(ngb, 4, A.mo_part, 1.0, A.g_motion + 4 * (size_t)jstep);
        k_adj_ghost_water<R><<<148 * 8, kAdjThreads, 0, h->stream>>>(P, V, A, h->body_acc[0], h->body_acc[1]);
        h->launches += 3;
    }
    k_adj_stage_ms<R><<<blocks(P.n_tot, 256), 256, 0, h->stream>>>(P, V, A, pred, X->dt);
    CK(cudaGetLastError());
    h->launches += 5;
    return SPH_OK;
}

// Reverse of one Euler predictor-corrector step (moving square) from the staged
// step-start state (body not yet moved): the step's start (time, body motion,
// translation) and sort are redone, the predicted state comes from stage slot j
// (or is recomputed into slot 0 when j < 0).  jstep: the step's index in the
// adjoint run.
template <typename R>
int adj_step_ms(sph_handle* h, bool first, int j, int jstep) {
    AdjCtx* X = h->adj;
    Adj& A = X->A;
    const double dt = X->dt;
    int rc;
    if (j < 0) {
        if ((rc = step_keep<R>(h, dt, 0, false))) return rc;
        j = 0;
    } else {
        const bool lists = !(X->pa && X->seg_kept[j]);
        if ((rc = step_begin<R>(h, dt)) || (rc = X->prep ? prep_restore(h, j, lists) : prepare<R>(h))) return rc;
        if (h->P.n_tot != X->seg_ntot[j]) return SPH_E_ARG;
    }
    const Params& P = h->P;
    Sorted<R>& D = sorted<R>(h);
    const int nb = blocks(P.n_tot, 256);
    const bool kept = X->pa && X->seg_kept[j];
    const Sorted<R> V = kept ? pa_view<R>(h, stage_view<R>(h, j, 0), j) : stage_view<R>(h, j, 0);
    const bool shift = h->cfg.shifting != 0;
    // a step that ended with the density re-initialisation (never a kept one)
    const bool mls = P.mls_order != 0 && (h->step_count + 1) % P.mls_every == 0;
    const bool pre = shift || mls;
    if (pre) {
        // the step end's shift reads the corrector RHS's pass A (B^-1, grad rho,
        // flags) and its shifting sum over the assigned ghosts, the
        // re-initialisation the ghosts' mass as that RHS assigned it: re-form them
        // first
        adj_rhs_ms_values<R>(h, V, kept ? j : -1);
        tic(h, PH_ADJ);
        if (shift) {
            k_shift_sum<R><<<nb, 256, 0, h->stream>>>(P, V, A);
            h->launches += 1;
        }
    }
    tic(h, PH_ADJ);
    const bool mls1 = mls && P.mls_order == 1;
    if (mls1) {
        // as in adj_step: the densities' adjoint goes to the corrector RHS's reverse
        k_adj_mls_end<R><<<nb, 256, 0, h->stream>>>(P, D, A, shift ? 1 : 0, X->mls_xe, X->mls_lam);
        k_adj_mls1_end<R><<<nb, 256, 0, h->stream>>>(P, D, X->mls_xe, X->mls_lam, X->mls_x, X->mls_r);
        k_adj_stage_end_ms<R><<<nb, 256, 0, h->stream>>>(P, D, A, dt, 0, X->mls_x, X->mls_r);
        h->launches += 3;
    } else if (mls) {
        // the shift's reverse, then that of the re-initialisation on the corrected
        // state (stage slot state 3) over the step's lists
        const Sorted<R> V3 = stage_view<R>(h, j, 3);
        const int nbo = blocks(P.n_tot, 128);
        k_adj_mls_end<R><<<nb, 256, 0, h->stream>>>(P, D, A, shift ? 1 : 0, X->mls_xe, X->mls_lam);
        if (P.mls_order == 6) {
            k_adj_mls_own<R, 6><<<nbo, 128, 0, h->stream>>>(P, V3, X->mls_lam, X->mls_cy, X->mls_xo);
            k_adj_mls_nbr<R, 6><<<nbo, 128, 0, h->stream>>>(P, V3, X->mls_lam, X->mls_cy, X->mls_xo, X->mls_xe,
                                                             X->mls_x, X->mls_r, X->mls_gm);
        } else {
            k_adj_mls_own<R, 3><<<nbo, 128, 0, h->stream>>>(P, V3, X->mls_lam, X->mls_cy, X->mls_xo);
            k_adj_mls_nbr<R, 3><<<nbo, 128, 0, h->stream>>>(P, V3, X->mls_lam, X->mls_cy, X->mls_xo, X->mls_xe,
                                                             X->mls_x, X->mls_r, X->mls_gm);
        }
        k_adj_stage_end_ms<R><<<nb, 256, 0, h->stream>>>(P, D, A, dt, 0, X->mls_x, X->mls_r);
        h->launches += 4;
    } else {
        k_adj_stage_end_ms<R><<<nb, 256, 0, h->stream>>>(P, shift && kept ? pa_view<R>(h, D, j) : D, A, dt,
                                                          shift ? 1 : 0);
        h->launches += 1;
    }
    if ((rc = adj_rhs_ms<R>(h, V, 1, 1, X->loss == SPH_LOSS_DRAG, jstep, kept ? j : -1, pre, shift,
                            mls && !mls1 ? X->mls_gm : nullptr, mls1)))
        return rc;
    if (first) {
        // the fresh K1 of the first step was evaluated on the step-start state
        k_adj_load<R><<<nb, 256, 0, h->stream>>>(P, D, nullptr, nullptr);
        h->launches += 1;
        if ((rc = adj_rhs_ms<R>(h, D, 0, 0, false, jstep))) return rc;
    }
    tic(h, PH_ADJ);
    const int nba = blocks((long long)P.n_tot * kAdjLanes, kAdjThreads);
    k_adj_nu_sum<<<1, 1024, 0, h->stream>>>((first ? 2 : 1) * nba, A.nu_part + (first ? 0 : nba), A.nu_acc);
    // with library ghost assignment the body moved by u_body dt at the step start:
    // dL/du_body += dt sum_body dL/dx
    if (P.ghost_assign) {
        k_adj_body_pos<R><<<nb, 256, 0, h->stream>>>(P, D, A, A.mo_part);
        k_adj_motion_sum<<<1, 1024, 0, h->stream>>>(nb, 2, A.mo_part, dt, A.g_motion + 4 * (size_t)jstep);
        h->launches += 2;
    }
    k_adj_scatter<R><<<nb, 256, 0, h->stream>>>(P, D, A, first ? 1 : 0);
    h->launches += 2;
    CK(cudaGetLastError());
    tic(h, -1);
    if (h->ev_used > 4096) timing_flush(h);
    return SPH_OK;
}

template <typename R>
int adjoint_backward(sph_handle* h, double dloss, double* g_vel0, double* g_rho0, double* g_pos0,
                     double* g_params) {
    AdjCtx* X = h->adj;
    if (!X || !X->valid || X->n_host != h->n_host) return SPH_E_ARG;
    Adj& A = X->A;
    const int n = h->n_host;
    const bool stored = X->stage_slots >= X->every;
    int rc;
    X->dloss = dloss;
    X->have_grad = false;
    SchedGuard guard{h};
    if (!X->motion.empty()) {
        h->sched = X->motion.data(); h->sched_step0 = X->step0; h->sched_n = X->nsteps;
    }
    const bool ms = h->P.ms != 0;
    if (ms) CK(cudaMemsetAsync(A.g_motion, 0, sizeof(double) * 4 * (size_t)X->nsteps, h->stream));
    // seed from the final state
    if ((rc = unsort<R>(h)) || (rc = snap_io(h, X->ck, X->nseg, n, false))) return rc;
    k_adj_seed<<<blocks(n, 256), 256, 0, h->stream>>>(n, X->loss, dloss, h->S.type, h->S.vel, h->S.mass, X->target,
                                                     A);
    h->launches += 1;
    CK(cudaMemsetAsync(A.nu_acc, 0, sizeof(double), h->stream));
    for (int c = X->nseg - 1; c >= 0; --c) {
        const int s0 = c * X->every, s1 = std::min(s0 + X->every, X->nsteps);
        // re-run the segment from its checkpoint, keeping every step-start state
        // (and the stage states when they fit)
        if ((rc = snap_io(h, X->ck, c, n, false))) return rc;
        h->step_count = X->step0 + s0;
        h->t_phys = X->t0 + s0 * X->dt;
        for (int j = s0; j < s1; ++j) {
            if ((rc = unsort<R>(h)) || (rc = snap_io(h, X->seg, j - s0, n, true))) return rc;
            if (stored) rc = step_keep<R>(h, X->dt, j - s0, j + 1 < s1);
            else if (j + 1 < s1) rc = run_steps<R>(h, 1, X->dt);
            if (rc) return rc;
        }
        for (int j = s1 - 1; j >= s0; --j) {
            if ((rc = snap_io(h, X->seg, j - s0, n, false))) return rc;
            h->step_count = X->step0 + j;
            h->t_phys = X->t0 + j * X->dt;
            if (ms) rc = adj_step_ms<R>(h, X->step0 + j == 0, stored ? j - s0 : -1, j);
            else rc = adj_step<R>(h, X->step0 + j == 0, stored ? j - s0 : -1);
            if (rc) return rc;
        }
    }
    timing_flush(h);
    if ((rc = read_status(h))) return rc;
    // gradients with respect to the state the forward started from (id order)
    if (g_vel0) {
        k_deinterleave<<<blocks(n, 256), 256, 0, h->stream>>>(n, A.lv, h->d_xfer);
        CK(cudaMemcpyAsync(g_vel0, h->d_xfer, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    if (g_pos0) {
        k_deinterleave<<<blocks(n, 256), 256, 0, h->stream>>>(n, A.lx, h->d_xfer);
        CK(cudaMemcpyAsync(g_pos0, h->d_xfer, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    if (g_rho0) CK(cudaMemcpyAsync(g_rho0, A.lrho, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    if (g_params) CK(cudaMemcpyAsync(g_params, A.nu_acc, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    // the handle continues from the forward's final state
    if ((rc = snap_io(h, X->ck, X->nseg, n, false))) return rc;
    h->step_count = X->step0 + X->nsteps;
    h->t_phys = X->t0 + X->nsteps * X->dt;
    if (!X->motion.empty()) {
        const double* m = X->motion.data() + 4 * (size_t)(X->nsteps - 1);
        h->body_vel[0] = m[0]; h->body_vel[1] = m[1]; h->body_acc[0] = m[2]; h->body_acc[1] = m[3];
    }
    h->have_rhs = false;
    X->have_grad = true;
    return SPH_OK;
}

// Dispatch on the pair precision of the handle.
#define DISPATCH(h, fn, ...) ((h)->mixed ? fn<float>(__VA_ARGS__) : fn<double>(__VA_ARGS__))

void destroy(sph_handle* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_sorted(h->D64);
    free_sorted(h->D32);
    if (h->adj) { adj_free_all(h->adj); delete h->adj; }
    void* ptrs[] = {h->S.pos, h->S.vel, h->S.rho, h->S.mass, h->S.smass, h->S.type, h->S.itype, h->S.blabel, h->d_bf,
                    h->S.r_drho, h->S.r_acc,
                    h->S.r_avg, h->S.cnt, h->S.off, h->S.lr_cnt, h->S.lr_off, h->S.tb_cnt, h->S.tb_off, h->keys_in, h->keys_out, h->vals_in, h->vals_out, h->cub_tmp,
                    h->d_status, h->d_int, h->d_part, h->d_diag, h->d_xfer, h->d_export, h->d_off64, h->d_cnt_id,
                    h->d_mls, h->d_ghost_ids};
    for (void* p : ptrs) if (p) cudaFree(p);
    for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
    if (h->copy_stream) { cudaStreamSynchronize(h->copy_stream); cudaStreamDestroy(h->copy_stream); }
    if (h->snap_ready) cudaEventDestroy(h->snap_ready);
    if (h->snap_done) cudaEventDestroy(h->snap_done);
    if (h->d_snap) cudaFree(h->d_snap);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

int init_impl(const sph_config* cfg, int n_capacity, sph_handle** out) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return SPH_E_NODEVICE;
    sph_handle* h = new (std::nothrow) sph_handle();
    if (!h) return SPH_E_CAPACITY;
    h->cfg = *cfg;
    int rc = derive_params(*cfg, h->P);
    if (rc) { delete h; return rc; }
    CK(cudaGetDevice(&h->device));
    h->mixed = cfg->precision == SPH_PREC_MIXED;
    h->cap_host = n_capacity;
    // periodic image capacity: the edge bands, 1.5x the uniform-density estimate
    if (cfg->periodic) {
        const double fx = h->P.band / (cfg->box_hi[0] - cfg->box_lo[0]);
        const double fy = h->P.band / (cfg->box_hi[1] - cfg->box_lo[1]);
        const double est = (double)n_capacity * (2 * fx + 2 * fy + 4 * fx * fy);
        h->cap_img = (int)(1.5 * est) + 256;
    }
    h->cap_tot = h->cap_host + h->cap_img;
    const int cap = h->cap_tot;
    h->ncells = h->P.gnx * h->P.gny;
    h->key_bits = 1;
    while ((1LL << h->key_bits) <= (long long)h->ncells) h->key_bits++;
    h->dead_key = (unsigned)((1ULL << h->key_bits) - 1);
    h->P.nbr_stride = cap;
    CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&h->snap_ready, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&h->snap_done, cudaEventDisableTiming));
    // staging
    CK(dalloc(&h->S.pos, cap)); CK(dalloc(&h->S.vel, cap)); CK(dalloc(&h->S.rho, cap));
    CK(dalloc(&h->S.mass, cap)); CK(dalloc(&h->S.smass, cap)); CK(dalloc(&h->S.type, cap));
    CK(dalloc(&h->S.itype, cap));
    CK(dalloc(&h->S.blabel, cap)); CK(cudaMemset(h->S.blabel, 0, sizeof(int) * (size_t)cap));
    CK(dalloc(&h->d_bf, (size_t)6 * blocks(cap, kRedThreads) + 6));
    CK(dalloc(&h->S.r_drho, h->cap_host)); CK(dalloc(&h->S.r_acc, h->cap_host)); CK(dalloc(&h->S.r_avg, h->cap_host));
    CK(dalloc(&h->S.cnt, cap)); CK(dalloc(&h->S.off, cap));
    CK(dalloc(&h->S.lr_cnt, cap)); CK(dalloc(&h->S.lr_off, cap));
    CK(dalloc(&h->S.tb_cnt, cap)); CK(dalloc(&h->S.tb_off, cap));
    // sort
    CK(dalloc(&h->keys_in, cap)); CK(dalloc(&h->keys_out, cap));
    CK(dalloc(&h->vals_in, cap)); CK(dalloc(&h->vals_out, cap));
    {
        size_t b1 = 0, b2 = 0, b3 = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, b1, h->keys_in, h->keys_out, h->vals_in, h->vals_out, cap, 0,
                                        h->key_bits, h->stream);
        cub::DeviceScan::ExclusiveSum(nullptr, b2, h->S.cnt, h->S.off, cap, h->stream);
        long long* dummy = nullptr;
        cub::DeviceScan::ExclusiveSum(nullptr, b3, dummy, dummy, cap, h->stream);
        h->cub_bytes = std::max(b1, std::max(b2, b3)) + 1024;
        CK(cudaMalloc(&h->cub_tmp, h->cub_bytes));
    }
    CK(dalloc(&h->d_status, 1)); CK(cudaMemset(h->d_status, 0, sizeof(unsigned)));
    CK(dalloc(&h->d_int, 4));
    CK(dalloc(&h->d_part, 2 * 148 * 4)); CK(dalloc(&h->d_diag, 2));
    CK(dalloc(&h->d_xfer, (size_t)6 * h->cap_host));
    if (cfg->mls_order) CK(dalloc(&h->d_mls, cap));
    if (h->mixed) rc = alloc_sorted(h->D32, cap, h->P.max_nbr, h->ncells);
    else rc = alloc_sorted(h->D64, cap, h->P.max_nbr, h->ncells);
    if (rc) { destroy(h); return rc; }
    *out = h;
    return SPH_OK;
}

template <typename R>
int get_state_impl(sph_handle* h, int n, double* pos, double* vel, double* rho, double* press) {
    int rc = unsort<R>(h);
    if (rc) return rc;
    // one pass packs x, v (column-major), rho and the pressure (status_equation
    // on the device) into the transfer buffer; the requested blocks are then
    // copied back with a single wait at the end
    k_snapshot<<<blocks(n, 256), 256, 0, h->stream>>>(h->P, n, h->S.pos, h->S.vel, h->S.rho, h->d_xfer);
    CK(cudaGetLastError());
    h->launches += 1;
    const size_t nn = (size_t)n;
    if (pos) CK(cudaMemcpyAsync(pos, h->d_xfer, sizeof(double) * 2 * nn, cudaMemcpyDeviceToHost, h->stream));
    if (vel) CK(cudaMemcpyAsync(vel, h->d_xfer + 2 * nn, sizeof(double) * 2 * nn, cudaMemcpyDeviceToHost, h->stream));
    if (rho) CK(cudaMemcpyAsync(rho, h->d_xfer + 4 * nn, sizeof(double) * nn, cudaMemcpyDeviceToHost, h->stream));
    if (press) CK(cudaMemcpyAsync(press, h->d_xfer + 5 * nn, sizeof(double) * nn, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return SPH_OK;
}

}  // namespace

// The configuration-to-parameter mapping, shared with sph_noalloc.cu.
namespace sph {
int derive_params_shared(const sph_config& c, Params& P) { return derive_params(c, P); }
}  // namespace sph

// ===========================================================================
// C-ABI
// ===========================================================================
extern "C" {

const char* sph_strerror(int code) {
    int k = -code;
    if (k < 0 || k >= (int)(sizeof(kMessages) / sizeof(kMessages[0]))) return "unknown status";
    return kMessages[k];
}

int sph_init(const sph_config* cfg, int n_capacity, sph_handle** out) {
    if (!cfg || !out || n_capacity <= 0) return SPH_E_ARG;
    *out = nullptr;
    return init_impl(cfg, n_capacity, out);
}

int sph_free(sph_handle* h) {
    if (!h) return SPH_E_ARG;
    destroy(h);
    return SPH_OK;
}

int sph_set_state(sph_handle* h, int n, const double* pos, const double* vel, const double* rho,
                  const double* mass, const int* type, const double* sps_mass) {
    if (!h || !pos || !vel || !rho || !mass || !type || n <= 0) return SPH_E_ARG;
    if (n > h->cap_host) return SPH_E_CAPACITY;
    CK(cudaSetDevice(h->device));
    h->n_host = n;
    CK(cudaMemcpyAsync(h->d_xfer, pos, sizeof(double) * 2 * n, cudaMemcpyHostToDevice, h->stream));
    k_interleave<<<blocks(n, 256), 256, 0, h->stream>>>(n, h->d_xfer, h->S.pos);
    CK(cudaMemcpyAsync(h->d_xfer + 2 * (size_t)n, vel, sizeof(double) * 2 * n, cudaMemcpyHostToDevice, h->stream));
    k_interleave<<<blocks(n, 256), 256, 0, h->stream>>>(n, h->d_xfer + 2 * (size_t)n, h->S.vel);
    CK(cudaMemcpyAsync(h->S.rho, rho, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->S.mass, mass, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->S.smass, sps_mass ? sps_mass : mass, sizeof(double) * n, cudaMemcpyHostToDevice,
                       h->stream));
    CK(cudaMemcpyAsync(h->S.type, type, sizeof(int) * n, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->S.itype, type, sizeof(int) * n, cudaMemcpyHostToDevice, h->stream));
    {
        // the ghost assignment works one warp per ghost over this list
        std::vector<int> g;
        for (int i = 0; i < n; ++i)
            if (type[i] == SPH_TYPE_FIX_GHOST) g.push_back(i);
        if (!h->d_ghost_ids) CK(dalloc(&h->d_ghost_ids, h->cap_host));
        h->n_ghost = (int)g.size();
        if (!g.empty())
            CK(cudaMemcpyAsync(h->d_ghost_ids, g.data(), sizeof(int) * g.size(), cudaMemcpyHostToDevice, h->stream));
    }
    h->P.has_body = 0;
    for (int c = 0; c < 6; ++c) h->bf[c] = 0.0;
    h->bf_pending = false;
    CK(cudaMemsetAsync(h->S.r_drho, 0, sizeof(double) * n, h->stream));
    CK(cudaMemsetAsync(h->S.r_acc, 0, sizeof(double2) * n, h->stream));
    CK(cudaMemsetAsync(h->S.r_avg, 0, sizeof(double2) * n, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->staging_valid = true;
    h->sorted_valid = false;
    h->have_rhs = false;
    h->step_count = 0;
    h->t_phys = 0.0;
    CK(cudaMemsetAsync(h->S.blabel, 0, sizeof(int) * (size_t)n, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return SPH_OK;
}

int sph_update_state(sph_handle* h, int n, const double* pos, const double* vel, const double* rho) {
    if (!h || n != h->n_host || n <= 0 || !pos || !vel || !rho) return SPH_E_ARG;
    CK(cudaSetDevice(h->device));
    int rc = h->mixed ? unsort<float>(h) : unsort<double>(h);
    if (rc) return rc;
    CK(cudaMemcpyAsync(h->d_xfer, pos, sizeof(double) * 2 * n, cudaMemcpyHostToDevice, h->stream));
    k_interleave<<<blocks(n, 256), 256, 0, h->stream>>>(n, h->d_xfer, h->S.pos);
    CK(cudaMemcpyAsync(h->d_xfer + 2 * (size_t)n, vel, sizeof(double) * 2 * n, cudaMemcpyHostToDevice, h->stream));
    k_interleave<<<blocks(n, 256), 256, 0, h->stream>>>(n, h->d_xfer + 2 * (size_t)n, h->S.vel);
    CK(cudaMemcpyAsync(h->S.rho, rho, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    CK(cudaGetLastError());
    // the copies from page-locked buffers run asynchronously: finish them before
    // returning, since the caller owns (and may refill) its arrays afterwards
    CK(cudaStreamSynchronize(h->stream));
    h->launches += 2;
    h->staging_valid = true;
    h->sorted_valid = false;
    return SPH_OK;
}

int sph_set_initial_type(sph_handle* h, int n, const int* initial_type) {
    if (!h || n != h->n_host || n <= 0 || !initial_type) return SPH_E_ARG;
    CK(cudaSetDevice(h->device));
    int rc = h->mixed ? unsort<float>(h) : unsort<double>(h);
    if (rc) return rc;
    CK(cudaMemcpyAsync(h->S.itype, initial_type, sizeof(int) * n, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    int body = 0;
    for (int i = 0; i < n; ++i) body |= initial_type[i] == SPH_TYPE_BODY;
    h->P.has_body = body;
    h->sorted_valid = false;
    return SPH_OK;
}

int sph_set_boundary_labels(sph_handle* h, int n, const int* labels) {
    if (!h || n != h->n_host || n <= 0 || !labels) return SPH_E_ARG;
    CK(cudaSetDevice(h->device));
    int rc = h->mixed ? unsort<float>(h) : unsort<double>(h);
    if (rc) return rc;
    CK(cudaMemcpyAsync(h->S.blabel, labels, sizeof(int) * n, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->sorted_valid = false;
    return SPH_OK;
}

int sph_set_body_motion(sph_handle* h, const double vel[2], const double acc[2]) {
    if (!h || !vel || !acc) return SPH_E_ARG;
    for (int k = 0; k < 2; ++k) { h->body_vel[k] = vel[k]; h->body_acc[k] = acc[k]; }
    return SPH_OK;
}

int sph_set_time(sph_handle* h, double t) {
    if (!h) return SPH_E_ARG;
    h->t_phys = t;
    return SPH_OK;
}

int sph_snapshot_wait(sph_handle* h) {
    if (!h) return SPH_E_ARG;
    if (h->snap_pending) {
        CK(cudaSetDevice(h->device));
        CK(cudaEventSynchronize(h->snap_done));
        h->snap_pending = false;
    }
    return SPH_OK;
}

int sph_snapshot_query(sph_handle* h) {
    if (!h) return SPH_E_ARG;
    if (!h->snap_pending) return SPH_OK;
    CK(cudaSetDevice(h->device));
    const cudaError_t e = cudaEventQuery(h->snap_done);
    if (e == cudaErrorNotReady) return SPH_PENDING;
    CK(e);
    h->snap_pending = false;
    return SPH_OK;
}

int sph_snapshot_begin(sph_handle* h, int n, double* pos, double* vel, double* rho, double* press) {
    if (!h || n != h->n_host || n <= 0) return SPH_E_ARG;
    int rc = sph_snapshot_wait(h);               // the device buffer is reused
    if (rc) return rc;
    CK(cudaSetDevice(h->device));
    if (!h->d_snap) CK(dalloc(&h->d_snap, (size_t)6 * h->cap_host));
    rc = h->mixed ? unsort<float>(h) : unsort<double>(h);
    if (rc) return rc;
    k_snapshot<<<blocks(n, 256), 256, 0, h->stream>>>(h->P, n, h->S.pos, h->S.vel, h->S.rho, h->d_snap);
    CK(cudaGetLastError());
    h->launches += 1;
    CK(cudaEventRecord(h->snap_ready, h->stream));
    CK(cudaStreamWaitEvent(h->copy_stream, h->snap_ready, 0));
    const size_t nn = (size_t)n;
    if (pos) CK(cudaMemcpyAsync(pos, h->d_snap, sizeof(double) * 2 * nn, cudaMemcpyDeviceToHost, h->copy_stream));
    if (vel)
        CK(cudaMemcpyAsync(vel, h->d_snap + 2 * nn, sizeof(double) * 2 * nn, cudaMemcpyDeviceToHost, h->copy_stream));
    if (rho) CK(cudaMemcpyAsync(rho, h->d_snap + 4 * nn, sizeof(double) * nn, cudaMemcpyDeviceToHost, h->copy_stream));
    if (press)
        CK(cudaMemcpyAsync(press, h->d_snap + 5 * nn, sizeof(double) * nn, cudaMemcpyDeviceToHost, h->copy_stream));
    CK(cudaEventRecord(h->snap_done, h->copy_stream));
    h->snap_pending = true;
    return SPH_OK;
}

namespace {
// Restart image: header, then the per-particle arrays in the order below.
struct RestartHeader {
    char magic[8];            // "SPHB200R"
    int32_t version;          // 1
    int32_t n;
    int64_t step_count;
    double t_phys;
    double body_vel[2];
    double body_acc[2];
};
static_assert(sizeof(RestartHeader) == 64, "restart header is 64 bytes");
constexpr size_t kRestartPerParticle = 2 * 16 + 3 * 8 + 3 * 4 + 8 + 2 * 16;   // 108 bytes
}  // namespace

size_t sph_restart_size(int n) {
    return n > 0 ? sizeof(RestartHeader) + kRestartPerParticle * (size_t)n : 0;
}

int sph_restart_save(sph_handle* h, void* buf, size_t bytes) {
    if (!h || !buf || h->n_host <= 0) return SPH_E_ARG;
    const int n = h->n_host;
    if (bytes < sph_restart_size(n)) return SPH_E_CAPACITY;
    CK(cudaSetDevice(h->device));
    int rc = h->mixed ? unsort<float>(h) : unsort<double>(h);
    if (rc) return rc;
    RestartHeader hd{};
    memcpy(hd.magic, "SPHB200R", 8);
    hd.version = 1;
    hd.n = n;
    hd.step_count = h->step_count;
    hd.t_phys = h->t_phys;
    for (int k = 0; k < 2; ++k) { hd.body_vel[k] = h->body_vel[k]; hd.body_acc[k] = h->body_acc[k]; }
    char* p = static_cast<char*>(buf);
    memcpy(p, &hd, sizeof(hd));
    p += sizeof(hd);
    const size_t nn = (size_t)n;
    auto get = [&](const void* src, size_t each) -> int {
        CK(cudaMemcpyAsync(p, src, each * nn, cudaMemcpyDeviceToHost, h->stream));
        p += each * nn;
        return SPH_OK;
    };
    if ((rc = get(h->S.pos, 16)) || (rc = get(h->S.vel, 16)) || (rc = get(h->S.rho, 8)) || (rc = get(h->S.mass, 8)) ||
        (rc = get(h->S.smass, 8)) || (rc = get(h->S.type, 4)) || (rc = get(h->S.itype, 4)) ||
        (rc = get(h->S.blabel, 4)) || (rc = get(h->S.r_drho, 8)) || (rc = get(h->S.r_acc, 16)) ||
        (rc = get(h->S.r_avg, 16)))
        return rc;
    CK(cudaStreamSynchronize(h->stream));
    return SPH_OK;
}

int sph_restart_load(sph_handle* h, const void* buf, size_t bytes) {
    if (!h || !buf || bytes < sizeof(RestartHeader)) return SPH_E_ARG;
    RestartHeader hd;
    memcpy(&hd, buf, sizeof(hd));
    if (memcmp(hd.magic, "SPHB200R", 8) != 0 || hd.version != 1 || hd.n <= 0) return SPH_E_ARG;
    const int n = hd.n;
    if (bytes < sph_restart_size(n)) return SPH_E_ARG;
    if (n > h->cap_host) return SPH_E_CAPACITY;
    CK(cudaSetDevice(h->device));
    int rc = sph_snapshot_wait(h);
    if (rc) return rc;
    const char* p = static_cast<const char*>(buf) + sizeof(hd);
    const size_t nn = (size_t)n;
    // host-side views of the arrays the host bookkeeping needs
    const int* type = reinterpret_cast<const int*>(p + (2 * 16 + 3 * 8) * nn);
    const int* itype = type + nn;
    const int* labels = itype + nn;
    for (size_t i = 0; i < nn; ++i)
        if (labels[i] == -9) return SPH_E_CONFIG;     // radius free slip: not built
    auto put = [&](void* dst, size_t each) -> int {
        CK(cudaMemcpyAsync(dst, p, each * nn, cudaMemcpyHostToDevice, h->stream));
        p += each * nn;
        return SPH_OK;
    };
    if ((rc = put(h->S.pos, 16)) || (rc = put(h->S.vel, 16)) || (rc = put(h->S.rho, 8)) || (rc = put(h->S.mass, 8)) ||
        (rc = put(h->S.smass, 8)) || (rc = put(h->S.type, 4)) || (rc = put(h->S.itype, 4)) ||
        (rc = put(h->S.blabel, 4)) || (rc = put(h->S.r_drho, 8)) || (rc = put(h->S.r_acc, 16)) ||
        (rc = put(h->S.r_avg, 16)))
        return rc;
    std::vector<int> g;
    int body = 0;
    for (size_t i = 0; i < nn; ++i) {
        if (type[i] == SPH_TYPE_FIX_GHOST) g.push_back((int)i);
        body |= itype[i] == SPH_TYPE_BODY;
    }
    if (!h->d_ghost_ids) CK(dalloc(&h->d_ghost_ids, h->cap_host));
    h->n_ghost = (int)g.size();
    if (!g.empty())
        CK(cudaMemcpyAsync(h->d_ghost_ids, g.data(), sizeof(int) * g.size(), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->n_host = n;
    h->P.has_body = body;
    for (int c = 0; c < 6; ++c) h->bf[c] = 0.0;
    h->bf_pending = false;
    h->staging_valid = true;
    h->sorted_valid = false;
    h->have_rhs = false;
    h->step_count = hd.step_count;
    h->t_phys = hd.t_phys;
    for (int k = 0; k < 2; ++k) { h->body_vel[k] = hd.body_vel[k]; h->body_acc[k] = hd.body_acc[k]; }
    return SPH_OK;
}

int sph_get_state(sph_handle* h, int n, double* pos, double* vel, double* rho, double* press) {
    if (!h || n != h->n_host || n <= 0) return SPH_E_ARG;
    CK(cudaSetDevice(h->device));
    return DISPATCH(h, get_state_impl, h, n, pos, vel, rho, press);
}

int sph_find_particle_pair(sph_handle* h, long long pair_cap, int* pair_i, int* pair_j, double* w, double* dwdx,
                           long long* pair_number) {
    if (!h || !pair_number || h->n_host <= 0) return SPH_E_ARG;
    if (pair_cap > 0 && (!pair_i || !pair_j)) return SPH_E_ARG;
    CK(cudaSetDevice(h->device));
    int rc = DISPATCH(h, prepare, h);
    if (rc) return rc;
    rc = read_status(h);
    if (rc) return rc;
    return DISPATCH(h, find_pairs, h, pair_cap, pair_i, pair_j, w, dwdx, pair_number);
}

int sph_rhs(sph_handle* h, double* drhodt, double* acc, double* avg_vel, int* fs, int* near_fs) {
    if (!h || h->n_host <= 0) return SPH_E_ARG;
    CK(cudaSetDevice(h->device));
    int rc = DISPATCH(h, prepare, h);
    if (rc) return rc;
    h->bf_every_rhs = true;
    rc = DISPATCH(h, rhs, h, 0);
    h->bf_every_rhs = false;
    if (rc) return rc;
    timing_flush(h);
    rc = read_status(h);
    if (rc) return rc;
    rc = DISPATCH(h, export_fields, h);
    if (rc) return rc;
    const size_t n = (size_t)h->n_host;
    std::vector<double> buf(7 * n);
    CK(cudaMemcpyAsync(buf.data(), h->d_export, sizeof(double) * 7 * n, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (size_t i = 0; i < n; ++i) {
        if (drhodt) drhodt[i] = buf[i];
        if (acc) { acc[i] = buf[n + i]; acc[n + i] = buf[2 * n + i]; }
        if (avg_vel) { avg_vel[i] = buf[3 * n + i]; avg_vel[n + i] = buf[4 * n + i]; }
        if (fs) fs[i] = (int)buf[5 * n + i];
        if (near_fs) near_fs[i] = (int)buf[6 * n + i];
    }
    return SPH_OK;
}

int sph_get_field(sph_handle* h, int field, double* out) {
    if (!h || !out || !h->have_rhs) return SPH_E_ARG;
    CK(cudaSetDevice(h->device));
    int first, count;
    switch (field) {
        case SPH_FIELD_FRA_V: first = 7; count = 1; break;
        case SPH_FIELD_BINV: first = 8; count = 4; break;
        case SPH_FIELD_TAU: first = 12; count = 3; break;
        case SPH_FIELD_GRADS: first = 15; count = 8; break;
        default: return SPH_E_ARG;
    }
    int rc = DISPATCH(h, export_fields, h);
    if (rc) return rc;
    const size_t n = (size_t)h->n_host;
    CK(cudaMemcpyAsync(out, h->d_export + first * n, sizeof(double) * count * n, cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return SPH_OK;
}

int sph_step(sph_handle* h, int nsteps, double dt, sph_diag* out) {
    if (!h || nsteps < 0 || !(dt > 0) || h->n_host <= 0) return SPH_E_ARG;
    CK(cudaSetDevice(h->device));
    int rc = DISPATCH(h, run_steps, h, nsteps, dt);
    if (rc) return rc;
    if (out) return DISPATCH(h, diagnostics, h, out);
    return SPH_OK;
}

int sph_diagnostics(sph_handle* h, sph_diag* out) {
    if (!h || !out || h->n_host <= 0) return SPH_E_ARG;
    CK(cudaSetDevice(h->device));
    return DISPATCH(h, diagnostics, h, out);
}

int sph_adjoint_forward(sph_handle* h, const sph_adj_config* cfg, double* loss) {
    if (!h || !cfg || h->n_host <= 0 || cfg->nsteps <= 0 || cfg->checkpoint_every <= 0 || !(cfg->dt > 0))
        return SPH_E_ARG;
    if (cfg->loss != SPH_LOSS_VELOCITY_MISFIT && cfg->loss != SPH_LOSS_KINETIC_ENERGY && cfg->loss != SPH_LOSS_DRAG)
        return SPH_E_ARG;
    if (cfg->loss == SPH_LOSS_VELOCITY_MISFIT && !cfg->target_vel) return SPH_E_ARG;
    int rc = adj_config_ok(h, cfg->loss);
    if (rc) return rc;
    CK(cudaSetDevice(h->device));
    return DISPATCH(h, adjoint_forward, h, cfg, loss);
}

int sph_adjoint_backward(sph_handle* h, double dloss, double* g_vel0, double* g_rho0, double* g_pos0,
                         double* g_params) {
    if (!h) return SPH_E_ARG;
    CK(cudaSetDevice(h->device));
    return DISPATCH(h, adjoint_backward, h, dloss, g_vel0, g_rho0, g_pos0, g_params);
}

int sph_adjoint_motion_gradient(sph_handle* h, double* g_motion) {
    if (!h || !g_motion || !h->adj || !h->adj->have_grad) return SPH_E_ARG;
    CK(cudaSetDevice(h->device));
    AdjCtx* X = h->adj;
    const size_t bytes = sizeof(double) * 4 * (size_t)X->nsteps;
    if (!h->P.ms) {
        memset(g_motion, 0, bytes);
        return SPH_OK;
    }
    CK(cudaMemcpyAsync(g_motion, X->A.g_motion, bytes, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return SPH_OK;
}

int sph_get_timings(sph_handle* h, sph_timings* out) {
    if (!h || !out) return SPH_E_ARG;
    timing_flush(h);
    out->sort_ms = h->t_ms[PH_SORT];
    out->pass_a_ms = h->t_ms[PH_A];
    out->surface_ms = h->t_ms[PH_SURF];
    out->pass_c_ms = h->t_ms[PH_C];
    out->update_ms = h->t_ms[PH_UPDATE];
    out->images_ms = h->t_ms[PH_IMAGES];
    out->total_ms = h->t_total;
    out->rhs_evaluations = h->n_rhs;
    out->steps = h->n_steps;
    out->kernel_launches = h->launches;
    out->adjoint_ms = h->t_ms[PH_ADJ];
    return SPH_OK;
}

int sph_reset_timings(sph_handle* h) {
    if (!h) return SPH_E_ARG;
    timing_flush(h);
    for (double& t : h->t_ms) t = 0;
    h->t_total = 0;
    h->n_rhs = 0;
    h->n_steps = 0;
    h->launches = 0;
    return SPH_OK;
}

}  // extern "C"
