// common.cuh -- parameters, precision traits and small device helpers of libsph_b200.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "../../include/sph_b200.h"

namespace sph {

// Status bits set on the device (atomicOr) and turned into SPH_E_* on the host.
enum : unsigned {
    ST_DOMAIN = 1u << 0,     // particle outside the cell grid
    ST_NBR_OVERFLOW = 1u << 1,   // neighbour list capacity exceeded
    ST_SKIN = 1u << 2,       // moved further than half the list skin
    ST_NONFINITE = 1u << 3,  // NaN / Inf in the state
    ST_PAIR_OVERFLOW = 1u << 4,
};

// Everything a kernel needs, derived once on the host from sph_config.
// The default-real literals of the reference are rounded through float when
// reference_literals is set (the same rounding as ifort's default reals).
struct Params {
    // switches
    int kernel_model, solver, renorm, quirks, pair_rule, shifting, muscl, xsph;
    int dsph;                     // Solver_Normalized_Delta_SPH_SPS (Taylor-Green)
    int ms, hllc, laplacian, free_surface, integrator, has_body;
    int mls_order, mls_every;     // density re-initialisation (0: off)
    double mls_alpha3;            // alpha^3 added to the moment matrix diagonal
    // ghost assignment (moving-square driver)
    int ghost_assign, wall_bc, ghost_cells;
    double ghost_h, ghost_r, ghost_kf, shock_t, grav[2];
    // kernel / pair search
    double h, r_cut, cut_min, kfactor, gauss_e9, q_zero;
    double r2_list;          // squared neighbour-list radius (support * (1 + skin))
    float r2_list32;         // the same for the mixed path's FP32 test on the hi positions,
                             // widened to cover their rounding (a superset of the FP64 list)
    // equation of state
    double rho0, c0sq, sqrt_c0, eos_b, pb;
    int eos;
    // solver coefficients
    double nu, alpha, beta, fai, delta, delta_alpha, eps;
    double sv;               // support volume PI*(kernel_scale*h)^2
    double fs_thr, c1414, pi;
    double sps_dl, sps_c012, sps_23, sps_blin;
    // shifting
    double shift_beta, shift_R, shift_max, w_dx;
    int shift_n;
    // periodic box
    double box_lo[2], box_hi[2], band;
    // cell grid (row-major, cell edge >= list radius)
    double gx0, gy0, cs;
    int gnx, gny;
    // sizes
    int n_host, n_tot, max_nbr, nbr_stride;
    double skin_half2;       // (skin/2)^2: allowed squared displacement since the list build
};

template <typename R> struct VT;
template <> struct VT<double> { using V2 = double2; using V4 = double4; };
template <> struct VT<float> { using V2 = float2; using V4 = float4; };

template <typename R> __host__ __device__ inline typename VT<R>::V2 mk2(R a, R b);
template <> __host__ __device__ inline double2 mk2<double>(double a, double b) { return make_double2(a, b); }
template <> __host__ __device__ inline float2 mk2<float>(float a, float b) { return make_float2(a, b); }
template <typename R> __host__ __device__ inline typename VT<R>::V4 mk4(R a, R b, R c, R d);
template <> __host__ __device__ inline double4 mk4<double>(double a, double b, double c, double d) { return make_double4(a, b, c, d); }
template <> __host__ __device__ inline float4 mk4<float>(float a, float b, float c, float d) { return make_float4(a, b, c, d); }

// Particles whose rates are assembled and integrated: water; the moving-square
// driver also integrates inlet/outlet particles (Moving_Square.../Single_step_compute.f90:273,
// SPH_Time_Iteration.f90:316).
__device__ __forceinline__ bool integrated(const Params& P, int t) {
    return t == SPH_TYPE_WATER || (P.ms && t <= SPH_TYPE_INLET);
}

__device__ __forceinline__ double pw3(double x) { return x * x * x; }
__device__ __forceinline__ double pw4(double x) { double x2 = x * x; return x2 * x2; }
__device__ __forceinline__ double pw7(double x) { double x2 = x * x; double x4 = x2 * x2; return x4 * x2 * x; }
__device__ __forceinline__ float pw3(float x) { return x * x * x; }
__device__ __forceinline__ float pw4(float x) { float x2 = x * x; return x2 * x2; }

// status_equation (Taylor_Green_Vortex/status_equation.f90:60-63,
// Moving_Square.../Status_Equation.f90:56-76), always in FP64.
__device__ __forceinline__ void eos64(const Params& P, double rho, double& p, double& c) {
    double r = rho / P.rho0;
    if (P.eos == SPH_EOS_TAIT) p = P.eos_b * (pw7(r) - 1.0) + P.pb;
    else p = P.c0sq * (rho - P.rho0) + P.pb;
    c = P.sqrt_c0 * pw3(r);
}

// Exact replica of the reference's support test
//   distance = sqrt(dot(dx,dx));  distance <= kernel_scale*h  .and.  distance >= 1.0E-7
// (find_particle_pair.f90:79-87) with the products and the sum rounded
// separately (no FMA), so the pair set is bit-identical to the CPU's.
__device__ __forceinline__ bool in_support(const Params& P, double dx, double dy, double& d) {
    double s = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
    d = __dsqrt_rn(s);
    return d <= P.r_cut && d >= P.cut_min;
}

// A product rounded on its own (never fused into a following add).
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

// Plain accumulator for the FP64 path.
struct DSum {
    double s;
    __device__ __forceinline__ void init() { s = 0.0; }
    __device__ __forceinline__ void add(double x) { s += x; }
    __device__ __forceinline__ double val() const { return s; }
};

// The mixed path's sums: FP32 terms added in FP64 (one conversion and one FP64
// add per term; a compensated FP32 TwoSum takes seven FP32 operations for a
// sum of about the same accuracy).
struct WSum {
    double s;
    __device__ __forceinline__ void init() { s = 0.0; }
    __device__ __forceinline__ void add(float x) { s += (double)x; }
    __device__ __forceinline__ float val() const { return (float)s; }
};

template <typename R> struct Acc;
template <> struct Acc<double> { using T = DSum; };
template <> struct Acc<float> { using T = WSum; };

// compute_kernel for one pair: W and grad_a W(x_a - x_b) = f(d) (x_a - x_b).
// Improved Gaussian: Taylor_Green_Vortex/compute_kernel.f90:122-134.
// Wendland C2: Moving_Square.../Compute_Kernel.f90:179-193.
template <typename R>
__device__ __forceinline__ void kernel_w_dw(const Params& P, R d, R px, R py, R& w, R& gx, R& gy) {
    const R h = (R)P.h;
    const R factor = (R)P.kfactor;
    R q = d / h;
    if (P.kernel_model == SPH_KERNEL_GAUSSIAN) {
        R e = exp(-(q * q));
        w = (e - (R)P.gauss_e9) * factor;
        R g = (e * (R(-2) * q));
        R dh = d * h;
        gx = g * px / dh * factor;
        gy = g * py / dh * factor;
    } else {
        R t = R(1) - q / R(2);
        w = factor * (R(1) + R(2) * q) * pw4(t);
        R g = factor * (R(-5) * q * pw3(t));
        R dh = d * h;
        gx = g * px / dh;
        gy = g * py / dh;
    }
    if (q <= (R)P.q_zero) { gx = R(0); gy = R(0); }
}

}  // namespace sph
