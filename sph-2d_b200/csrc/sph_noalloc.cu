// sph_noalloc.cu -- find_particle_pair for callers that cannot allocate GPU memory.
//
// Some hosts cannot call cudaMalloc from the place where they need a pair
// list: a Fortran or C host whose GPU memory is owned and pooled by another
// framework, code that runs while that framework forbids allocations, or a
// deployment with a fixed memory budget.  They own the input and output
// buffers already and only need the search itself.  This entry point does the
// whole search -- cell binning, counting sort, pair counting, prefix sums and
// emission -- with all of its working memory in one file-scope __device__ array
// of fixed size (kScratchBytes, about 2.4 MiB), so it calls no cudaMalloc, no
// cudaFree and no allocating library routine.  The array is part of the loaded
// module: every GPU that loads the library holds it until the process exits.
//
// Limits: at most kMaxParticles particles and kMaxCells background cells
// (cells of edge kernel_scale * h over cfg->grid_lo .. grid_hi plus one cell
// on each side); larger inputs are rejected with SPH_E_CAPACITY.
// All calls share the one array and each call leaves its contents behind; the
// call clears what must start at zero.  Two calls whose GPU work overlaps
// (different host threads, or different streams without ordering between them)
// race on the array and give wrong results: serialise them.
// At most kMaxPairsPerParticle pairs (i, j > i) per particle: beyond that the
// call returns SPH_E_CAPACITY with *pair_number = -1 (a larger pair_cap does
// not help).
// The first call on a device resolves the array's device address with
// cudaGetSymbolAddress (the host-side symbol is only a stand-in, not a device
// address) and caches it per device; make that first call before any stream
// capture.  The cached address belongs to the device context of that first
// call: after cudaDeviceReset the module is loaded again and the cache is
// stale, so a process that resets a device must not call this entry point on
// it afterwards.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "common.cuh"

namespace sph {
int derive_params_shared(const sph_config& c, Params& P);   // sph_b200.cu
}

using namespace sph;

namespace {

constexpr int kMaxParticles = 65536;
constexpr int kMaxCells = 65536;
constexpr int kScanThreads = 1024;
constexpr int kMaxDevices = 64;
constexpr int kMaxPairsPerParticle = 256;   // pairs (i, j > i) one thread sorts by j

// scratch layout (byte offsets)
constexpr size_t kOffCellOf = 0;                                               // int[kMaxParticles]
constexpr size_t kOffCellCount = kOffCellOf + sizeof(int) * kMaxParticles;      // int[kMaxCells]
constexpr size_t kOffCellStart = kOffCellCount + sizeof(int) * kMaxCells;       // int[kMaxCells + 1]
constexpr size_t kOffFill = kOffCellStart + sizeof(int) * (kMaxCells + 256);    // int[kMaxCells]
constexpr size_t kOffSorted = kOffFill + sizeof(int) * kMaxCells;               // int[kMaxParticles]
constexpr size_t kOffPairCount = kOffSorted + sizeof(int) * kMaxParticles;      // long long[kMaxParticles]
constexpr size_t kOffPairOff = kOffPairCount + sizeof(long long) * kMaxParticles;   // long long[kMaxParticles]
constexpr size_t kOffTotals = kOffPairOff + sizeof(long long) * kMaxParticles;  // long long[4]
constexpr size_t kScratchBytes = kOffTotals + 256;

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct Scratch {
    int* cell_of;
    int* cell_count;
    int* cell_start;
    int* fill;
    int* sorted;
    long long* pair_count;
    long long* pair_off;
    long long* totals;    // [0] pairs, [1] status bits
};

Scratch carve(unsigned char* base) {
    Scratch s;
    s.cell_of = (int*)(base + kOffCellOf);
    s.cell_count = (int*)(base + kOffCellCount);
    s.cell_start = (int*)(base + kOffCellStart);
    s.fill = (int*)(base + kOffFill);
    s.sorted = (int*)(base + kOffSorted);
    s.pair_count = (long long*)(base + kOffPairCount);
    s.pair_off = (long long*)(base + kOffPairOff);
    s.totals = (long long*)(base + kOffTotals);
    return s;
}

std::mutex g_setup_mutex;
unsigned char* g_scratch_dev[kMaxDevices] = {};

// Once per device, with that device current: the device address of the array.
int scratch_address(unsigned char** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return SPH_E_NODEVICE;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_dev[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            fprintf(stderr, "libsph_b200: cudaGetSymbolAddress(g_noalloc_scratch) failed: %s\n", cudaGetErrorString(e));
            return SPH_E_CUDA;
        }
        g_scratch_dev[dev] = (unsigned char*)p;
    }
    *out = g_scratch_dev[dev];
    return SPH_OK;
}

__global__ void na_clear(Scratch s, int ncells) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells; c += gridDim.x * blockDim.x) s.cell_count[c] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) { s.totals[0] = 0; s.totals[1] = 0; }
}

// Background cell of every particle (type 120 and 0 are not binned,
// Assign_boundary_particles.f90:82), counted per cell.
__global__ void na_bin(Params P, int n, const double* pos, const int* type, Scratch s) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int t = type[i];
    s.cell_of[i] = -1;
    if (t == SPH_TYPE_ILL || t == 0) return;
    double fx = floor((pos[i] - P.gx0) / P.cs), fy = floor((pos[n + i] - P.gy0) / P.cs);
    int cx = (int)fx, cy = (int)fy;
    if (!(fx >= 0.0 && fy >= 0.0 && cx < P.gnx && cy < P.gny)) {
        atomicOr((unsigned long long*)&s.totals[1], (unsigned long long)ST_DOMAIN);
        return;
    }
    int c = cy * P.gnx + cx;
    s.cell_of[i] = c;
    atomicAdd(&s.cell_count[c], 1);
}

// Exclusive scan with one block: each thread scans a contiguous chunk.
template <typename T, typename TO>
__device__ void block_exclusive_scan(const T* in, TO* out, int n, TO* total) {
    __shared__ TO part[kScanThreads];
    const int per = (n + kScanThreads - 1) / kScanThreads;
    const int b0 = threadIdx.x * per, b1 = min(n, b0 + per);
    TO s = 0;
    for (int k = b0; k < b1; ++k) s += (TO)in[k];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int off = 1; off < kScanThreads; off <<= 1) {
        TO v = threadIdx.x >= off ? part[threadIdx.x - off] : (TO)0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    TO run = threadIdx.x == 0 ? (TO)0 : part[threadIdx.x - 1];
    for (int k = b0; k < b1; ++k) { TO v = (TO)in[k]; out[k] = run; run += v; }
    if (threadIdx.x == kScanThreads - 1 && total) *total = part[kScanThreads - 1];
}

__global__ void na_scan_cells(Scratch s, int ncells) {
    block_exclusive_scan<int, int>(s.cell_count, s.cell_start, ncells, nullptr);
    __syncthreads();
    for (int c = threadIdx.x; c < ncells; c += blockDim.x) s.fill[c] = s.cell_start[c];
    if (threadIdx.x == 0) s.cell_start[ncells] = s.cell_start[ncells - 1] + s.cell_count[ncells - 1];
}

__global__ void na_scatter(int n, Scratch s) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = s.cell_of[i];
    if (c < 0) return;
    s.sorted[atomicAdd(&s.fill[c], 1)] = i;
}

__device__ __forceinline__ bool na_pair_allowed(int rule, int ti, int tj) {
    if (rule == SPH_PAIRS_ONE_FLUID) return ti == SPH_TYPE_WATER || tj == SPH_TYPE_WATER;
    if (ti == -2 && tj == -2) return false;
    if (ti == -3 && tj == -3) return false;
    if (ti == -201 && tj == -201) return false;
    return true;
}

// Pairs (i, j > i) of particle i over its 3x3 cells (find_particle_pair.f90:64-123).
// emit == false: count; emit == true: write them sorted by j.
template <bool EMIT>
__global__ void na_pairs(Params P, int n, const double* pos, const int* type, Scratch s, long long cap, int* pi,
                         int* pj, double* w, double* dwdx) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = s.cell_of[i];
    if (c < 0) { if (!EMIT) s.pair_count[i] = 0; return; }
    const int cx = c % P.gnx, cy = c / P.gnx;
    const double xi = pos[i], yi = pos[n + i];
    const int ti = type[i];
    int js[kMaxPairsPerParticle];
    int m = 0;
    long long cnt = 0;
    for (int gy = max(cy - 1, 0); gy <= min(cy + 1, P.gny - 1); ++gy) {
        for (int gx = max(cx - 1, 0); gx <= min(cx + 1, P.gnx - 1); ++gx) {
            const int cc = gy * P.gnx + gx;
            for (int k = s.cell_start[cc]; k < s.cell_start[cc + 1]; ++k) {
                const int j = s.sorted[k];
                if (j <= i) continue;
                if (!na_pair_allowed(P.pair_rule, ti, type[j])) continue;
                double d;
                if (!in_support(P, xi - pos[j], yi - pos[n + j], d)) continue;
                ++cnt;
                if (EMIT && m < kMaxPairsPerParticle) {
                    int q = m++;
                    while (q > 0 && js[q - 1] > j) { js[q] = js[q - 1]; --q; }
                    js[q] = j;
                }
            }
        }
    }
    if (!EMIT) {
        s.pair_count[i] = cnt;
        if (cnt > kMaxPairsPerParticle) atomicOr((unsigned long long*)&s.totals[1], (unsigned long long)ST_PAIR_OVERFLOW);
        return;
    }
    long long o = s.pair_off[i];
    for (int k = 0; k < m; ++k, ++o) {
        if (o >= cap) return;
        const int j = js[k];
        const double dx = xi - pos[j], dy = yi - pos[n + j];
        double d;
        in_support(P, dx, dy, d);
        double ww, gx, gy;
        kernel_w_dw<double>(P, d, dx, dy, ww, gx, gy);
        pi[o] = i + 1;
        pj[o] = j + 1;
        if (w) w[o] = ww;
        if (dwdx) { dwdx[o] = gx; dwdx[cap + o] = gy; }
    }
}

__global__ void na_scan_pairs(int n, Scratch s) {
    block_exclusive_scan<long long, long long>(s.pair_count, s.pair_off, n, &s.totals[0]);
}

}  // namespace

extern "C" int sph_find_particle_pair_noalloc(const sph_config* cfg, int n, const double* d_pos, const int* d_type,
                                              long long pair_cap, int* d_pair_i, int* d_pair_j, double* d_w,
                                              double* d_dwdx, long long* pair_number, void* stream) {
    if (!cfg || !d_pos || !d_type || !pair_number || n <= 0) return SPH_E_ARG;
    if (pair_cap > 0 && (!d_pair_i || !d_pair_j)) return SPH_E_ARG;
    Params P;
    int rc = derive_params_shared(*cfg, P);
    if (rc) return rc;
    // cells of edge = support radius: the 3x3 stencil covers every pair
    const double cs = P.r_cut;
    P.cs = cs;
    P.gx0 = cfg->grid_lo[0] - cs;
    P.gy0 = cfg->grid_lo[1] - cs;
    P.gnx = (int)ceil((cfg->grid_hi[0] - cfg->grid_lo[0]) / cs) + 3;
    P.gny = (int)ceil((cfg->grid_hi[1] - cfg->grid_lo[1]) / cs) + 3;
    const long long ncells = (long long)P.gnx * P.gny;
    if (n > kMaxParticles || ncells > kMaxCells) {
        fprintf(stderr,
                "libsph_b200: sph_find_particle_pair_noalloc: %d particles / %lld cells exceed the static "
                "scratch limits (%d particles, %d cells)\n", n, ncells, kMaxParticles, kMaxCells);
        return SPH_E_CAPACITY;
    }
    unsigned char* base = nullptr;
    rc = scratch_address(&base);
    if (rc) return rc;
    Scratch s = carve(base);
    cudaStream_t st = (cudaStream_t)stream;
    const int nb = (n + 127) / 128;
    na_clear<<<64, 256, 0, st>>>(s, (int)ncells);
    na_bin<<<nb, 128, 0, st>>>(P, n, d_pos, d_type, s);
    na_scan_cells<<<1, kScanThreads, 0, st>>>(s, (int)ncells);
    na_scatter<<<nb, 128, 0, st>>>(n, s);
    na_pairs<false><<<nb, 128, 0, st>>>(P, n, d_pos, d_type, s, 0, nullptr, nullptr, nullptr, nullptr);
    na_scan_pairs<<<1, kScanThreads, 0, st>>>(n, s);
    // a rejected launch (an invalid stream, say) must not let the copy below
    // return the totals an earlier call left in the array
    if (cudaGetLastError() != cudaSuccess) return SPH_E_CUDA;
    long long totals[2] = {0, 0};
    if (cudaMemcpyAsync(totals, s.totals, sizeof(totals), cudaMemcpyDeviceToHost, st) != cudaSuccess) return SPH_E_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return SPH_E_CUDA;
    *pair_number = totals[0];
    if (totals[1] & ST_DOMAIN) return SPH_E_DOMAIN;
    if (totals[1] & ST_PAIR_OVERFLOW) {
        // more than kMaxPairsPerParticle pairs (i, j > i) for one particle: no
        // pair_cap helps, so the count is reported as -1
        *pair_number = -1;
        return SPH_E_CAPACITY;
    }
    if (pair_cap <= 0) return SPH_OK;       // count only, as sph_find_particle_pair
    na_pairs<true><<<nb, 128, 0, st>>>(P, n, d_pos, d_type, s, pair_cap, d_pair_i, d_pair_j, d_w, d_dwdx);
    if (cudaGetLastError() != cudaSuccess) return SPH_E_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return SPH_E_CUDA;
    return totals[0] > pair_cap ? SPH_E_CAPACITY : SPH_OK;
}
