// tdp_noalloc.cu -- electrostatic potential on a grid that allocates no
// device memory (tdp_potential_noalloc in include/tholedipole_b200.h).
//
// tdp_get_potential copies the grid and the result through device buffers it
// allocates on every call.  Some callers cannot allow that: a host program
// (an MD engine, a framework) whose pool allocator has reserved the GPU's
// memory up front and hands out every byte itself, and code that must not
// hit the implicit device synchronisation that cudaMalloc/cudaFree can cause.
// This variant takes every input and output as a device pointer the caller
// owns, and keeps its only scratch -- the per-atom-chunk partial sums of each
// grid point -- in a fixed file-scope device array.
//
// The array is TDP_NOALLOC_SCRATCH_DOUBLES doubles (8 MiB); every GPU that
// loads this library holds it until the process exits.  All calls share it,
// so calls that overlap on the GPU (on different streams, or from several
// threads) race on it and must be serialised by the caller.  Each call writes
// every scratch slot it later reads, so nothing needs clearing between calls.
//
// The array's device address is looked up once per device and kept for the
// life of the process.  A cudaDeviceReset unloads the module and invalidates
// that address, so the entry point must not be used on a device after the
// host program has reset it.
#include "tholedipole_b200.h"
#include "tdp_common.cuh"

#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

namespace {

static __device__ __align__(256) double g_potential_scratch[TDP_NOALLOC_SCRATCH_DOUBLES];

constexpr int kPtsPerBlock = 128;   // grid points (threads) per block
constexpr int kAtomStage = 128;     // atoms staged in shared memory per step
constexpr int kMaxDevices = 64;

// Device address of the scratch array, resolved once per device.
void* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;
thread_local char g_noalloc_error[256] = "";

int noalloc_fail(int code, const char* msg) {
    snprintf(g_noalloc_error, sizeof g_noalloc_error, "%s", msg);
    return code;
}

// Partial potential of one chunk of atoms at one grid point, the terms of
// calculateElectrostaticPotentialForParticleGridPoint (ReferenceTholeDipoleForce.cpp:1348-1372):
// q/r - (mu_perm + mu_ind).(r_i - g)/r^3, FP64, minimum image when periodic.
__global__ void k_potential_partial(int n, int ng, int chunk, int periodic, double bx, double by, double bz,
                                    const double* __restrict__ pos, const double* __restrict__ charge,
                                    const double* __restrict__ dip, const double* __restrict__ grid,
                                    double* __restrict__ scratch) {
    __shared__ double s_p[kAtomStage][3];
    __shared__ double s_q[kAtomStage];
    __shared__ double s_d[kAtomStage][3];
    const int g = blockIdx.x * kPtsPerBlock + threadIdx.x;
    const int a0 = blockIdx.y * chunk;
    const int a1 = min(a0 + chunk, n);
    double gx = 0.0, gy = 0.0, gz = 0.0;
    if (g < ng) {
        gx = grid[3 * g];
        gy = grid[3 * g + 1];
        gz = grid[3 * g + 2];
    }
    const double L[3] = {bx, by, bz};
    double inv[3];
    for (int k = 0; k < 3; k++) inv[k] = L[k] > 0.0 ? 1.0 / L[k] : 0.0;
    double pot = 0.0;
    for (int base = a0; base < a1; base += kAtomStage) {
        __syncthreads();
        for (int k = threadIdx.x; k < kAtomStage; k += kPtsPerBlock) {
            int i = base + k;
            if (i < a1) {
                for (int c = 0; c < 3; c++) {
                    s_p[k][c] = pos[3 * i + c];
                    s_d[k][c] = dip[3 * i + c];
                }
                s_q[k] = charge[i];
            }
        }
        __syncthreads();
        const int m = min(kAtomStage, a1 - base);
        for (int k = 0; k < m; k++) {
            double d[3] = {s_p[k][0] - gx, s_p[k][1] - gy, s_p[k][2] - gz};
            if (periodic)
                for (int c = 0; c < 3; c++)
                    if (L[c] > 0.0) d[c] = tdp::fold_d(d[c], L[c], inv[c]);
            double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            double rr1 = 1.0 / r, rr3 = rr1 * rr1 * rr1;
            double p = s_q[k] * rr1;
            p -= (s_d[k][0] * d[0] + s_d[k][1] * d[1] + s_d[k][2] * d[2]) * rr3;
            pot += p;
        }
    }
    if (g < ng) scratch[(size_t)blockIdx.y * ng + g] = pot;
}

// out[g] = sum over chunks, in chunk order (deterministic).
__global__ void k_potential_reduce(int ng, int nsplit, const double* __restrict__ scratch, double* __restrict__ out) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ng) return;
    double s = 0.0;
    for (int k = 0; k < nsplit; k++) s += scratch[(size_t)k * ng + g];
    out[g] = s;
}

}  // namespace

namespace tdp {
// Read by tdp_last_error(NULL) (tdp_capi.cu); cleared when a create fails.
__attribute__((visibility("hidden"))) const char* noalloc_error_message() { return g_noalloc_error; }
__attribute__((visibility("hidden"))) void noalloc_clear_error() { g_noalloc_error[0] = '\0'; }
}  // namespace tdp

extern "C" int tdp_potential_noalloc(int32_t num_particles, const double* positions, const double* charges,
                                     const double* total_dipoles, int32_t num_points, const double* grid,
                                     int32_t periodic, const double* box3, double* out, void* stream) {
    g_noalloc_error[0] = '\0';
    // A non-sticky error left by the caller's earlier CUDA work would
    // otherwise be reported below as this call's own launch failure.
    (void)cudaGetLastError();
    if (num_particles < 0 || num_points < 0)
        return noalloc_fail(TDP_ERR_INVALID_ARGUMENT, "tdp_potential_noalloc: negative size");
    if (num_points == 0) return TDP_OK;
    if (!grid || !out || (num_particles > 0 && (!positions || !charges || !total_dipoles)) ||
        (periodic && !box3))
        return noalloc_fail(TDP_ERR_INVALID_ARGUMENT, "tdp_potential_noalloc: NULL pointer argument");
    if ((size_t)num_points > (size_t)TDP_NOALLOC_SCRATCH_DOUBLES) {
        char buf[160];
        snprintf(buf, sizeof buf, "tdp_potential_noalloc: %d grid points exceed the %d-point scratch limit",
                 num_points, TDP_NOALLOC_SCRATCH_DOUBLES);
        return noalloc_fail(TDP_ERR_INVALID_ARGUMENT, buf);
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return noalloc_fail(TDP_ERR_CUDA, "tdp_potential_noalloc: no usable current CUDA device");
    void* scratch = nullptr;
    {
        // First call on this device: resolve the device address of the
        // scratch array with this device current.
        std::lock_guard<std::mutex> lock(g_scratch_mutex);
        if (!g_scratch_addr[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_potential_scratch);
            if (e != cudaSuccess || !p) {
                (void)cudaGetLastError();  // leave no error of this lookup behind
                char buf[200];
                snprintf(buf, sizeof buf, "tdp_potential_noalloc: cudaGetSymbolAddress failed: %s",
                         cudaGetErrorString(e));
                return noalloc_fail(TDP_ERR_CUDA, buf);
            }
            g_scratch_addr[dev] = p;
        }
        scratch = g_scratch_addr[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (num_particles == 0) {
        cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double) * (size_t)num_points, st);
        return e == cudaSuccess ? TDP_OK : noalloc_fail(TDP_ERR_CUDA, cudaGetErrorString(e));
    }
    // Split the atoms so that small grids still fill the GPU, within the scratch.
    const int gblocks = (num_points + kPtsPerBlock - 1) / kPtsPerBlock;
    int nsplit = (4 * 148 + gblocks - 1) / gblocks;
    const int max_by_atoms = (num_particles + kAtomStage - 1) / kAtomStage;
    const int max_by_scratch = (int)((size_t)TDP_NOALLOC_SCRATCH_DOUBLES / (size_t)num_points);
    nsplit = nsplit < max_by_atoms ? nsplit : max_by_atoms;
    nsplit = nsplit < max_by_scratch ? nsplit : max_by_scratch;
    if (nsplit < 1) nsplit = 1;
    int chunk = (num_particles + nsplit - 1) / nsplit;
    nsplit = (num_particles + chunk - 1) / chunk;
    double bx = periodic ? box3[0] : 0.0, by = periodic ? box3[1] : 0.0, bz = periodic ? box3[2] : 0.0;
    dim3 grid2(gblocks, nsplit);
    k_potential_partial<<<grid2, kPtsPerBlock, 0, st>>>(num_particles, num_points, chunk, periodic ? 1 : 0, bx, by, bz,
                                                        positions, charges, total_dipoles, grid,
                                                        static_cast<double*>(scratch));
    k_potential_reduce<<<(num_points + 255) / 256, 256, 0, st>>>(num_points, nsplit,
                                                                 static_cast<const double*>(scratch), out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(TDP_ERR_CUDA, cudaGetErrorString(e));
    return TDP_OK;
}
