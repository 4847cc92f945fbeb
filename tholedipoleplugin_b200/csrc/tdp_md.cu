// tdp_md.cu -- rigid-water velocity Verlet (RATTLE) behind
// include/tholedipole_b200_md.h: device kernels (one thread per water) and the
// same per-water steps on host arrays (threads over ranges of waters).  The
// three distance constraints are iterated (Gauss-Seidel SHAKE/RATTLE) to a
// relative tolerance of 1e-12 with a fixed iteration cap, so every loop is
// bounded.
#include "tholedipole_b200.h"
#include "tholedipole_b200_md.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <thread>
#include <vector>

namespace {

constexpr int kMaxConstraintIter = 200;
constexpr double kTol = 1e-12;

struct W {
    double x[3][3];
};

__host__ __device__ inline void load(const double* a, int w, W& o) {
    for (int k = 0; k < 3; k++)
        for (int c = 0; c < 3; c++) o.x[k][c] = a[9 * w + 3 * k + c];
}
__host__ __device__ inline void store(double* a, int w, const W& o) {
    for (int k = 0; k < 3; k++)
        for (int c = 0; c < 3; c++) a[9 * w + 3 * k + c] = o.x[k][c];
}

// Constraint p joins atoms (0, 1), (0, 2), (1, 2).
__host__ __device__ inline int pair_a(int p) { return p == 2 ? 1 : 0; }
__host__ __device__ inline int pair_b(int p) { return p == 0 ? 1 : 2; }

// One water: v += dt/2 F/m, x += dt v, SHAKE along the pre-drift bonds.
__host__ __device__ inline void kick_drift_one(int w, double doh, double dhh, double mo, double mh, double dt,
                                               double* pos, double* vel, const double* frc) {
    W x0, v, f;
    load(pos, w, x0);
    load(vel, w, v);
    load(frc, w, f);
    const double inv[3] = {1.0 / mo, 1.0 / mh, 1.0 / mh};
    const double d2[3] = {doh * doh, doh * doh, dhh * dhh};
    W x;
    for (int k = 0; k < 3; k++)
        for (int c = 0; c < 3; c++) {
            v.x[k][c] += 0.5 * dt * f.x[k][c] * inv[k];
            x.x[k][c] = x0.x[k][c] + dt * v.x[k][c];
        }
    // SHAKE along the pre-drift bond vectors.
    for (int it = 0; it < kMaxConstraintIter; it++) {
        bool done = true;
        for (int p = 0; p < 3; p++) {
            const int a = pair_a(p), b = pair_b(p);
            double s[3], r0[3];
            for (int c = 0; c < 3; c++) {
                s[c] = x.x[a][c] - x.x[b][c];
                r0[c] = x0.x[a][c] - x0.x[b][c];
            }
            double ss = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
            double diff = d2[p] - ss;
            if (fabs(diff) > kTol * d2[p]) done = false;
            double sr = s[0] * r0[0] + s[1] * r0[1] + s[2] * r0[2];
            double g = diff / (2.0 * sr * (inv[a] + inv[b]));
            for (int c = 0; c < 3; c++) {
                x.x[a][c] += g * r0[c] * inv[a];
                x.x[b][c] -= g * r0[c] * inv[b];
                v.x[a][c] += g * r0[c] * inv[a] / dt;
                v.x[b][c] -= g * r0[c] * inv[b] / dt;
            }
        }
        if (done) break;
    }
    store(pos, w, x);
    store(vel, w, v);
}

__host__ __device__ inline void rattle(const W& x, W& v, const double inv[3], const double d2[3]) {
    for (int it = 0; it < kMaxConstraintIter; it++) {
        bool done = true;
        for (int p = 0; p < 3; p++) {
            const int a = pair_a(p), b = pair_b(p);
            double r[3], dv[3];
            for (int c = 0; c < 3; c++) {
                r[c] = x.x[a][c] - x.x[b][c];
                dv[c] = v.x[a][c] - v.x[b][c];
            }
            double rv = r[0] * dv[0] + r[1] * dv[1] + r[2] * dv[2];
            double vn = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]) * sqrt(d2[p]);
            if (fabs(rv) > kTol * (vn + 1e-300)) done = false;
            double k = rv / (d2[p] * (inv[a] + inv[b]));
            for (int c = 0; c < 3; c++) {
                v.x[a][c] -= k * r[c] * inv[a];
                v.x[b][c] += k * r[c] * inv[b];
            }
        }
        if (done) break;
    }
}

// One water: v += dt/2 F/m (frc may be null), then RATTLE.
__host__ __device__ inline void kick_one(int w, double doh, double dhh, double mo, double mh, double dt,
                                         const double* pos, double* vel, const double* frc) {
    W x, v, f;
    load(pos, w, x);
    load(vel, w, v);
    const double inv[3] = {1.0 / mo, 1.0 / mh, 1.0 / mh};
    const double d2[3] = {doh * doh, doh * doh, dhh * dhh};
    if (frc) {
        load(frc, w, f);
        for (int k = 0; k < 3; k++)
            for (int c = 0; c < 3; c++) v.x[k][c] += 0.5 * dt * f.x[k][c] * inv[k];
    }
    rattle(x, v, inv, d2);
    store(vel, w, v);
}

__global__ void k_kick_drift(int nw, double doh, double dhh, double mo, double mh, double dt, double* pos,
                             double* vel, const double* frc) {
    int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nw) return;
    kick_drift_one(w, doh, dhh, mo, mh, dt, pos, vel, frc);
}

__global__ void k_kick(int nw, double doh, double dhh, double mo, double mh, double dt, const double* pos,
                       double* vel, const double* frc) {
    int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nw) return;
    kick_one(w, doh, dhh, mo, mh, dt, pos, vel, frc);
}

__global__ void k_kinetic(int nw, double mo, double mh, const double* vel, double* out) {
    __shared__ double red[256];
    int w = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (w < nw)
        for (int k = 0; k < 3; k++) {
            double m = k == 0 ? mo : mh;
            for (int c = 0; c < 3; c++) {
                double vv = vel[9 * w + 3 * k + c];
                e += 0.5 * m * vv * vv;
            }
        }
    red[threadIdx.x] = e;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(out, red[0]);
}

// Host loop over waters, split across up to 16 threads (each water independent).
template <class F>
void host_each(int nw, F&& fn) {
    unsigned hw = std::thread::hardware_concurrency();
    int nt = (int)std::max(1u, std::min(16u, hw ? hw : 1u));
    nt = std::min(nt, std::max(1, nw / 1024));
    if (nt <= 1) {
        for (int w = 0; w < nw; w++) fn(w);
        return;
    }
    std::vector<std::thread> th;
    th.reserve(nt);
    for (int t = 0; t < nt; t++) {
        const int w0 = (int)((long long)nw * t / nt), w1 = (int)((long long)nw * (t + 1) / nt);
        try {
            th.emplace_back([w0, w1, &fn] {
                for (int w = w0; w < w1; w++) fn(w);
            });
        } catch (...) {
            // No thread available: this range runs on the calling thread.
            for (int w = w0; w < w1; w++) fn(w);
        }
    }
    for (auto& t : th) t.join();
}

int status(cudaError_t e) { return e == cudaSuccess ? TDP_OK : TDP_ERR_CUDA; }

}  // namespace

extern "C" {

int tdp_md_kick_drift(int32_t nw, double doh, double dhh, double mo, double mh, double dt, double* pos, double* vel,
                      const double* frc, void* stream) {
    if (nw < 0 || !pos || !vel || !frc) return TDP_ERR_INVALID_ARGUMENT;
    if (nw == 0) return TDP_OK;
    k_kick_drift<<<(nw + 127) / 128, 128, 0, (cudaStream_t)stream>>>(nw, doh, dhh, mo, mh, dt, pos, vel, frc);
    return status(cudaGetLastError());
}

int tdp_md_kick(int32_t nw, double doh, double dhh, double mo, double mh, double dt, const double* pos, double* vel,
                const double* frc, void* stream) {
    if (nw < 0 || !pos || !vel || !frc) return TDP_ERR_INVALID_ARGUMENT;
    if (nw == 0) return TDP_OK;
    k_kick<<<(nw + 127) / 128, 128, 0, (cudaStream_t)stream>>>(nw, doh, dhh, mo, mh, dt, pos, vel, frc);
    return status(cudaGetLastError());
}

int tdp_md_constrain_velocities(int32_t nw, double doh, double dhh, double mo, double mh, const double* pos,
                                double* vel, void* stream) {
    if (nw < 0 || !pos || !vel) return TDP_ERR_INVALID_ARGUMENT;
    if (nw == 0) return TDP_OK;
    k_kick<<<(nw + 127) / 128, 128, 0, (cudaStream_t)stream>>>(nw, doh, dhh, mo, mh, 0.0, pos, vel, nullptr);
    return status(cudaGetLastError());
}

int tdp_md_host_kick_drift(int32_t nw, double doh, double dhh, double mo, double mh, double dt, double* pos,
                           double* vel, const double* frc) {
    if (nw < 0 || !pos || !vel || !frc) return TDP_ERR_INVALID_ARGUMENT;
    host_each(nw, [=](int w) { kick_drift_one(w, doh, dhh, mo, mh, dt, pos, vel, frc); });
    return TDP_OK;
}

int tdp_md_host_kick(int32_t nw, double doh, double dhh, double mo, double mh, double dt, const double* pos,
                     double* vel, const double* frc) {
    if (nw < 0 || !pos || !vel) return TDP_ERR_INVALID_ARGUMENT;
    host_each(nw, [=](int w) { kick_one(w, doh, dhh, mo, mh, dt, pos, vel, frc); });
    return TDP_OK;
}

int tdp_md_kinetic_energy(int32_t nw, double mo, double mh, const double* vel, double* out, void* stream) {
    if (nw < 0 || !vel || !out) return TDP_ERR_INVALID_ARGUMENT;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double), st);
    if (e != cudaSuccess) return TDP_ERR_CUDA;
    if (nw == 0) return TDP_OK;
    k_kinetic<<<(nw + 255) / 256, 256, 0, st>>>(nw, mo, mh, vel, out);
    return status(cudaGetLastError());
}

}  // extern "C"
