// tdp_md.cu -- rigid-water velocity Verlet (RATTLE) behind
// include/tholedipole_b200_md.h: device kernels (one thread per water) and the
// same per-water steps on host arrays (threads over ranges of waters).  The
// three distance constraints of a water are solved together: Newton steps on
// the 3x3 linearised system for the positions (matrix SHAKE: quadratic
// convergence, 3-4 steps to the relative tolerance of 1e-12) and the exact
// 3x3 linear solve for the velocities (RATTLE), refined while the tolerance
// is not met.  A singular system falls back to one Gauss-Seidel sweep; every
// loop has a fixed iteration cap.
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

// eps(k, q): +1 when atom k is the first atom of constraint q, -1 when the second.
__host__ __device__ inline double eps_kq(int k, int q) {
    return (k == pair_a(q) ? 1.0 : 0.0) - (k == pair_b(q) ? 1.0 : 0.0);
}

// g = A^-1 b by the adjugate; false when A is singular.
__host__ __device__ inline bool solve3(const double A[3][3], const double b[3], double g[3]) {
    const double c00 = A[1][1] * A[2][2] - A[1][2] * A[2][1];
    const double c01 = A[1][2] * A[2][0] - A[1][0] * A[2][2];
    const double c02 = A[1][0] * A[2][1] - A[1][1] * A[2][0];
    const double det = A[0][0] * c00 + A[0][1] * c01 + A[0][2] * c02;
    if (!(fabs(det) > 0.0) || !isfinite(det)) return false;
    const double id = 1.0 / det;
    const double inv[3][3] = {
        {c00 * id, (A[0][2] * A[2][1] - A[0][1] * A[2][2]) * id, (A[0][1] * A[1][2] - A[0][2] * A[1][1]) * id},
        {c01 * id, (A[0][0] * A[2][2] - A[0][2] * A[2][0]) * id, (A[0][2] * A[1][0] - A[0][0] * A[1][2]) * id},
        {c02 * id, (A[0][1] * A[2][0] - A[0][0] * A[2][1]) * id, (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * id}};
    for (int i = 0; i < 3; i++) g[i] = inv[i][0] * b[0] + inv[i][1] * b[1] + inv[i][2] * b[2];
    return true;
}

// C_pq: change of constraint p's bond vector per unit multiplier of
// constraint q along q's direction, eps(a_p, q)/m_a_p - eps(b_p, q)/m_b_p.
__host__ __device__ inline void coupling(const double inv[3], double C[3][3]) {
    for (int p = 0; p < 3; p++)
        for (int q = 0; q < 3; q++)
            C[p][q] = eps_kq(pair_a(p), q) * inv[pair_a(p)] - eps_kq(pair_b(p), q) * inv[pair_b(p)];
}

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
    // SHAKE along the pre-drift bond vectors r0: atom k moves by
    // sum_q eps(k, q) g_q r0_q / m_k; Newton steps on sigma_p = |s_p|^2 - d_p^2.
    double r0[3][3], C[3][3];
    for (int p = 0; p < 3; p++)
        for (int c = 0; c < 3; c++) r0[p][c] = x0.x[pair_a(p)][c] - x0.x[pair_b(p)][c];
    coupling(inv, C);
    for (int it = 0; it < kMaxConstraintIter; it++) {
        double sv[3][3], sig[3];
        bool done = true;
        for (int p = 0; p < 3; p++) {
            for (int c = 0; c < 3; c++) sv[p][c] = x.x[pair_a(p)][c] - x.x[pair_b(p)][c];
            sig[p] = sv[p][0] * sv[p][0] + sv[p][1] * sv[p][1] + sv[p][2] * sv[p][2] - d2[p];
            if (fabs(sig[p]) > kTol * d2[p]) done = false;
        }
        if (done) break;
        double A[3][3], rhs[3], g[3];
        for (int p = 0; p < 3; p++) {
            rhs[p] = -sig[p];
            for (int q = 0; q < 3; q++)
                A[p][q] = 2.0 * C[p][q] * (sv[p][0] * r0[q][0] + sv[p][1] * r0[q][1] + sv[p][2] * r0[q][2]);
        }
        if (!solve3(A, rhs, g)) {
            // Degenerate geometry: one Gauss-Seidel sweep of classic SHAKE.
            for (int p = 0; p < 3; p++) {
                const int a = pair_a(p), b = pair_b(p);
                double sp[3];
                for (int c = 0; c < 3; c++) sp[c] = x.x[a][c] - x.x[b][c];
                const double diff = d2[p] - (sp[0] * sp[0] + sp[1] * sp[1] + sp[2] * sp[2]);
                const double sr = sp[0] * r0[p][0] + sp[1] * r0[p][1] + sp[2] * r0[p][2];
                const double gp = diff / (2.0 * sr * (inv[a] + inv[b]));
                for (int c = 0; c < 3; c++) {
                    x.x[a][c] += gp * r0[p][c] * inv[a];
                    x.x[b][c] -= gp * r0[p][c] * inv[b];
                    v.x[a][c] += gp * r0[p][c] * inv[a] / dt;
                    v.x[b][c] -= gp * r0[p][c] * inv[b] / dt;
                }
            }
            continue;
        }
        for (int q = 0; q < 3; q++) {
            const int a = pair_a(q), b = pair_b(q);
            for (int c = 0; c < 3; c++) {
                x.x[a][c] += g[q] * r0[q][c] * inv[a];
                x.x[b][c] -= g[q] * r0[q][c] * inv[b];
                v.x[a][c] += g[q] * r0[q][c] * inv[a] / dt;
                v.x[b][c] -= g[q] * r0[q][c] * inv[b] / dt;
            }
        }
    }
    store(pos, w, x);
    store(vel, w, v);
}

// Velocities onto the constraints: r_p . (v_a - v_b) = 0 for the current
// bonds r_p; atom k's velocity changes by -sum_q eps(k, q) k_q r_q / m_k, which
// is linear in k: B k = r . dv with B_pq = C_pq (r_p . r_q), solved exactly
// and refined while the tolerance is not met.
__host__ __device__ inline void rattle(const W& x, W& v, const double inv[3], const double d2[3]) {
    double r[3][3], C[3][3], B[3][3];
    for (int p = 0; p < 3; p++)
        for (int c = 0; c < 3; c++) r[p][c] = x.x[pair_a(p)][c] - x.x[pair_b(p)][c];
    coupling(inv, C);
    for (int p = 0; p < 3; p++)
        for (int q = 0; q < 3; q++) B[p][q] = C[p][q] * (r[p][0] * r[q][0] + r[p][1] * r[q][1] + r[p][2] * r[q][2]);
    for (int it = 0; it < kMaxConstraintIter; it++) {
        double rv[3];
        bool done = true;
        for (int p = 0; p < 3; p++) {
            const int a = pair_a(p), b = pair_b(p);
            double dv[3];
            for (int c = 0; c < 3; c++) dv[c] = v.x[a][c] - v.x[b][c];
            rv[p] = r[p][0] * dv[0] + r[p][1] * dv[1] + r[p][2] * dv[2];
            const double vn = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]) * sqrt(d2[p]);
            if (fabs(rv[p]) > kTol * (vn + 1e-300)) done = false;
        }
        if (done) break;
        double k[3];
        if (!solve3(B, rv, k)) {
            // Degenerate geometry: one Gauss-Seidel sweep.
            for (int p = 0; p < 3; p++) {
                const int a = pair_a(p), b = pair_b(p);
                double dv[3];
                for (int c = 0; c < 3; c++) dv[c] = v.x[a][c] - v.x[b][c];
                const double kp = (r[p][0] * dv[0] + r[p][1] * dv[1] + r[p][2] * dv[2]) / (d2[p] * (inv[a] + inv[b]));
                for (int c = 0; c < 3; c++) {
                    v.x[a][c] -= kp * r[p][c] * inv[a];
                    v.x[b][c] += kp * r[p][c] * inv[b];
                }
            }
            continue;
        }
        for (int q = 0; q < 3; q++) {
            const int a = pair_a(q), b = pair_b(q);
            for (int c = 0; c < 3; c++) {
                v.x[a][c] -= k[q] * r[q][c] * inv[a];
                v.x[b][c] += k[q] * r[q][c] * inv[b];
            }
        }
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
