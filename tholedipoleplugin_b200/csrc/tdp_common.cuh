// tdp_common.cuh -- shared types and device helpers of the sm_100a
// TholeDipoleForce kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tdp {

constexpr int kTile = 32;          // atoms per tile (one warp's i-atoms, one j-subtile)
constexpr int kVecThreads = 256;   // threads per block of the O(N) vector kernels

template <class R> struct Vec4T;
template <> struct Vec4T<float> { typedef float4 type; };
template <> struct Vec4T<double> { typedef double4 type; };

// Parameters every pair kernel needs, passed by value.
struct PairParams {
    int n;                 // particles
    int n_tiles;           // ceil(n / kTile)
    int periodic;          // 1: orthorhombic minimum image from the box diagonal
    double box[3];
    double inv_box[3];
    double half_box_tol[3];  // box/2 minus a rounding margin (FP32 fold ambiguity test)
    float damp_r2;         // squared distance beyond which a*u^3 >= 50 for every pair
    float rinv4_power;     // 1: rInvVec[4] = 1/r^4; 0: the constant rinv4_fill
    float rinv4_fill;
    int mutual;            // polarization type is Mutual (adds the Uind-Uind terms)
    int band_tiles;        // 32-atom tiles per band of the pair kernels (1..16)
    int n_bands;           // bands covering the n_tiles real tiles
    int lab_energy;        // 1: undamped unit-scale tile pairs take the lab-frame energy walk
};

__device__ __forceinline__ float rsqrt_r(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsqrt_r(double x) { return rsqrt(x); }
__device__ __forceinline__ float exp_r(float x) { return expf(x); }
__device__ __forceinline__ double exp_r(double x) { return exp(x); }
__device__ __forceinline__ float sqrt_r(float x) { return sqrtf(x); }
__device__ __forceinline__ double sqrt_r(double x) { return sqrt(x); }

// Minimum image of one component in FP64, as ReferencePmeTholeDipoleForce::
// getPeriodicDelta (d -= L*floor(d/L + 0.5)), with the reciprocal precomputed.
__device__ __forceinline__ double fold_d(double d, double L, double invL) {
    return d - L * floor(d * invL + 0.5);
}

// FP32 minimum image: round-to-nearest via the 1.5*2^23 constant (valid for
// |d/L| < 2^22), three FP32-pipe operations and no conversion instruction.
__device__ __forceinline__ float fold_f(float d, float L, float invL) {
    const float magic = 12582912.0f;
    float t = __fadd_rn(__fmaf_rn(d, invL, magic), -magic);
    return __fmaf_rn(-t, L, d);
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
template <class T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Sum over a block of kVecThreads threads; result valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* smem) {
    v = warp_sum(v);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) smem[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) r += smem[k];
    __syncthreads();
    return r;
}

// Deterministic sum of m block partials, same order in every block.
__device__ __forceinline__ double sum_partials(const double* p, int m, double* smem) {
    double v = 0.0;
    for (int k = threadIdx.x; k < m; k += blockDim.x) v += p[k];
    double s = block_sum(v, smem);
    if (threadIdx.x == 0) smem[32] = s;
    __syncthreads();
    s = smem[32];
    __syncthreads();
    return s;
}

}  // namespace tdp
