// tdp_batch.cu -- many isolated clusters (NoCutoff systems) evaluated in one
// persistent launch: the tdp_batch_* entry points of include/tholedipole_b200.h.
//
// Device side.  Each CTA pulls clusters from a work queue ordered by
// decreasing size and keeps the whole cluster in shared memory: FP64
// positions, parameters, permanent field, induced dipoles and the CG vectors,
// plus centroid-relative float4 (or double4) records for the pair arithmetic.
// Inside the CTA it runs the reference evaluation end to end -- lab-frame
// rotation, permanent field, induced dipoles, pair energy/force/torque and
// torque mapping (ReferenceTholeDipoleForce.cpp, "RTDF.cpp", :117-124 and
// :1117-1155) -- with the per-pair device functions of the box kernels
// (tdp_pairs.cuh, tdp_frames.cuh), so the semantics are the same by
// construction.  Mutual polarization is the box path's conjugate gradient in
// y = mu/sqrt(alpha) with FP64 vectors and block reductions, the reference's
// RMS-dipole-change stopping test and a true-residual check before accepting.
//
// Tile shape.  A pair pass splits the CTA's threads evenly over the
// cluster's atoms (floor(T/n) or one more consecutive lanes per atom, at most
// the lane cap): lane l of atom i takes j = l, l+L, ..., leaves its partial
// sums in shared memory, and the atom's lanes are added in lane order, so
// small clusters still occupy the CTA and no thread idles on large ones.  The
// CTA size and the lane cap are the tile shape; tdp_batch_compute picks them
// on the first call by timing every candidate on the batch itself.
//
// Host side.  The launch (queue reset + kernel) is captured once in a CUDA
// graph and replayed; one call is: positions in, graph, then forces and
// per-cluster energies out.
#include "tholedipole_b200.h"
#include "tdp_f32x2.cuh"
#include "tdp_frames.cuh"
#include "tdp_host.h"
#include "tdp_pairs.cuh"
#include "tdp_adjoint.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <numeric>
#include <string>
#include <vector>

namespace tdp {
namespace {

struct BatchArgs {
    int num_clusters;
    int max_atoms, max_exc, korder, lmax;
    int polarization;  // TDP_DIRECT / TDP_MUTUAL / TDP_EXTRAPOLATED
    int max_iter;
    double target_eps;
    double damp_r2;
    double rinv4_power, rinv4_fill;
    // Mixed form: 1 = permanent field and energy/force pass in FP64, FP32 only
    // in the CG matvec; 0 = every pair pass in FP32.
    int fp64_passes;
    const int* order;   // clusters by decreasing size
    const int* coff;    // num_clusters+1 atom offsets
    const double* pos;  // n*3
    const double* charge;
    const double* dip_mol;
    const double* alpha;
    const double* thole;
    const int4* axis;   // (type, z, x, y), global indices
    const int* exc_off;
    const int* exc_j;
    const double* exc_m;
    const double* exc_s;
    const int* users_off;
    const int2* users;  // (frame atom, role), global
    const double* coef; // extrapolation coefficients
    int* queue;
    double* forces;     // n*3, written
    double* mu_out;     // n*3 induced dipoles
    double* energy;     // per cluster
    int* iters;         // per cluster
    double* eps;        // per cluster
};

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Per-atom double slots of the work region: CG (y, r, p, q) or the
// extrapolation history plus one field; forces and torques afterwards.
__host__ __device__ inline int work_slots(int korder) { return 3 * korder + 3 > 12 ? 3 * korder + 3 : 12; }

template <class R>
__host__ __device__ inline size_t batch_smem(int M, int X, int korder) {
    typedef typename Vec4T<R>::type V4;
    size_t b = 0;
    b += sizeof(double) * ((size_t)M * (3 + 3 + 3 + 1 + 1 + work_slots(korder)) + 64);
    b += sizeof(unsigned long long) * (size_t)M;   // exception-partner window masks
    b += sizeof(double) * 7 * 512;                  // per-thread partial sums of the pair passes
    b = align_up(b, 32);
    b += sizeof(V4) * 3 * (size_t)M;
    b = align_up(b, 16);
    b += sizeof(int4) * (size_t)M;
    b += sizeof(int) * ((size_t)M + 1 + (size_t)X);
    b = align_up(b, 8);
    b += sizeof(R) * 2 * (size_t)X;
    b = align_up(b, 16);
    b += sizeof(double) * 5 * (size_t)M;            // FP64 lab dipoles, charges, Thole factors
    return align_up(b, 16);
}

template <class R>
struct Cl {
    typedef typename Vec4T<R>::type V4;
    double *pos, *E, *mu, *alpha, *salpha, *w, *red;
    // Exception partners of atom i by offset: bit d (d < 63) set if atom
    // i + d - 32 is listed, bit 63 set if a partner lies outside that window.
    unsigned long long* emask;
    double* part;   // 7 per thread: partial sums of the pair passes, reduced per atom in lane order
    V4 *posq, *dipt, *vec;
    int4* axis;
    int *eoff, *ej;
    R *em, *es;
    double *lab64, *q64, *th64;   // FP64 lab-frame dipoles (3 per atom), charges, Thole factors
    int M;
};

template <class R>
__device__ Cl<R> carve(char* base, int M, int X, int korder) {
    typedef typename Vec4T<R>::type V4;
    Cl<R> c;
    c.M = M;
    double* d = reinterpret_cast<double*>(base);
    c.pos = d; d += 3 * M;
    c.E = d; d += 3 * M;
    c.mu = d; d += 3 * M;
    c.alpha = d; d += M;
    c.salpha = d; d += M;
    c.w = d; d += (size_t)work_slots(korder) * M;
    c.red = d; d += 64;
    c.emask = reinterpret_cast<unsigned long long*>(d);
    d += M;
    c.part = d;
    d += 7 * 512;
    size_t off = align_up((size_t)(reinterpret_cast<char*>(d) - base), 32);
    V4* v = reinterpret_cast<V4*>(base + off);
    c.posq = v; v += M;
    c.dipt = v; v += M;
    c.vec = v; v += M;
    off = align_up((size_t)(reinterpret_cast<char*>(v) - base), 16);
    int4* a = reinterpret_cast<int4*>(base + off);
    c.axis = a; a += M;
    int* ip = reinterpret_cast<int*>(a);
    c.eoff = ip; ip += M + 1;
    c.ej = ip; ip += X;
    off = align_up((size_t)(reinterpret_cast<char*>(ip) - base), 8);
    R* rp = reinterpret_cast<R*>(base + off);
    c.em = rp; rp += X;
    c.es = rp; rp += X;
    off = align_up((size_t)(reinterpret_cast<char*>(rp) - base), 16);
    double* dd = reinterpret_cast<double*>(base + off);
    c.lab64 = dd; dd += 3 * M;
    c.q64 = dd; dd += M;
    c.th64 = dd;
    return c;
}

// Block sum in a fixed order (deterministic for a given CTA size).
__device__ __forceinline__ double bsum(double v, double* red) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    const int nw = blockDim.x >> 5;
    for (int k = 0; k < nw; k++) s += red[k];
    return s;
}

// Two block sums in one pass (one pair of barriers), each in the fixed order of bsum.
__device__ __forceinline__ void bsum2(double& a, double& b, double* red) {
    a = warp_sum(a);
    b = warp_sum(b);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) {
        red[w] = a;
        red[32 + w] = b;
    }
    __syncthreads();
    double sa = 0.0, sb = 0.0;
    const int nw = blockDim.x >> 5;
    for (int k = 0; k < nw; k++) {
        sa += red[k];
        sb += red[32 + k];
    }
    a = sa;
    b = sb;
}


// Thread split of a pair pass over the atoms [base, base + na) of a cluster:
// with T = min(blockDim.x, na * lmax) threads in use, atom base + a gets the
// contiguous threads [first(a), first(a + 1)), first(a) = ceil(a T / na), so
// every atom has floor(T / na) or one more lanes and all T threads work.
// Each thread leaves K partial sums in part; split_sum adds an atom's lanes
// in lane order (deterministic for a given CTA size and lmax).
struct Split {
    int a, l, L, T;
    bool act;
};
__device__ __forceinline__ int split_first(int a, int na, int T) { return (a * T + na - 1) / na; }
__device__ __forceinline__ Split split(int na, int lmax) {
    Split q;
    q.T = min((int)blockDim.x, na * lmax);
    const int t = threadIdx.x;
    q.act = t < q.T;
    q.a = q.act ? (t * na) / q.T : 0;
    const int f0 = split_first(q.a, na, q.T);
    q.l = t - f0;
    q.L = split_first(q.a + 1, na, q.T) - f0;
    return q;
}
// Sum k of atom a (thread a < na calls it after a barrier).
__device__ __forceinline__ double split_sum(const double* part, int K, int k, int a, int na, int T) {
    const int f0 = split_first(a, na, T), f1 = split_first(a + 1, na, T);
    double v = 0.0;
    for (int u = f0; u < f1; u++) v += part[K * u + k];
    return v;
}

// (M, I) scales of the pair (i, j) from i's local exception list, scanned
// only when i's partner mask says j can be on it.
template <class R>
__device__ __forceinline__ void pair_scales(const Cl<R>& c, int i, int j, R& m, R& s) {
    m = R(1);
    s = R(1);
    const unsigned long long w = c.emask[i];
    const unsigned d = (unsigned)(j - i + 32);
    if (d < 63u ? ((w >> d) & 1ull) == 0ull : (w >> 63) == 0ull) return;
    for (int e = c.eoff[i]; e < c.eoff[i + 1]; e++)
        if (c.ej[e] == j) {
            m = c.em[e];
            s = c.es[e];
        }
}

// FP32 lane loop of cluster_matvec: the lane's J atoms j and j + L ride in the
// halves of f32x2 registers (pair_matvec per half, I scale applied per half).
// A half without a pair (j == i, past the cluster's end, or I scale 0) gets
// the distance (1, 0, 0) and scale 0, so nothing non-finite enters.
__device__ __forceinline__ void matvec_lane_x2(const Cl<float>& c, int n, int i, int l, int L, float damp_r2,
                                               float& fx, float& fy, float& fz) {
    const float4 pi = c.posq[i];
    const float ti = c.vec[i].w;
    const f2 OX = bc2(pi.x), OY = bc2(pi.y), OZ = bc2(pi.z), THREE = bc2(3.0f);
    f2 FX = 0, FY = 0, FZ = 0;
    for (int ja = l; ja < n; ja += 2 * L) {
        const int jb = ja + L;
        float ma, sa, mb, sb = 0.0f;
        pair_scales(c, i, ja, ma, sa);
        if (ja == i) sa = 0.0f;
        if (jb < n) {
            pair_scales(c, i, jb, mb, sb);
            if (jb == i) sb = 0.0f;
        }
        const float4 pa = c.posq[ja], va = c.vec[ja];
        const float4 pb = c.posq[jb < n ? jb : ja], vb = c.vec[jb < n ? jb : ja];
        float dxa = pa.x - pi.x, dya = pa.y - pi.y, dza = pa.z - pi.z;
        float dxb = pb.x - pi.x, dyb = pb.y - pi.y, dzb = pb.z - pi.z;
        if (sa == 0.0f) {
            dxa = 1.0f;
            dya = dza = 0.0f;
        }
        if (sb == 0.0f) {
            dxb = 1.0f;
            dyb = dzb = 0.0f;
        }
        const f2 DX = pk2(dxa, dxb), DY = pk2(dya, dyb), DZ = pk2(dza, dzb);
        const f2 R2 = fma2(DX, DX, fma2(DY, DY, mul2(DZ, DZ)));
        float r2a, r2b;
        un2(R2, r2a, r2b);
        const f2 RINV = pk2(rsqrt_r(r2a), rsqrt_r(r2b));
        const f2 RINV2 = mul2(RINV, RINV);
        f2 RR3 = mul2(RINV, RINV2);
        f2 RR5 = mul2(mul2(THREE, RR3), RINV2);
        if (r2a < damp_r2 || r2b < damp_r2) {
            float ra, rb, r3a, r3b, r5a, r5b;
            un2(RINV, ra, rb);
            un2(RR3, r3a, r3b);
            un2(RR5, r5a, r5b);
            damp_field<float>(r2a, ra, ti, va.w, damp_r2, r3a, r5a);
            damp_field<float>(r2b, rb, ti, vb.w, damp_r2, r3b, r5b);
            RR3 = pk2(r3a, r3b);
            RR5 = pk2(r5a, r5b);
        }
        const f2 S = pk2(sa, sb);
        const f2 VX = pk2(va.x, vb.x), VY = pk2(va.y, vb.y), VZ = pk2(va.z, vb.z);
        const f2 DD = mul2(RR5, fma2(VX, DX, fma2(VY, DY, mul2(VZ, DZ))));
        const f2 NRR3 = mul2(RR3, bc2(-1.0f));
        FX = fma2(S, fma2(NRR3, VX, mul2(DD, DX)), FX);
        FY = fma2(S, fma2(NRR3, VY, mul2(DD, DY)), FY);
        FZ = fma2(S, fma2(NRR3, VZ, mul2(DD, DZ)), FZ);
    }
    float lo, hi;
    un2(FX, lo, hi);
    fx += lo + hi;
    un2(FY, lo, hi);
    fy += lo + hi;
    un2(FZ, lo, hi);
    fz += lo + hi;
}

// out[i] = sum_j I_ij T_ij v_j with v in c.vec (the mutual field of the operand).
// Ends with a CTA barrier: out is complete and visible on return.
template <class R>
__device__ void cluster_matvec(const Cl<R>& c, int n, int lmax, R damp_r2, double* out) {
    typedef typename Vec4T<R>::type V4;
    for (int base = 0; base < n; base += blockDim.x) {
        const int na = min(n - base, (int)blockDim.x);
        const Split sp = split(na, lmax);
        const int i = base + sp.a;
        R fx = 0, fy = 0, fz = 0;
        if constexpr (sizeof(R) == 4) {
            if (sp.act) matvec_lane_x2(c, n, i, sp.l, sp.L, (float)damp_r2, fx, fy, fz);
        } else if (sp.act) {
            const V4 pi = c.posq[i];
            const R ti = c.vec[i].w;
            for (int j = sp.l; j < n; j += sp.L) {
                if (j == i) continue;
                R m, s;
                pair_scales(c, i, j, m, s);
                if (s == R(0)) continue;
                const V4 pj = c.posq[j], vj = c.vec[j];
                const R dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
                const R r2 = dx * dx + dy * dy + dz * dz;
                R tx = 0, ty = 0, tz = 0;
                pair_matvec<R>(dx, dy, dz, r2, vj.x, vj.y, vj.z, ti, vj.w, damp_r2, tx, ty, tz);
                fx += s * tx;
                fy += s * ty;
                fz += s * tz;
            }
        }
        double* pt = c.part + 3 * threadIdx.x;
        pt[0] = (double)fx;
        pt[1] = (double)fy;
        pt[2] = (double)fz;
        __syncthreads();
        if ((int)threadIdx.x < na)
            for (int k = 0; k < 3; k++)
                out[3 * (base + threadIdx.x) + k] = split_sum(c.part, 3, k, threadIdx.x, na, sp.T);
        __syncthreads();
    }
}

template <class R>
__device__ __forceinline__ void set_vec(const Cl<R>& c, int i, double x, double y, double z) {
    typename Vec4T<R>::type v = c.vec[i];
    v.x = (R)x;
    v.y = (R)y;
    v.z = (R)z;
    c.vec[i] = v;
}

// CG residual of y: r = S (E + T mu) - y (T mu already in tq), p = r, operand
// S p; returns r.r and writes sum alpha |r|^2 into *ee.
template <class R>
__device__ double cg_residual(const Cl<R>& c, int n, const double* y, double* r, double* p, const double* tq,
                              double* ee) {
    double rr = 0.0, e2 = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double sa = c.salpha[i];
        for (int k = 0; k < 3; k++) {
            const double rv = (c.E[3 * i + k] + tq[3 * i + k]) * sa - y[3 * i + k];
            r[3 * i + k] = rv;
            p[3 * i + k] = rv;
            rr += rv * rv;
            e2 += sa * sa * rv * rv;
        }
        set_vec(c, i, sa * p[3 * i], sa * p[3 * i + 1], sa * p[3 * i + 2]);
    }
    bsum2(rr, e2, c.red);
    *ee = e2;
    return rr;
}

// ---- per-cluster stages shared by the forward (k_batch) and reverse
// (k_batch_adjoint) kernels; each ends with its writes visible to the CTA.

// Cluster atoms [a0, a0 + n) into shared memory: FP64 positions, local axis
// atoms, polarizabilities, the local exception list with its partner masks,
// and the pair records (FP32 relative to the centroid in the mixed form).
template <class R>
__device__ __forceinline__ void cluster_load(const Cl<R>& c, const BatchArgs& A, int a0, int n) {
    typedef typename Vec4T<R>::type V4;
    const int e0 = A.exc_off[a0];
    double cx = 0, cy = 0, cz = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int gi = a0 + i;
        for (int k = 0; k < 3; k++) c.pos[3 * i + k] = A.pos[3 * (size_t)gi + k];
        cx += c.pos[3 * i];
        cy += c.pos[3 * i + 1];
        cz += c.pos[3 * i + 2];
        const int4 ax = A.axis[gi];
        c.axis[i] = make_int4(ax.x, ax.y >= 0 ? ax.y - a0 : -1, ax.z >= 0 ? ax.z - a0 : -1,
                              ax.w >= 0 ? ax.w - a0 : -1);
        const double al = A.alpha[gi];
        c.alpha[i] = al;
        c.salpha[i] = al > 0.0 ? sqrt(al) : 0.0;
        c.eoff[i] = A.exc_off[gi] - e0;
        unsigned long long w = 0ull;
        for (int e = A.exc_off[gi]; e < A.exc_off[gi + 1]; e++) {
            const int j = A.exc_j[e] - a0;
            c.ej[e - e0] = j;
            c.em[e - e0] = (R)A.exc_m[e];
            c.es[e - e0] = (R)A.exc_s[e];
            const unsigned d = (unsigned)(j - i + 32);
            w |= d < 63u ? 1ull << d : 1ull << 63;
        }
        c.emask[i] = w;
    }
    if (threadIdx.x == 0) c.eoff[n] = A.exc_off[a0 + n] - e0;
    cx = bsum(cx, c.red) / n;
    cy = bsum(cy, c.red) / n;
    cz = bsum(cz, c.red) / n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        V4 pq;
        if (sizeof(R) == 4) {
            pq.x = (R)(c.pos[3 * i] - cx);
            pq.y = (R)(c.pos[3 * i + 1] - cy);
            pq.z = (R)(c.pos[3 * i + 2] - cz);
        } else {
            pq.x = (R)c.pos[3 * i];
            pq.y = (R)c.pos[3 * i + 1];
            pq.z = (R)c.pos[3 * i + 2];
        }
        pq.w = (R)A.charge[a0 + i];
        c.posq[i] = pq;
    }
    __syncthreads();
}

// Lab-frame permanent dipoles (RTDF.cpp:432-571) into c.dipt (.w: Thole factor).
template <class R>
__device__ __forceinline__ void cluster_lab(const Cl<R>& c, const BatchArgs& A, int a0, int n) {
    typedef typename Vec4T<R>::type V4;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double Rm[3][3], sy;
        frame_rows(c.pos, c.axis[i], i, Rm, sy);
        const double* dm = A.dip_mol + 3 * (size_t)(a0 + i);
        const double d0 = dm[0], d1 = sy * dm[1], d2 = dm[2];
        double lab[3];
        for (int k = 0; k < 3; k++) lab[k] = 0.0 + d0 * Rm[0][k] + d1 * Rm[1][k] + d2 * Rm[2][k];
        V4 dv;
        dv.x = (R)lab[0];
        dv.y = (R)lab[1];
        dv.z = (R)lab[2];
        dv.w = (R)A.thole[a0 + i];
        c.dipt[i] = dv;
        for (int k = 0; k < 3; k++) c.lab64[3 * i + k] = lab[k];
        c.q64[i] = A.charge[a0 + i];
        c.th64[i] = A.thole[a0 + i];
    }
    __syncthreads();
}

// Permanent field into c.E, then mu = alpha E and the operand records = mu.
template <class R>
__device__ __forceinline__ void cluster_fixed_field(const Cl<R>& c, const BatchArgs& A, int n, R damp_r2) {
    typedef typename Vec4T<R>::type V4;
    for (int base = 0; base < n; base += blockDim.x) {
        const int na = min(n - base, (int)blockDim.x);
        const Split sp = split(na, A.lmax);
        const int i = base + sp.a;
        R fx = 0, fy = 0, fz = 0;
        if (sp.act) {
            const V4 pi = c.posq[i];
            const R ti = c.dipt[i].w;
            for (int j = sp.l; j < n; j += sp.L) {
                if (j == i) continue;
                R m, s;
                pair_scales(c, i, j, m, s);
                if (m == R(0)) continue;
                const V4 pj = c.posq[j], dj = c.dipt[j];
                const R dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
                const R r2 = dx * dx + dy * dy + dz * dz;
                R tx = 0, ty = 0, tz = 0;
                pair_fixed<R>(dx, dy, dz, r2, pj.w, dj.x, dj.y, dj.z, ti, dj.w, damp_r2, tx, ty, tz);
                fx += m * tx;
                fy += m * ty;
                fz += m * tz;
            }
        }
        double* pt = c.part + 3 * threadIdx.x;
        pt[0] = (double)fx;
        pt[1] = (double)fy;
        pt[2] = (double)fz;
        __syncthreads();
        if ((int)threadIdx.x < na)
            for (int k = 0; k < 3; k++)
                c.E[3 * (base + threadIdx.x) + k] = split_sum(c.part, 3, k, threadIdx.x, na, sp.T);
        __syncthreads();
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double al = c.alpha[i];
        for (int k = 0; k < 3; k++) c.mu[3 * i + k] = al * c.E[3 * i + k];
        V4 v;
        v.x = (R)c.mu[3 * i];
        v.y = (R)c.mu[3 * i + 1];
        v.z = (R)c.mu[3 * i + 2];
        v.w = c.dipt[i].w;
        c.vec[i] = v;
    }
    __syncthreads();
}

// cluster_fixed_field with FP64 pair arithmetic on the FP64 coordinates,
// dipoles, charges and Thole factors (the mixed form's FP64 passes).
template <class R>
__device__ __forceinline__ void cluster_fixed_field64(const Cl<R>& c, const BatchArgs& A, int n) {
    typedef typename Vec4T<R>::type V4;
    const double damp_r2 = A.damp_r2;
    for (int base = 0; base < n; base += blockDim.x) {
        const int na = min(n - base, (int)blockDim.x);
        const Split sp = split(na, A.lmax);
        const int i = base + sp.a;
        double fx = 0, fy = 0, fz = 0;
        if (sp.act) {
            const double pix = c.pos[3 * i], piy = c.pos[3 * i + 1], piz = c.pos[3 * i + 2];
            const double ti = c.th64[i];
            for (int j = sp.l; j < n; j += sp.L) {
                if (j == i) continue;
                R m, s;
                pair_scales(c, i, j, m, s);
                if (m == R(0)) continue;
                const double dx = c.pos[3 * j] - pix, dy = c.pos[3 * j + 1] - piy, dz = c.pos[3 * j + 2] - piz;
                const double r2 = dx * dx + dy * dy + dz * dz;
                double tx = 0, ty = 0, tz = 0;
                pair_fixed<double>(dx, dy, dz, r2, c.q64[j], c.lab64[3 * j], c.lab64[3 * j + 1], c.lab64[3 * j + 2],
                                   ti, c.th64[j], damp_r2, tx, ty, tz);
                fx += (double)m * tx;
                fy += (double)m * ty;
                fz += (double)m * tz;
            }
        }
        double* pt = c.part + 3 * threadIdx.x;
        pt[0] = fx;
        pt[1] = fy;
        pt[2] = fz;
        __syncthreads();
        if ((int)threadIdx.x < na)
            for (int k = 0; k < 3; k++)
                c.E[3 * (base + threadIdx.x) + k] = split_sum(c.part, 3, k, threadIdx.x, na, sp.T);
        __syncthreads();
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double al = c.alpha[i];
        for (int k = 0; k < 3; k++) c.mu[3 * i + k] = al * c.E[3 * i + k];
        V4 v;
        v.x = (R)c.mu[3 * i];
        v.y = (R)c.mu[3 * i + 1];
        v.z = (R)c.mu[3 * i + 2];
        v.w = c.dipt[i].w;
        c.vec[i] = v;
    }
    __syncthreads();
}

template <class R>
__device__ __forceinline__ void cluster_field_any(const Cl<R>& c, const BatchArgs& A, int n, R damp_r2) {
    if (sizeof(R) == 4 && A.fp64_passes) cluster_fixed_field64(c, A, n);
    else cluster_fixed_field(c, A, n, damp_r2);
}

// Mutual polarization: CG in y = mu / sqrt(alpha) on (I - S T S) y = S E from
// mu = alpha E (c.mu), stopping on the RMS Jacobi-step change (true residual
// confirmed) at target or after cap iterations; leaves mu in c.mu.
template <class R>
__device__ __forceinline__ void cluster_cg(const Cl<R>& c, int n, int lmax, R damp_r2, double target, int cap,
                                           int& it, double& eps) {
    const int n3 = 3 * n;
    double* y = c.w;
    double* r = c.w + 3 * c.M;
    double* p = c.w + 6 * c.M;
    double* q = c.w + 9 * c.M;
    for (int k = threadIdx.x; k < n3; k += blockDim.x) y[k] = c.salpha[k / 3] * c.E[k];
    cluster_matvec(c, n, lmax, damp_r2, q);
    double ee;
    double rr = cg_residual(c, n, y, r, p, q, &ee);
    eps = sqrt(ee / n);
    bool is_true = true;
    while (true) {
        if (!(eps <= 1.0e300)) break;  // non-finite
        if (eps <= target || it >= cap) {
            if (is_true) break;
            // Accept only on the true residual of the current iterate.
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                const double sa = c.salpha[i];
                set_vec(c, i, sa * y[3 * i], sa * y[3 * i + 1], sa * y[3 * i + 2]);
            }
            __syncthreads();
            cluster_matvec(c, n, lmax, damp_r2, q);
            rr = cg_residual(c, n, y, r, p, q, &ee);
            eps = sqrt(ee / n);
            is_true = true;
            continue;
        }
        __syncthreads();
        cluster_matvec(c, n, lmax, damp_r2, q);  // T S p
        double pq = 0.0;
        for (int k = threadIdx.x; k < n3; k += blockDim.x) {
            const double qv = p[k] - c.salpha[k / 3] * q[k];
            q[k] = qv;
            pq += p[k] * qv;
        }
        pq = bsum(pq, c.red);
        const double a = rr / pq;
        double rr2 = 0.0, e2 = 0.0;
        for (int k = threadIdx.x; k < n3; k += blockDim.x) {
            const double sa = c.salpha[k / 3];
            y[k] += a * p[k];
            const double rv = r[k] - a * q[k];
            r[k] = rv;
            rr2 += rv * rv;
            e2 += sa * sa * rv * rv;
        }
        bsum2(rr2, e2, c.red);
        eps = sqrt(e2 / n);
        const double beta = rr2 / rr;
        rr = rr2;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const double sa = c.salpha[i];
            for (int k = 0; k < 3; k++) p[3 * i + k] = r[3 * i + k] + beta * p[3 * i + k];
            set_vec(c, i, sa * p[3 * i], sa * p[3 * i + 1], sa * p[3 * i + 2]);
        }
        it++;
        is_true = false;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n3; k += blockDim.x) c.mu[k] = c.salpha[k / 3] * y[k];
}

template <class R>
__global__ void __launch_bounds__(512) k_batch(BatchArgs A) {
    typedef typename Vec4T<R>::type V4;
    extern __shared__ __align__(32) char smem_raw[];
    const Cl<R> c = carve<R>(smem_raw, A.max_atoms, A.max_exc, A.korder);
    __shared__ int s_slot;
    const R damp_r2 = (R)A.damp_r2;
    const R rv4p = (R)A.rinv4_power, rv4f = (R)A.rinv4_fill;
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) s_slot = atomicAdd(A.queue, 1);
        __syncthreads();
        const int slot = s_slot;
        if (slot >= A.num_clusters) break;
        const int cid = A.order[slot];
        const int a0 = A.coff[cid], n = A.coff[cid + 1] - a0;
        if (n <= 0) {
            if (threadIdx.x == 0) {
                A.energy[cid] = 0.0;
                A.iters[cid] = 0;
                A.eps[cid] = 0.0;
            }
            continue;
        }
        cluster_load(c, A, a0, n);
        cluster_lab(c, A, a0, n);
        cluster_field_any(c, A, n, damp_r2);

        // ---- induced dipoles ---------------------------------------------------------------
        int it = 0;
        double eps = 1.0e50;
        const int n3 = 3 * n;
        if (A.polarization == TDP_MUTUAL) {
            cluster_cg(c, n, A.lmax, damp_r2, A.target_eps, A.max_iter, it, eps);
        } else if (A.polarization == TDP_EXTRAPOLATED) {
            // Perturbation-theory extrapolation (RTDF.cpp:853-909).
            double* hist = c.w;                               // korder slots of 3M
            double* fld = c.w + (size_t)A.korder * 3 * c.M;   // 3M
            for (int k = threadIdx.x; k < n3; k += blockDim.x) hist[k] = c.mu[k];
            for (int o = 1; o < A.korder; o++) {
                __syncthreads();
                cluster_matvec(c, n, A.lmax, damp_r2, fld);
                for (int i = threadIdx.x; i < n; i += blockDim.x) {
                    for (int k = 0; k < 3; k++) {
                        const double v = (c.E[3 * i + k] + fld[3 * i + k]) * c.alpha[i];
                        c.mu[3 * i + k] = v;
                        hist[(size_t)o * 3 * c.M + 3 * i + k] = v;
                    }
                    set_vec(c, i, c.mu[3 * i], c.mu[3 * i + 1], c.mu[3 * i + 2]);
                }
            }
            __syncthreads();
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                for (int k = 0; k < 3; k++) {
                    double acc = 0.0;
                    for (int o = 0; o < A.korder; o++) acc += hist[(size_t)o * 3 * c.M + 3 * i + k] * A.coef[o];
                    c.mu[3 * i + k] = acc;
                }
                set_vec(c, i, c.mu[3 * i], c.mu[3 * i + 1], c.mu[3 * i + 2]);
            }
            __syncthreads();
            cluster_matvec(c, n, A.lmax, damp_r2, fld);
            double e2 = 0.0;
            for (int k = threadIdx.x; k < n3; k += blockDim.x) {
                const double dl = (c.E[k] + fld[k]) * c.alpha[k / 3] - c.mu[k];
                e2 += dl * dl;
            }
            eps = sqrt(bsum(e2, c.red) / n);
            it = A.korder;
        }
        __syncthreads();

        // ---- energy, forces, torques (RTDF.cpp:129-393) ------------------------------------
        // The operand records now carry the induced dipoles.
        for (int i = threadIdx.x; i < n; i += blockDim.x) set_vec(c, i, c.mu[3 * i], c.mu[3 * i + 1], c.mu[3 * i + 2]);
        __syncthreads();
        double* frc = c.w;
        double* trq = c.w + 3 * c.M;
        double en = 0.0;
        const bool e64 = sizeof(R) == 4 && A.fp64_passes;
        const bool lab_ok = A.rinv4_power == 0.0 && A.rinv4_fill == 0.0;
        for (int base = 0; base < n; base += blockDim.x) {
            const int na = min(n - base, (int)blockDim.x);
            const Split sp = split(na, A.lmax);
            const int i = base + sp.a;
            double f[6] = {0, 0, 0, 0, 0, 0};
            if (sp.act && e64) {
                // FP64 pair arithmetic on the FP64 records; pairs beyond the
                // damping range with unit scales take the lab-frame form.
                const EAtom<double> me{c.q64[i], c.lab64[3 * i], c.lab64[3 * i + 1], c.lab64[3 * i + 2],
                                       c.mu[3 * i], c.mu[3 * i + 1], c.mu[3 * i + 2], c.th64[i]};
                const double pix = c.pos[3 * i], piy = c.pos[3 * i + 1], piz = c.pos[3 * i + 2];
                const bool mutual = A.polarization == TDP_MUTUAL;
                for (int j = sp.l; j < n; j += sp.L) {
                    if (j == i) continue;
                    R mr, sr;
                    pair_scales(c, i, j, mr, sr);
                    const double m = mr, s = sr;
                    if (m == 0.0 && s == 0.0) continue;
                    const EAtom<double> other{c.q64[j], c.lab64[3 * j], c.lab64[3 * j + 1], c.lab64[3 * j + 2],
                                              c.mu[3 * j], c.mu[3 * j + 1], c.mu[3 * j + 2], c.th64[j]};
                    const double dx = c.pos[3 * j] - pix, dy = c.pos[3 * j + 1] - piy, dz = c.pos[3 * j + 2] - piz;
                    const double r2 = dx * dx + dy * dy + dz * dz;
                    bool yzd = fabs(dy) > 1e-5 || fabs(dz) > 1e-5;
                    if (!yzd) yzd = (piy != c.pos[3 * j + 1]) || (piz != c.pos[3 * j + 2]);
                    double fx = 0, fy = 0, fz = 0, tx = 0, ty = 0, tz = 0, e = 0;
                    if (lab_ok && m == 1.0 && s == 1.0 && !(r2 < A.damp_r2)) {
                        double gx = 0, gy = 0, gz = 0, ux = 0, uy = 0, uz = 0;
                        const double kap = mutual ? 1.0 : -1.0;
                        if (i < j)
                            pair_energy_lab<double>(dx, dy, dz, r2, yzd, me, other, kap, fx, fy, fz, tx, ty, tz, gx, gy,
                                                    gz, ux, uy, uz, e);
                        else
                            pair_energy_lab<double>(-dx, -dy, -dz, r2, yzd, other, me, kap, gx, gy, gz, ux, uy, uz, fx,
                                                    fy, fz, tx, ty, tz, e);
                        if (i > j) e = 0.0;
                    } else if (i < j) {
                        pair_energy<double, true>(dx, dy, dz, r2, yzd, me, other, m, s, A.damp_r2, A.rinv4_power,
                                                  A.rinv4_fill, mutual, fx, fy, fz, tx, ty, tz, e);
                    } else {
                        pair_energy<double, false>(-dx, -dy, -dz, r2, yzd, other, me, m, s, A.damp_r2, A.rinv4_power,
                                                   A.rinv4_fill, mutual, fx, fy, fz, tx, ty, tz, e);
                    }
                    f[0] += fx;
                    f[1] += fy;
                    f[2] += fz;
                    f[3] += tx;
                    f[4] += ty;
                    f[5] += tz;
                    en += e;
                }
            } else if (sp.act) {
                const V4 pi = c.posq[i], di = c.dipt[i], ui = c.vec[i];
                const EAtom<R> me{pi.w, di.x, di.y, di.z, ui.x, ui.y, ui.z, di.w};
                const double yi = c.pos[3 * i + 1], zi = c.pos[3 * i + 2];
                for (int j = sp.l; j < n; j += sp.L) {
                    if (j == i) continue;
                    R m, s;
                    pair_scales(c, i, j, m, s);
                    if (m == R(0) && s == R(0)) continue;
                    const V4 pj = c.posq[j], dj = c.dipt[j], uj = c.vec[j];
                    const EAtom<R> other{pj.w, dj.x, dj.y, dj.z, uj.x, uj.y, uj.z, dj.w};
                    const R dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
                    const R r2 = dx * dx + dy * dy + dz * dz;
                    // formQIRotationMatrix's test on the raw positions (RTDF.cpp:584).
                    bool yzd = fabs(dy) > R(1e-5) || fabs(dz) > R(1e-5);
                    if (!yzd) yzd = (yi != c.pos[3 * j + 1]) || (zi != c.pos[3 * j + 2]);
                    R fx = 0, fy = 0, fz = 0, tx = 0, ty = 0, tz = 0, e = 0;
                    if (i < j)
                        pair_energy<R, true>(dx, dy, dz, r2, yzd, me, other, m, s, damp_r2, rv4p, rv4f,
                                             A.polarization == TDP_MUTUAL, fx, fy, fz, tx, ty, tz, e);
                    else
                        pair_energy<R, false>(-dx, -dy, -dz, r2, yzd, other, me, m, s, damp_r2, rv4p, rv4f,
                                              A.polarization == TDP_MUTUAL, fx, fy, fz, tx, ty, tz, e);
                    f[0] += fx;
                    f[1] += fy;
                    f[2] += fz;
                    f[3] += tx;
                    f[4] += ty;
                    f[5] += tz;
                    en += e;
                }
            }
            double* pt = c.part + 6 * threadIdx.x;
            for (int k = 0; k < 6; k++) pt[k] = f[k];
            __syncthreads();
            if ((int)threadIdx.x < na) {
                const int a = base + threadIdx.x;
                for (int k = 0; k < 3; k++) {
                    frc[3 * a + k] = split_sum(c.part, 6, k, threadIdx.x, na, sp.T);
                    trq[3 * a + k] = split_sum(c.part, 6, 3 + k, threadIdx.x, na, sp.T);
                }
            }
            __syncthreads();
        }
        en = bsum(en, c.red);  // its barriers also order the frc/trq writes before the gather

        // ---- torque mapping (RTDF.cpp:915-1115), gathered per receiving atom -------------
        for (int a = threadIdx.x; a < n; a += blockDim.x) {
            const int ga = a0 + a;
            d3 F = {frc[3 * a], frc[3 * a + 1], frc[3 * a + 2]};
            for (int k = A.users_off[ga]; k < A.users_off[ga + 1]; k++) {
                const int2 u = A.users[k];
                const int fi = u.x - a0;
                const d3 T = {trq[3 * fi], trq[3 * fi + 1], trq[3 * fi + 2]};
                F = F + torque_role_force(c.pos, c.axis[fi], fi, u.y, T);
            }
            A.forces[3 * (size_t)ga] = F.x;
            A.forces[3 * (size_t)ga + 1] = F.y;
            A.forces[3 * (size_t)ga + 2] = F.z;
            for (int k = 0; k < 3; k++) A.mu_out[3 * (size_t)ga + k] = c.mu[3 * a + k];
        }
        if (threadIdx.x == 0) {
            A.energy[cid] = en;
            A.iters[cid] = it;
            A.eps[cid] = eps;
        }
    }
}


// ---------------------------------------------------------------------------
// Reverse pass (tdp_batch_adjoint): per cluster, the chain of tdp_adjoint
// (tdp_adjoint.cu) in one CTA -- torque-map VJP, pair VJPs, one adjoint solve
// of the cluster's (alpha^-1 - T) system (Mutual), the permanent-field and
// mutual-field VJPs and the rotation transpose -- from the forward's induced
// dipoles, with every per-atom vector in shared memory.  The pair VJPs run in
// FP64; the adjoint solve uses the form's matvec (FP32 pair arithmetic with
// FP64 vectors in the mixed form) to 1e-12 of the right-hand side's scale.
// ---------------------------------------------------------------------------
struct AdjArgs {
    const double* gF;   // n*3 dL/dF (NULL: zero)
    const double* gE;   // per-cluster dL/dE (NULL: zero)
    double* grads;      // n*6: dq, dalpha, dthole, dmu_mol[3]
    int* iters;         // per-cluster adjoint CG iterations
    double* eps;        // per-cluster final adjoint residual (Jacobi-step units)
    int* queue;
};

// FP64 per-atom arrays of the reverse pass, after the forward's layout.
struct AdjCl {
    double *gF, *gT, *a8, *b5, *ct, *lab, *q, *th, *muf, *amu, *lam, *etm, *part;
};
__host__ __device__ inline size_t adj_extra_doubles(int M) { return (size_t)M * 38 + 8 * 512; }

template <class R>
__host__ __device__ inline size_t batch_adjoint_smem(int M, int X, int korder) {
    return batch_smem<R>(M, X, korder) + sizeof(double) * adj_extra_doubles(M);
}

template <class R>
__device__ AdjCl carve_adj(char* base, int M, int X, int korder) {
    double* d = reinterpret_cast<double*>(base + batch_smem<R>(M, X, korder));
    AdjCl g;
    g.gF = d; d += 3 * M;
    g.gT = d; d += 3 * M;
    g.a8 = d; d += 8 * M;
    g.b5 = d; d += 5 * M;
    g.ct = d; d += M;
    g.lab = d; d += 3 * M;
    g.q = d; d += M;
    g.th = d; d += M;
    g.muf = d; d += 3 * M;
    g.amu = d; d += 3 * M;
    g.lam = d; d += 3 * M;
    g.etm = d; d += 3 * M;   // 38 M so far
    g.part = d;               // 8 per thread
    return g;
}

// out := T x over the cluster (operand records set from x).
template <class R>
__device__ __forceinline__ void cluster_apply_t(const Cl<R>& c, int n, int lmax, R damp_r2, const double* x,
                                                double* out) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) set_vec(c, i, x[3 * i], x[3 * i + 1], x[3 * i + 2]);
    __syncthreads();
    cluster_matvec(c, n, lmax, damp_r2, out);
}

template <class R>
__global__ void __launch_bounds__(512) k_batch_adjoint(BatchArgs A, AdjArgs G) {
    extern __shared__ __align__(32) char smem_raw[];
    const Cl<R> c = carve<R>(smem_raw, A.max_atoms, A.max_exc, A.korder);
    const AdjCl g = carve_adj<R>(smem_raw, A.max_atoms, A.max_exc, A.korder);
    __shared__ int s_slot;
    const R damp_r2 = (R)A.damp_r2;
    PairParams P{};
    P.periodic = 0;
    P.damp_r2 = (float)A.damp_r2;
    P.rinv4_power = (float)A.rinv4_power;
    P.rinv4_fill = (float)A.rinv4_fill;
    P.mutual = A.polarization == TDP_MUTUAL ? 1 : 0;
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) s_slot = atomicAdd(G.queue, 1);
        __syncthreads();
        const int slot = s_slot;
        if (slot >= A.num_clusters) break;
        const int cid = A.order[slot];
        const int a0 = A.coff[cid], n = A.coff[cid + 1] - a0;
        if (n <= 0) {
            if (threadIdx.x == 0) {
                G.iters[cid] = 0;
                G.eps[cid] = 0.0;
            }
            continue;
        }
        P.n = n;
        cluster_load(c, A, a0, n);
        cluster_lab(c, A, a0, n);
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const int gi = a0 + i;
            double Rm[3][3], sy;
            frame_rows(c.pos, c.axis[i], i, Rm, sy);
            const double* dm = A.dip_mol + 3 * (size_t)gi;
            const double d0 = dm[0], d1 = sy * dm[1], d2 = dm[2];
            for (int k = 0; k < 3; k++) {
                g.lab[3 * i + k] = 0.0 + d0 * Rm[0][k] + d1 * Rm[1][k] + d2 * Rm[2][k];
                g.muf[3 * i + k] = A.mu_out[3 * (size_t)gi + k];
                g.gF[3 * i + k] = G.gF ? G.gF[3 * (size_t)gi + k] : 0.0;
            }
            g.q[i] = A.charge[gi];
            g.th[i] = A.thole[gi];
        }
        const double gE = G.gE ? G.gE[cid] : 0.0;
        // Permanent field of the forward into c.E (also sets c.mu = alpha E).
        cluster_field_any(c, A, n, damp_r2);
        for (int k = threadIdx.x; k < 3 * n; k += blockDim.x) g.etm[k] = c.E[k];

        // ---- g_tau = M^T g (k_torque_vjp) -------------------------------------------------
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const int4 ax = c.axis[i];
            double o[3] = {0.0, 0.0, 0.0};
            if (ax.x != TDP_NO_AXIS_TYPE) {
                const int atoms[4] = {i, ax.y, ax.z, ax.w};
                for (int role = 0; role < 4; role++) {
                    const int at = atoms[role];
                    if (at < 0) continue;
                    if (role == 2 && ax.x == TDP_ZONLY) continue;
                    if (role == 3 && !(ax.x == TDP_ZBISECT || ax.x == TDP_THREEFOLD)) continue;
                    for (int k = 0; k < 3; k++) {
                        const d3 e = {k == 0 ? 1.0 : 0.0, k == 1 ? 1.0 : 0.0, k == 2 ? 1.0 : 0.0};
                        const d3 f = torque_role_force(c.pos, ax, i, role, e);
                        o[k] += f.x * g.gF[3 * at] + f.y * g.gF[3 * at + 1] + f.z * g.gF[3 * at + 2];
                    }
                }
            }
            for (int k = 0; k < 3; k++) g.gT[3 * i + k] = o[k];
        }
        __syncthreads();
        const adj::AtomData AD{c.pos, g.q, g.lab, g.muf, g.th, nullptr};

        // ---- a = pair VJPs (k_pair_vjp): 8 per atom ----------------------------------------
        for (int base = 0; base < n; base += blockDim.x) {
            const int na = min(n - base, (int)blockDim.x);
            const Split sp = split(na, A.lmax);
            const int i = base + sp.a;
            double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            if (sp.act)
                for (int j = sp.l; j < n; j += sp.L) {
                    if (j == i) continue;
                    R m, s;
                    pair_scales(c, i, j, m, s);
                    if (m == R(0) && s == R(0)) continue;
                    adj::visit_pair(P, AD, g.gF, g.gT, gE, i, j, (double)m, (double)s, acc);
                }
            for (int k = 0; k < 8; k++) g.part[8 * threadIdx.x + k] = acc[k];
            __syncthreads();
            if ((int)threadIdx.x < na)
                for (int k = 0; k < 8; k++)
                    g.a8[8 * (base + threadIdx.x) + k] = split_sum(g.part, 8, k, threadIdx.x, na, sp.T);
            __syncthreads();
        }
        double s2 = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x)
            for (int k = 0; k < 3; k++) {
                const double v = g.a8[8 * i + 4 + k];
                g.amu[3 * i + k] = v;
                s2 += (c.alpha[i] * v) * (c.alpha[i] * v);
            }
        s2 = bsum(s2, c.red);

        // ---- adjoint solve and the field VJPs ----------------------------------------------
        int it = 0;
        double eps = 0.0;
        if (A.polarization == TDP_MUTUAL) {
            // E + T mu of the forward, for the polarizability gradient.
            cluster_apply_t(c, n, A.lmax, damp_r2, g.muf, g.lam);
            for (int k = threadIdx.x; k < 3 * n; k += blockDim.x) g.etm[k] += g.lam[k];
            // A lambda = a_mu: the forward's CG with E := a_mu, from lambda = alpha a_mu.
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                for (int k = 0; k < 3; k++) {
                    c.E[3 * i + k] = g.amu[3 * i + k];
                    c.mu[3 * i + k] = c.alpha[i] * g.amu[3 * i + k];
                }
                set_vec(c, i, c.mu[3 * i], c.mu[3 * i + 1], c.mu[3 * i + 2]);
            }
            __syncthreads();
            // 1e-12 of the right-hand side's scale in FP64; 1e-6 in the mixed
            // form, whose true residual is limited by the FP32 matvec near 1e-7.
            const double target = fmax(sqrt(s2 / n) * (sizeof(R) == 8 ? 1e-12 : 1e-6), 1e-300);
            eps = 1.0e50;
            cluster_cg(c, n, A.lmax, damp_r2, target, A.max_iter > 1000 ? A.max_iter : 1000, it, eps);
            __syncthreads();
            for (int k = threadIdx.x; k < 3 * n; k += blockDim.x) g.lam[k] = c.mu[k];
            __syncthreads();
            // a_mu + T lambda (into amu) for the polarizability gradient.
            cluster_apply_t(c, n, A.lmax, damp_r2, g.lam, c.E);
            for (int k = threadIdx.x; k < 3 * n; k += blockDim.x) g.amu[k] += c.E[k];
        } else {
            // Direct: mu = alpha E, so lambda = alpha a_mu and dL/dalpha = a_mu . E.
            for (int i = threadIdx.x; i < n; i += blockDim.x)
                for (int k = 0; k < 3; k++) g.lam[3 * i + k] = c.alpha[i] * g.amu[3 * i + k];
        }
        __syncthreads();
        // b = d/d(q, lab, t) of lambda . Efix (k_fixed_vjp), c_t = d/dt of lambda^T T mu.
        for (int base = 0; base < n; base += blockDim.x) {
            const int na = min(n - base, (int)blockDim.x);
            const Split sp = split(na, A.lmax);
            const int k = base + sp.a;
            double acc[6] = {0, 0, 0, 0, 0, 0};
            if (sp.act)
                for (int j = sp.l; j < n; j += sp.L) {
                    if (j == k) continue;
                    R m, s;
                    pair_scales(c, k, j, m, s);
                    if (m != R(0)) adj::fixed_vjp_visit(P, AD, g.lam, k, j, (double)m, acc);
                    if (A.polarization == TDP_MUTUAL && s != R(0))
                        acc[5] += adj::matvec_t_visit(P, AD, g.lam, k, j, (double)s);
                }
            for (int u = 0; u < 6; u++) g.part[8 * threadIdx.x + u] = acc[u];
            __syncthreads();
            if ((int)threadIdx.x < na) {
                const int a = base + threadIdx.x;
                for (int u = 0; u < 5; u++) g.b5[5 * a + u] = split_sum(g.part, 8, u, threadIdx.x, na, sp.T);
                g.ct[a] = split_sum(g.part, 8, 5, threadIdx.x, na, sp.T);
            }
            __syncthreads();
        }

        // ---- rotation transpose and assembly (k_rotation_vjp, k_adjoint_assemble) ---------
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const int gi = a0 + i;
            double Rm[3][3], sy;
            frame_rows(c.pos, c.axis[i], i, Rm, sy);
            double gl[3];
            for (int k = 0; k < 3; k++) gl[k] = g.a8[8 * i + 1 + k] + g.b5[5 * i + 1 + k];
            double* o = G.grads + 6 * (size_t)gi;
            o[0] = g.a8[8 * i] + g.b5[5 * i];
            double ga = 0.0;
            for (int k = 0; k < 3; k++) ga += g.amu[3 * i + k] * g.etm[3 * i + k];
            o[1] = ga;
            o[2] = g.a8[8 * i + 7] + g.b5[5 * i + 4] + g.ct[i];
            for (int j = 0; j < 3; j++) {
                const double v = Rm[j][0] * gl[0] + Rm[j][1] * gl[1] + Rm[j][2] * gl[2];
                o[3 + j] = j == 1 ? sy * v : v;
            }
        }
        if (threadIdx.x == 0) {
            G.iters[cid] = it;
            G.eps[cid] = eps;
        }
    }
}

}  // namespace
}  // namespace tdp

using namespace tdp;

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
struct tdp_batch {
    int n = 0, nc = 0;
    int precision = TDP_PRECISION_MIXED;
    int polarization = TDP_MUTUAL;
    int max_atoms = 0, max_exc = 0;
    std::vector<int> coff;
    std::vector<double> extrap;
    BatchArgs args{};
    std::vector<void*> owned;
    cudaStream_t stream = nullptr;
    int device = 0, num_sms = 148;
    size_t smem_optin = 0;
    // Tile shape: CTA size, largest lanes per atom, CTAs in the persistent grid.
    bool tuned = false;
    int threads = 128, lmax = 8, ctas = 148;
    double tile_ms = 0.0;
    std::vector<double> tune_ms;  // per candidate, in tdp_batch_tile_candidates order
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0.0;
    bool have_results = false;
    // Reverse pass (allocated on the first tdp_batch_adjoint).
    AdjArgs adj{};
    int adj_ctas = 0;
    std::string err;
};

namespace {

thread_local std::string g_batch_create_error;

struct TileShape {
    int threads, lmax;
};
const TileShape kShapes[] = {{64, 4},  {64, 16},  {128, 4},  {128, 8},  {128, 16}, {128, 32},
                             {256, 4}, {256, 8},  {256, 16}, {256, 32}, {512, 8},  {512, 32}};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);

int batch_fail(tdp_batch* b, const TdpError& e) {
    if (b) b->err = e.msg;
    else g_batch_create_error = e.msg;
    return e.code;
}

size_t smem_for(const tdp_batch* b) {
    int korder = std::max(1, (int)b->extrap.size());
    int M = std::max(1, b->max_atoms);
    return b->precision == TDP_PRECISION_DOUBLE ? batch_smem<double>(M, b->max_exc, korder)
                                                : batch_smem<float>(M, b->max_exc, korder);
}

const void* kernel_for(const tdp_batch* b) {
    return b->precision == TDP_PRECISION_DOUBLE ? (const void*)k_batch<double> : (const void*)k_batch<float>;
}

// CTAs of the persistent grid for a CTA size: every resident slot, at most one per cluster.
int grid_for(tdp_batch* b, int threads) {
    size_t smem = smem_for(b);
    const void* k = kernel_for(b);
    TDP_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    TDP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem));
    if (per_sm < 1) return 0;
    return std::max(1, std::min(b->nc, per_sm * b->num_sms));
}

void launch(tdp_batch* b, int threads, int lmax, int ctas, cudaStream_t st) {
    BatchArgs a = b->args;
    a.lmax = lmax;
    size_t smem = smem_for(b);
    TDP_CUDA(cudaMemsetAsync(a.queue, 0, sizeof(int), st));
    if (b->precision == TDP_PRECISION_DOUBLE) k_batch<double><<<ctas, threads, smem, st>>>(a);
    else k_batch<float><<<ctas, threads, smem, st>>>(a);
    TDP_CUDA(cudaGetLastError());
}

void drop_graph(tdp_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

void build_graph(tdp_batch* b) {
    drop_graph(b);
    cudaStream_t cap = nullptr;
    TDP_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        try {
            launch(b, b->threads, b->lmax, b->ctas, cap);
        } catch (const TdpError&) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(cap, &g);
            if (g) cudaGraphDestroy(g);
            cudaStreamDestroy(cap);
            throw;
        }
        e = cudaStreamEndCapture(cap, &b->graph);
    }
    cudaStreamDestroy(cap);
    if (e != cudaSuccess) throw TdpError{TDP_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e)};
    TDP_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
}

double time_launch(tdp_batch* b, int threads, int lmax, int ctas, int reps) {
    TDP_CUDA(cudaEventRecord(b->ev0, b->stream));
    for (int r = 0; r < reps; r++) launch(b, threads, lmax, ctas, b->stream);
    TDP_CUDA(cudaEventRecord(b->ev1, b->stream));
    TDP_CUDA(cudaEventSynchronize(b->ev1));
    float ms = 0.f;
    TDP_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    return ms / reps;
}

// The autotuner: time every tile shape that fits on the batch (one warm-up
// launch, then two timed) and keep the fastest.  TDP_BATCH_TILE="threads,lanes"
// pins the shape instead.
void autotune(tdp_batch* b) {
    b->tune_ms.assign(kNumShapes, -1.0);
    int pin_t = 0, pin_l = 0;
    if (const char* env = getenv("TDP_BATCH_TILE")) sscanf(env, "%d,%d", &pin_t, &pin_l);
    double best = 1e300;
    int best_k = -1;
    for (int k = 0; k < kNumShapes; k++) {
        const TileShape s = kShapes[k];
        if (pin_t && (s.threads != pin_t || s.lmax != pin_l)) continue;
        int ctas = grid_for(b, s.threads);
        if (ctas <= 0) continue;
        launch(b, s.threads, s.lmax, ctas, b->stream);
        double ms = time_launch(b, s.threads, s.lmax, ctas, 2);
        b->tune_ms[k] = ms;
        if (ms < best) {
            best = ms;
            best_k = k;
        }
    }
    if (best_k < 0) throw TdpError{TDP_ERR_UNSUPPORTED, "no tile shape fits the largest cluster"};
    b->threads = kShapes[best_k].threads;
    b->lmax = kShapes[best_k].lmax;
    b->ctas = grid_for(b, b->threads);
    b->tile_ms = best;
    b->tuned = true;
    build_graph(b);
}

}  // namespace

extern "C" {

const char* tdp_batch_last_error(const tdp_batch* b) { return b ? b->err.c_str() : g_batch_create_error.c_str(); }

void tdp_batch_destroy(tdp_batch* b) {
    if (!b) return;
    drop_graph(b);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    for (void* p : b->owned) cudaFree(p);
    delete b;
}

int tdp_batch_create(const tdp_system_desc* desc, int32_t num_clusters, const int32_t* cluster_offsets,
                     tdp_batch** out) {
    if (!out) return TDP_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    tdp_batch* b = new tdp_batch();
    try {
        if (!desc) throw TdpError{TDP_ERR_INVALID_ARGUMENT, "desc is NULL"};
        const int n = desc->num_particles;
        if (n < 0 || num_clusters < 0) throw TdpError{TDP_ERR_INVALID_ARGUMENT, "negative size"};
        if (!cluster_offsets) throw TdpError{TDP_ERR_INVALID_ARGUMENT, "cluster_offsets is NULL"};
        if (n > 0 && (!desc->charges || !desc->molecular_dipoles || !desc->polarizabilities ||
                      !desc->thole_damping || !desc->axis_types || !desc->atom_z || !desc->atom_x || !desc->atom_y))
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, "a per-particle array is NULL"};
        if (desc->nonbonded_method != TDP_NO_CUTOFF)
            throw TdpError{TDP_ERR_UNSUPPORTED, "cluster batches are isolated systems: NoCutoff only"};
        if (desc->polarization_type < 0 || desc->polarization_type > 2)
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, "Polarization type not recognized."};
        if (desc->precision != TDP_PRECISION_MIXED && desc->precision != TDP_PRECISION_DOUBLE)
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, "unknown precision"};
        if (desc->solver != TDP_SOLVER_CG)
            throw TdpError{TDP_ERR_UNSUPPORTED, "cluster batches solve Mutual polarization by conjugate gradients"};
        if (cluster_offsets[0] != 0 || cluster_offsets[num_clusters] != n)
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, "cluster_offsets must run from 0 to num_particles"};
        for (int c = 0; c < num_clusters; c++)
            if (cluster_offsets[c + 1] < cluster_offsets[c])
                throw TdpError{TDP_ERR_INVALID_ARGUMENT, "cluster_offsets must be non-decreasing"};
        validate_axes(n, desc->axis_types, desc->atom_z, desc->atom_x, desc->atom_y);

        b->n = n;
        b->nc = num_clusters;
        b->precision = desc->precision;
        b->polarization = desc->polarization_type;
        b->coff.assign(cluster_offsets, cluster_offsets + num_clusters + 1);
        std::vector<int> cl_of(n);
        for (int c = 0; c < num_clusters; c++)
            for (int i = b->coff[c]; i < b->coff[c + 1]; i++) cl_of[i] = c;
        auto same = [&](int i, int j, const char* what) {
            if (j >= 0 && cl_of[j] != cl_of[i]) {
                char buf[200];
                snprintf(buf, sizeof buf, "particle %d: %s particle %d lies in another cluster", i, what, j);
                throw TdpError{TDP_ERR_INVALID_ARGUMENT, buf};
            }
        };
        std::vector<int> axis(4 * (size_t)n);
        for (int i = 0; i < n; i++) {
            axis[4 * i] = desc->axis_types[i];
            axis[4 * i + 1] = desc->atom_z[i];
            axis[4 * i + 2] = desc->atom_x[i];
            axis[4 * i + 3] = desc->atom_y[i];
            if (desc->axis_types[i] != TDP_NO_AXIS_TYPE) {
                same(i, desc->atom_z[i], "axis");
                same(i, desc->atom_x[i], "axis");
                if (desc->axis_types[i] == TDP_ZBISECT || desc->axis_types[i] == TDP_THREEFOLD)
                    same(i, desc->atom_y[i], "axis");
            }
        }
        auto exc = covalent_exceptions(n, desc->covalent12_offsets, desc->covalent12_atoms,
                                       desc->covalent13_offsets, desc->covalent13_atoms);
        std::vector<int> eoff(n + 1, 0), ej;
        std::vector<double> em, es;
        for (int i = 0; i < n; i++) {
            for (auto& t : exc[i]) {
                same(i, std::get<0>(t), "covalent");
                ej.push_back(std::get<0>(t));
                em.push_back(std::get<1>(t));
                es.push_back(std::get<2>(t));
            }
            eoff[i + 1] = (int)ej.size();
        }
        std::vector<int> uoff;
        std::vector<int2> users;
        torque_users(n, axis, uoff, users);

        std::vector<int> order(num_clusters);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
            return b->coff[x + 1] - b->coff[x] > b->coff[y + 1] - b->coff[y];
        });
        for (int c = 0; c < num_clusters; c++) {
            b->max_atoms = std::max(b->max_atoms, b->coff[c + 1] - b->coff[c]);
            b->max_exc = std::max(b->max_exc, eoff[b->coff[c + 1]] - eoff[b->coff[c]]);
        }
        if (desc->num_extrapolation_coefficients > 0 && desc->extrapolation_coefficients)
            b->extrap.assign(desc->extrapolation_coefficients,
                             desc->extrapolation_coefficients + desc->num_extrapolation_coefficients);
        else
            b->extrap = {-0.154, 0.017, 0.658, 0.474};  // RTDF.cpp:857-864

        TDP_CUDA(cudaGetDevice(&b->device));
        TDP_CUDA(cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device));
        int optin = 0;
        TDP_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device));
        b->smem_optin = (size_t)optin;
        if (smem_for(b) > b->smem_optin) {
            char buf[220];
            snprintf(buf, sizeof buf,
                     "largest cluster (%d atoms, %d exceptions) needs %zu bytes of shared memory; %d available",
                     b->max_atoms, b->max_exc, smem_for(b), optin);
            throw TdpError{TDP_ERR_UNSUPPORTED, buf};
        }

        BatchArgs& a = b->args;
        a.num_clusters = num_clusters;
        a.max_atoms = std::max(1, b->max_atoms);
        a.max_exc = b->max_exc;
        a.korder = std::max(1, (int)b->extrap.size());
        a.polarization = b->polarization;
        a.max_iter = std::max(0, desc->mutual_max_iterations);
        a.target_eps = desc->mutual_target_epsilon;
        std::vector<double> th(desc->thole_damping, desc->thole_damping + n);
        a.damp_r2 = damp_radius2(th);
        const bool r4 = (desc->flags & TDP_FLAG_DD_FORCE_R4) != 0;
        a.rinv4_power = r4 ? 1.0 : 0.0;
        a.rinv4_fill = 0.0;
        // TDP_BATCH_FP32_PASSES=1 runs every pair pass of the mixed form in
        // FP32 (for comparisons).
        a.fp64_passes = 1;
        if (const char* env = getenv("TDP_BATCH_FP32_PASSES"))
            if (atoi(env) == 1) a.fp64_passes = 0;

        auto& o = b->owned;
        int* d_order = dalloc<int>(num_clusters, o);
        int* d_coff = dalloc<int>(num_clusters + 1, o);
        double* d_pos = dalloc<double>(3 * (size_t)n, o);
        double* d_q = dalloc<double>(n, o);
        double* d_dm = dalloc<double>(3 * (size_t)n, o);
        double* d_al = dalloc<double>(n, o);
        double* d_th = dalloc<double>(n, o);
        int4* d_ax = dalloc<int4>(n, o);
        int* d_eoff = dalloc<int>(n + 1, o);
        int* d_ej = dalloc<int>(ej.size(), o);
        double* d_em = dalloc<double>(em.size(), o);
        double* d_es = dalloc<double>(es.size(), o);
        int* d_uoff = dalloc<int>(n + 1, o);
        int2* d_users = dalloc<int2>(users.size(), o);
        double* d_coef = dalloc<double>(b->extrap.size(), o);
        a.queue = dalloc<int>(1, o);
        a.forces = dalloc<double>(3 * (size_t)n, o);
        a.mu_out = dalloc<double>(3 * (size_t)n, o);
        a.energy = dalloc<double>(num_clusters, o);
        a.iters = dalloc<int>(num_clusters, o);
        a.eps = dalloc<double>(num_clusters, o);
        upload(d_order, order.data(), sizeof(int) * num_clusters);
        upload(d_coff, b->coff.data(), sizeof(int) * (num_clusters + 1));
        upload(d_q, desc->charges, sizeof(double) * n);
        upload(d_dm, desc->molecular_dipoles, sizeof(double) * 3 * n);
        upload(d_al, desc->polarizabilities, sizeof(double) * n);
        upload(d_th, desc->thole_damping, sizeof(double) * n);
        upload(d_ax, axis.data(), sizeof(int) * 4 * n);
        upload(d_eoff, eoff.data(), sizeof(int) * (n + 1));
        upload(d_ej, ej.data(), sizeof(int) * ej.size());
        upload(d_em, em.data(), sizeof(double) * em.size());
        upload(d_es, es.data(), sizeof(double) * es.size());
        upload(d_uoff, uoff.data(), sizeof(int) * (n + 1));
        upload(d_users, users.data(), sizeof(int2) * users.size());
        upload(d_coef, b->extrap.data(), sizeof(double) * b->extrap.size());
        a.order = d_order;
        a.coff = d_coff;
        a.pos = d_pos;
        a.charge = d_q;
        a.dip_mol = d_dm;
        a.alpha = d_al;
        a.thole = d_th;
        a.axis = d_ax;
        a.exc_off = d_eoff;
        a.exc_j = d_ej;
        a.exc_m = d_em;
        a.exc_s = d_es;
        a.users_off = d_uoff;
        a.users = d_users;
        a.coef = d_coef;
        TDP_CUDA(cudaEventCreate(&b->ev0));
        TDP_CUDA(cudaEventCreate(&b->ev1));
    } catch (const TdpError& e) {
        int code = batch_fail(nullptr, e);
        tdp_batch_destroy(b);
        return code;
    }
    *out = b;
    return TDP_OK;
}

int tdp_batch_set_stream(tdp_batch* b, void* stream) {
    if (!b) return TDP_ERR_INVALID_ARGUMENT;
    b->stream = static_cast<cudaStream_t>(stream);
    return TDP_OK;
}

int tdp_batch_compute(tdp_batch* b, const double* positions, int32_t on_device, double* forces, double* energies) {
    if (!b) return TDP_ERR_INVALID_ARGUMENT;
    try {
        if (b->n > 0 && !positions) throw TdpError{TDP_ERR_INVALID_ARGUMENT, "positions is NULL"};
        if (b->nc == 0) return TDP_OK;
        cudaStream_t st = b->stream;
        const size_t n3 = 3 * (size_t)b->n;
        if (n3)
            TDP_CUDA(cudaMemcpyAsync((void*)b->args.pos, positions, sizeof(double) * n3,
                                     on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
        if (!b->tuned) autotune(b);
        TDP_CUDA(cudaEventRecord(b->ev0, st));
        TDP_CUDA(cudaGraphLaunch(b->exec, st));
        TDP_CUDA(cudaEventRecord(b->ev1, st));
        const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        if (forces && n3) TDP_CUDA(cudaMemcpyAsync(forces, b->args.forces, sizeof(double) * n3, kind, st));
        if (energies) TDP_CUDA(cudaMemcpyAsync(energies, b->args.energy, sizeof(double) * b->nc, kind, st));
        TDP_CUDA(cudaEventSynchronize(b->ev1));
        float ms = 0.f;
        TDP_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
        b->last_ms = ms;
        if (!on_device) TDP_CUDA(cudaStreamSynchronize(st));
        TDP_CUDA(cudaGetLastError());
        b->have_results = true;
    } catch (const TdpError& e) {
        return batch_fail(b, e);
    }
    return TDP_OK;
}

int tdp_batch_get_induced_dipoles(tdp_batch* b, double* out) {
    if (!b || !out) return TDP_ERR_INVALID_ARGUMENT;
    try {
        if (!b->have_results) throw TdpError{TDP_ERR_INVALID_ARGUMENT, "no tdp_batch_compute yet"};
        if (b->n)
            TDP_CUDA(cudaMemcpyAsync(out, b->args.mu_out, sizeof(double) * 3 * b->n, cudaMemcpyDeviceToHost, b->stream));
        TDP_CUDA(cudaStreamSynchronize(b->stream));
    } catch (const TdpError& e) {
        return batch_fail(b, e);
    }
    return TDP_OK;
}

int tdp_batch_solver_stats(tdp_batch* b, int32_t* iterations, double* epsilons) {
    if (!b) return TDP_ERR_INVALID_ARGUMENT;
    try {
        if (!b->have_results) throw TdpError{TDP_ERR_INVALID_ARGUMENT, "no tdp_batch_compute yet"};
        if (iterations && b->nc)
            TDP_CUDA(cudaMemcpyAsync(iterations, b->args.iters, sizeof(int) * b->nc, cudaMemcpyDeviceToHost, b->stream));
        if (epsilons && b->nc)
            TDP_CUDA(cudaMemcpyAsync(epsilons, b->args.eps, sizeof(double) * b->nc, cudaMemcpyDeviceToHost, b->stream));
        TDP_CUDA(cudaStreamSynchronize(b->stream));
    } catch (const TdpError& e) {
        return batch_fail(b, e);
    }
    return TDP_OK;
}

int tdp_batch_tile(const tdp_batch* b, int32_t* threads, int32_t* lanes, int32_t* ctas, double* last_ms) {
    if (!b) return TDP_ERR_INVALID_ARGUMENT;
    if (threads) *threads = b->tuned ? b->threads : 0;
    if (lanes) *lanes = b->tuned ? b->lmax : 0;
    if (ctas) *ctas = b->tuned ? b->ctas : 0;
    if (last_ms) *last_ms = b->last_ms;
    return TDP_OK;
}

int tdp_batch_update_params(tdp_batch* b, const double* charges, const double* molecular_dipoles,
                            const double* polarizabilities, const double* thole_damping, int32_t on_device) {
    if (!b) return TDP_ERR_INVALID_ARGUMENT;
    try {
        const size_t n = (size_t)b->n;
        if (n == 0) return TDP_OK;
        if (!charges || !molecular_dipoles || !polarizabilities || !thole_damping)
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, "a per-particle array is NULL"};
        cudaStream_t st = b->stream;
        const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        BatchArgs& a = b->args;
        TDP_CUDA(cudaMemcpyAsync((void*)a.charge, charges, sizeof(double) * n, kind, st));
        TDP_CUDA(cudaMemcpyAsync((void*)a.dip_mol, molecular_dipoles, sizeof(double) * 3 * n, kind, st));
        TDP_CUDA(cudaMemcpyAsync((void*)a.alpha, polarizabilities, sizeof(double) * n, kind, st));
        TDP_CUDA(cudaMemcpyAsync((void*)a.thole, thole_damping, sizeof(double) * n, kind, st));
        // The damping radius follows the largest Thole factor.
        std::vector<double> th(n);
        if (on_device) {
            TDP_CUDA(cudaMemcpyAsync(th.data(), thole_damping, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
            TDP_CUDA(cudaStreamSynchronize(st));
        } else {
            th.assign(thole_damping, thole_damping + n);
        }
        const double dr2 = damp_radius2(th);
        if (dr2 != a.damp_r2) {
            a.damp_r2 = dr2;
            if (b->tuned) build_graph(b);
        }
        b->have_results = false;
    } catch (const TdpError& e) {
        return batch_fail(b, e);
    }
    return TDP_OK;
}

int tdp_batch_adjoint(tdp_batch* b, const double* dL_dF, const double* dL_dE, int32_t on_device, double* grads) {
    if (!b || !grads) return TDP_ERR_INVALID_ARGUMENT;
    try {
        if (b->nc == 0 || b->n == 0) return TDP_OK;
        if (!b->have_results) throw TdpError{TDP_ERR_INVALID_ARGUMENT, "tdp_batch_adjoint needs a previous tdp_batch_compute"};
        if (b->polarization == TDP_EXTRAPOLATED)
            throw TdpError{TDP_ERR_UNSUPPORTED, "tdp_batch_adjoint supports Direct and Mutual polarization"};
        cudaStream_t st = b->stream;
        const size_t n = (size_t)b->n;
        const int korder = std::max(1, (int)b->extrap.size());
        const int M = std::max(1, b->max_atoms);
        const size_t smem = b->precision == TDP_PRECISION_DOUBLE ? batch_adjoint_smem<double>(M, b->max_exc, korder)
                                                                 : batch_adjoint_smem<float>(M, b->max_exc, korder);
        if (smem > b->smem_optin) {
            char buf[200];
            snprintf(buf, sizeof buf, "the reverse pass of the largest cluster (%d atoms) needs %zu bytes of shared "
                     "memory; %zu available", b->max_atoms, smem, b->smem_optin);
            throw TdpError{TDP_ERR_UNSUPPORTED, buf};
        }
        const void* kern = b->precision == TDP_PRECISION_DOUBLE ? (const void*)k_batch_adjoint<double>
                                                                : (const void*)k_batch_adjoint<float>;
        const int threads = b->tuned ? b->threads : 128;
        const int lmax = b->tuned ? b->lmax : 8;
        AdjArgs& g = b->adj;
        if (!g.grads) {
            auto& o = b->owned;
            g.gF = dalloc<double>(3 * n, o);
            g.gE = dalloc<double>((size_t)b->nc, o);
            g.grads = dalloc<double>(6 * n, o);
            g.iters = dalloc<int>((size_t)b->nc, o);
            g.eps = dalloc<double>((size_t)b->nc, o);
            g.queue = dalloc<int>(1, o);
            TDP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            int per_sm = 0;
            TDP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
            if (per_sm < 1) throw TdpError{TDP_ERR_UNSUPPORTED, "the reverse pass does not fit an SM"};
            b->adj_ctas = std::max(1, std::min(b->nc, per_sm * b->num_sms));
        }
        const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        AdjArgs args = g;
        if (dL_dF) TDP_CUDA(cudaMemcpyAsync((void*)g.gF, dL_dF, sizeof(double) * 3 * n, kind, st));
        else args.gF = nullptr;
        if (dL_dE) TDP_CUDA(cudaMemcpyAsync((void*)g.gE, dL_dE, sizeof(double) * b->nc, kind, st));
        else args.gE = nullptr;
        TDP_CUDA(cudaMemsetAsync(g.queue, 0, sizeof(int), st));
        BatchArgs a = b->args;
        a.lmax = lmax;
        if (b->precision == TDP_PRECISION_DOUBLE) k_batch_adjoint<double><<<b->adj_ctas, threads, smem, st>>>(a, args);
        else k_batch_adjoint<float><<<b->adj_ctas, threads, smem, st>>>(a, args);
        TDP_CUDA(cudaGetLastError());
        TDP_CUDA(cudaMemcpyAsync(grads, g.grads, sizeof(double) * 6 * n,
                                 on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
        if (!on_device) TDP_CUDA(cudaStreamSynchronize(st));
    } catch (const TdpError& e) {
        return batch_fail(b, e);
    }
    return TDP_OK;
}

int tdp_batch_adjoint_stats(tdp_batch* b, int32_t* iterations, double* epsilons) {
    if (!b) return TDP_ERR_INVALID_ARGUMENT;
    try {
        if (!b->adj.grads) throw TdpError{TDP_ERR_INVALID_ARGUMENT, "no tdp_batch_adjoint yet"};
        if (iterations && b->nc)
            TDP_CUDA(cudaMemcpyAsync(iterations, b->adj.iters, sizeof(int) * b->nc, cudaMemcpyDeviceToHost, b->stream));
        if (epsilons && b->nc)
            TDP_CUDA(cudaMemcpyAsync(epsilons, b->adj.eps, sizeof(double) * b->nc, cudaMemcpyDeviceToHost, b->stream));
        TDP_CUDA(cudaStreamSynchronize(b->stream));
    } catch (const TdpError& e) {
        return batch_fail(b, e);
    }
    return TDP_OK;
}

int tdp_batch_tile_candidates(const tdp_batch* b, int32_t capacity, int32_t* threads, int32_t* lanes, double* ms) {
    if (!b) return TDP_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < kNumShapes && k < capacity; k++) {
        if (threads) threads[k] = kShapes[k].threads;
        if (lanes) lanes[k] = kShapes[k].lmax;
        if (ms) ms[k] = k < (int)b->tune_ms.size() ? b->tune_ms[k] : -1.0;
    }
    return kNumShapes;
}

}  // extern "C"
