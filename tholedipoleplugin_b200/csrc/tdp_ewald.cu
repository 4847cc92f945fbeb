// tdp_ewald.cu -- the Ewald mode of the box path (TDP_FLAG_EWALD).
//
// Model (oracle/ewald.py restates it in FP64): permanent multipoles P = (q, p),
// induced dipoles U = (0, mu), total T = (q, p + mu).  For a radial kernel set
// K = (K0, K1, K2, K3) and r = r_j - r_i, the pair energy of two charge+dipole
// sites is
//     E = q_i q_j K0 + [q_j (d_i.r) - q_i (d_j.r) + d_i.d_j] K1 - (d_i.r)(d_j.r) K2,
// its force on i  -[r (G0 K1 + G1 K2 + G2 K3) - K1 (q_j d_i - q_i d_j) + K2 ((d_j.r) d_i + (d_i.r) d_j)],
// and the field at i  -K1 (q_j r + d_j) + K2 (d_j.r) r.
// Bare kernels b = (1/r, 1/r^3, 3/r^5, 15/r^7), Ewald real-space kernels from
// erfc(alpha r) (Be), Thole factors l3, l5, l7 of the reference's damping
// (ReferenceTholeDipoleForce.cpp:646-676, "RTDF.cpp").  The energy functional
//     sum_pairs [ m E(P,P; b) + m (E(P,U) + E(U,P))(l b) + s E(U,U; l b) ] + 1/2 sum |mu|^2/alpha
// is summed over all periodic images: reciprocal space takes every bare term
// (smooth PME), real space the erfc part within the cutoff, and the nearest
// image of each pair the corrections for its scales and damping.  For an
// unscaled pair (m = s = 1) those corrections are -E(T,T; Kd) + E(P,P; Kd) with
// Kd = (0, (1-l3) b1, (1-l5) b2, (1-l7) b3), zero beyond the damping range,
// which the mode requires to lie inside the cutoff.  Scaled pairs (covalent
// partners) are masked out of the tile walk and evaluated separately in FP64.
//
// Work layout.  Atoms are in the spatially sorted slots of the field kernels
// (molecules along a Morton curve, 32-atom tiles).  A neighbour list of tiles
// (J tiles whose bounding box comes within the cutoff of I's, minimum image)
// is rebuilt at every evaluation.  One warp owns an I tile (lane = atom), walks
// its J tiles with the J records staged in shared memory and broadcast one per
// step, and keeps only its own side: every ordered pair is visited once, so
// each output is written by one lane in a fixed order and no atomics are
// needed.  Real-space results go to partial slot 0, reciprocal space (plus
// self terms) to slot 1; the solver kernels add the two slots.
//
// PME: order-5 cardinal B-splines, u_k = K_k frac(x_k / L_k); a site spreads
// q Th + d.grad Th onto the 125 points floor(u) - (0..4); the mixed form
// accumulates in 64-bit fixed point (2^-32 e, deterministic), the plain form
// in FP64.  R2C FFT, multiplication by C(m) = exp(-pi^2 m^2/alpha^2)/(pi V m^2)
// |b(m)|^2, C2R FFT, then each atom gathers -grad phi (and for forces the
// second derivatives) with the same weights.
#include "tdp_ewald.cuh"
#include "tdp_f32x2.cuh"
#include "tdp_frames.cuh"
#include "tdp_host.h"
#include "tdp_kernels.cuh"

#include <cufft.h>
#include <math.h>

#include <vector>

namespace tdp {

namespace {

constexpr int kEwWarps = 4;
constexpr int kEwThreads = 32 * kEwWarps;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kOrder = 5;
constexpr double kSqrtPi = 1.7724538509055160273;
constexpr double kPi = 3.1415926535897932385;
constexpr double kFixInv = 1.0 / 4294967296.0;   // 2^-32 e per unit of the fixed-point grid
// Neighbour-list entries: J tile | FOLD << 30 | SLOW << 31.
constexpr int kTileMask = (1 << 30) - 1;

struct EwParams {
    double alpha, ca, a2;   // alpha, 2 alpha/sqrt(pi), 2 alpha^2
    double rc2;             // cutoff^2
    double selfc;           // 4 alpha^3 / (3 sqrt(pi))
    int cap;                // neighbour-list row capacity
};

struct PmeGrid {
    int K[3];
    double L[3], invL[3], sc[3];   // sc = K/L
};

__device__ __forceinline__ float erfc_r(float x) { return erfcf(x); }
__device__ __forceinline__ double erfc_r(double x) { return erfc(x); }

// Real-space kernels of erfc(alpha r)/r:  B0 = erfc/r,
// B_{n+1} = ((2n+1) B_n + (2 alpha^2)^(n+1) / (alpha sqrt(pi)) e^(-alpha^2 r^2)) / r^2.
template <class R>
__device__ __forceinline__ void erfc_kernels(R r2, R rinv, R alpha, R ca, R a2, R& B0, R& B1, R& B2, R& B3) {
    R r = r2 * rinv;
    R x = alpha * r;
    R e = exp_r(-x * x);
    R rinv2 = rinv * rinv;
    B0 = erfc_r(x) * rinv;
    R t = ca * e;
    B1 = (B0 + t) * rinv2;
    t *= a2;
    B2 = (R(3) * B1 + t) * rinv2;
    t *= a2;
    B3 = (R(5) * B2 + t) * rinv2;
}

// exp(-a u^3) of the reference's Thole damping (width t_i t_j, a = min(t_i, t_j),
// undamped where t_i t_j = 0 or a u^3 >= 50), returned with a u^3; 0 if undamped.
template <class R>
__device__ __forceinline__ R thole_exp(R r, R ti, R tj, R& au3) {
    R w = ti * tj;
    au3 = R(0);
    if (w == R(0)) return R(0);
    R a = ti < tj ? ti : tj;
    R u = r / w;
    au3 = a * u * u * u;
    return au3 < R(50) ? exp_r(-au3) : R(0);
}

// Generic pair terms (see the file comment); adds the energy, the force on i
// and the field at i.
template <class R>
__device__ __forceinline__ void pair_ewald(R dx, R dy, R dz, R qi, R dix, R diy, R diz, R qj, R djx, R djy, R djz,
                                           R K0, R K1, R K2, R K3, R& e, R& fx, R& fy, R& fz, R& ex, R& ey, R& ez) {
    R dir = dix * dx + diy * dy + diz * dz;
    R djr = djx * dx + djy * dy + djz * dz;
    R didj = dix * djx + diy * djy + diz * djz;
    R G0 = qi * qj;
    R G1 = qj * dir - qi * djr + didj;
    R G2 = -dir * djr;
    e += G0 * K0 + G1 * K1 + G2 * K2;
    R c = G0 * K1 + G1 * K2 + G2 * K3;
    R a = djr * K2, b = dir * K2;
    fx -= dx * c - K1 * (qj * dix - qi * djx) + a * dix + b * djx;
    fy -= dy * c - K1 * (qj * diy - qi * djy) + a * diy + b * djy;
    fz -= dz * c - K1 * (qj * diz - qi * djz) + a * diz + b * djz;
    ex += -K1 * (qj * dx + djx) + a * dx;
    ey += -K1 * (qj * dy + djy) + a * dy;
    ez += -K1 * (qj * dz + djz) + a * dz;
}

// Field at i from (q_j, d_j) only.
template <class R>
__device__ __forceinline__ void pair_field_only(R dx, R dy, R dz, R qj, R djx, R djy, R djz, R K1, R K2, R& ex,
                                                R& ey, R& ez) {
    R a = K2 * (djx * dx + djy * dy + djz * dz);
    ex += -K1 * (qj * dx + djx) + a * dx;
    ey += -K1 * (qj * dy + djy) + a * dy;
    ez += -K1 * (qj * dz + djz) + a * dz;
}

__device__ __forceinline__ double fold1(double d, double L, double invL) {
    return L > 0.0 ? d - L * floor(d * invL + 0.5) : d;
}

// ---------------------------------------------------------------------------
// Neighbour list of tiles.
// ---------------------------------------------------------------------------
__global__ void k_ew_tiles(PairParams P, EwParams E, const double4* __restrict__ tctr, const double4* __restrict__ text,
                           const int2* __restrict__ exs_tiles, int* __restrict__ list, int* __restrict__ count,
                           int* __restrict__ overflow) {
    const int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (I >= P.n_tiles) return;
    const double4 cA = tctr[I], eA = text[I];
    const int2 et = exs_tiles[I];
    const bool ragged = (P.n & 31) != 0;
    const int last = P.n_tiles - 1;
    int written = 0;
    for (int J0 = 0; J0 < P.n_tiles; J0 += 32) {
        const int J = J0 + lane;
        bool keep = false;
        unsigned flags = 0u;
        if (J < P.n_tiles) {
            const double4 cB = tctr[J], eB = text[J];
            double dc[3] = {cB.x - cA.x, cB.y - cA.y, cB.z - cA.z};
            const double ea[3] = {eA.x, eA.y, eA.z}, eb[3] = {eB.x, eB.y, eB.z};
            double g2 = 0.0;
            bool fold = false;
            for (int k = 0; k < 3; k++) {
                dc[k] = fold1(dc[k], P.box[k], P.inv_box[k]);
                double g = fmax(fabs(dc[k]) - ea[k] - eb[k], 0.0);
                g2 += g * g;
                if (P.periodic && fabs(dc[k]) + ea[k] + eb[k] >= 0.5 * P.box[k] - 1e-9) fold = true;
            }
            keep = g2 < E.rc2;
            const bool slow = J == I || (ragged && (J == last || I == last)) || (J >= et.x && J <= et.y);
            flags = (fold ? (1u << 30) : 0u) | (slow ? (1u << 31) : 0u);
        }
        const unsigned bal = __ballot_sync(kFull, keep);
        if (keep) {
            const int pos = written + __popc(bal & ((1u << lane) - 1u));
            if (pos < E.cap) list[(size_t)I * E.cap + pos] = J | (int)flags;
        }
        written += __popc(bal);
    }
    if (lane == 0) {
        count[I] = written < E.cap ? written : E.cap;
        if (written > E.cap) atomicExch(overflow, 1);
    }
}

// Bits of the J-tile slots listed as covalent partners of slot i.
__device__ __forceinline__ unsigned partner_bits(const int* __restrict__ exs_j, int e0, int e1, int jbase) {
    unsigned b = 0u;
    for (int e = e0; e < e1; e++) {
        unsigned off = (unsigned)(exs_j[e] - jbase);
        if (off < 32u) b |= 1u << off;
    }
    return b;
}

// Minimum-image displacement of the tile pair: FP32 records are offsets from
// the tile centres, FP64 records absolute positions.
template <class R>
__device__ __forceinline__ void tile_shift(const PairParams& P, double4 cA, double4 cB, R px, R py, R pz, R& ox, R& oy,
                                           R& oz) {
    double dc[3] = {cB.x - cA.x, cB.y - cA.y, cB.z - cA.z};
    for (int k = 0; k < 3; k++) dc[k] = fold1(dc[k], P.box[k], P.inv_box[k]);
    if (sizeof(R) == 4) {
        ox = px - (R)dc[0];
        oy = py - (R)dc[1];
        oz = pz - (R)dc[2];
    } else {
        ox = px + (R)((cB.x - cA.x) - dc[0]);
        oy = py + (R)((cB.y - cA.y) - dc[1]);
        oz = pz + (R)((cB.z - cA.z) - dc[2]);
    }
}

template <class R>
__device__ __forceinline__ R fold_r(R d, double L, double invL) {
    if (sizeof(R) == 4) return (R)fold_f((float)d, (float)L, (float)invL);
    return (R)fold_d((double)d, L, invL);
}

// ---------------------------------------------------------------------------
// Real-space fields: KIND 0 = permanent field from (q, p) with M scales,
// KIND 1 = field of the operand v (vec_s) with I scales.
// ---------------------------------------------------------------------------
template <class R, int KIND, bool FOLD, bool SLOW>
__device__ __forceinline__ void ew_field_walk(const PairParams& P, const EwParams& E,
                                              const typename Vec4T<R>::type* __restrict__ sp,
                                              const typename Vec4T<R>::type* __restrict__ sv, int i, int jbase,
                                              R ox, R oy, R oz, R ti, unsigned partners, R rc2, R damp_r2, R& fx,
                                              R& fy, R& fz) {
    const R alpha = (R)E.alpha, ca = (R)E.ca, a2 = (R)E.a2;
#pragma unroll 2
    for (int s = 0; s < 32; s++) {
        const typename Vec4T<R>::type pj = sp[s], vj = sv[s];
        R dx = pj.x - ox, dy = pj.y - oy, dz = pj.z - oz;
        if (FOLD) {
            dx = fold_r(dx, P.box[0], P.inv_box[0]);
            dy = fold_r(dy, P.box[1], P.inv_box[1]);
            dz = fold_r(dz, P.box[2], P.inv_box[2]);
        }
        R r2 = dx * dx + dy * dy + dz * dz;
        bool act = r2 < rc2;
        if (SLOW) {
            const int j = jbase + s;
            act = act && j != i && i < P.n && j < P.n && !((partners >> s) & 1u);
        }
        if (!__any_sync(kFull, act)) continue;
        if (!act) r2 = R(1e30);
        R rinv = rsqrt_r(r2);
        R B0, B1, B2, B3;
        erfc_kernels<R>(r2, rinv, alpha, ca, a2, B0, B1, B2, B3);
        if (r2 < damp_r2) {
            R au3;
            R et = thole_exp<R>(r2 * rinv, ti, vj.w, au3);
            R b1 = rinv * rinv * rinv;
            B1 -= et * b1;
            B2 -= (R(1) + au3) * et * R(3) * b1 * rinv * rinv;
        }
        pair_field_only<R>(dx, dy, dz, KIND == 0 ? pj.w : R(0), vj.x, vj.y, vj.z, B1, B2, fx, fy, fz);
    }
}

// Exceptions of slot i (covalent partners with their M and I scales), FP64:
// erfc part within the cutoff, minus the bare term, plus the scaled, damped term.
// lab (KIND 0 only: the fused start of a warm-started solve, whose dipole
// records hold P = m + mu0): the partner's mu0 = P - m gets its I scale, i.e.
// (I - M) times the damped term of mu0 is added to the M-scaled field of P.
template <class R, int KIND>
__device__ __forceinline__ void ew_field_exceptions(const PairParams& P, const EwParams& E,
                                                    const double* __restrict__ pos_s,
                                                    const typename Vec4T<R>::type* __restrict__ posq_s,
                                                    const typename Vec4T<R>::type* __restrict__ src,
                                                    const int* __restrict__ exs_off, const int* __restrict__ exs_j,
                                                    const double* __restrict__ exs_m, const double* __restrict__ exs_s,
                                                    int i, double ti, double& fx, double& fy, double& fz,
                                                    const typename Vec4T<R>::type* __restrict__ lab = nullptr) {
    const int e0 = exs_off[i], e1 = exs_off[i + 1];
    const d3 pi = ld3(pos_s + 3 * i);
    for (int e = e0; e < e1; e++) {
        const int j = exs_j[e];
        const double sc = KIND == 0 ? exs_m[e] : exs_s[e];
        d3 pj = ld3(pos_s + 3 * j);
        double dx = fold1(pj.x - pi.x, P.box[0], P.inv_box[0]);
        double dy = fold1(pj.y - pi.y, P.box[1], P.inv_box[1]);
        double dz = fold1(pj.z - pi.z, P.box[2], P.inv_box[2]);
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt(r2);
        double b1 = rinv * rinv * rinv, b2 = 3.0 * b1 * rinv * rinv;
        double B0 = 0, B1 = 0, B2 = 0, B3 = 0;
        if (r2 < E.rc2) erfc_kernels<double>(r2, rinv, E.alpha, E.ca, E.a2, B0, B1, B2, B3);
        const typename Vec4T<R>::type vj = src[j];
        double au3;
        double et = thole_exp<double>(r2 * rinv, ti, (double)vj.w, au3);
        double l3 = 1.0 - et, l5 = 1.0 - (1.0 + au3) * et;
        double K1 = B1 - b1 + sc * l3 * b1, K2 = B2 - b2 + sc * l5 * b2;
        double qj = KIND == 0 ? (double)posq_s[j].w : 0.0;
        pair_field_only<double>(dx, dy, dz, qj, (double)vj.x, (double)vj.y, (double)vj.z, K1, K2, fx, fy, fz);
        if (KIND == 0 && lab) {
            const double ds = exs_s[e] - sc;
            if (ds != 0.0) {
                const typename Vec4T<R>::type mj = lab[j];
                pair_field_only<double>(dx, dy, dz, 0.0, (double)vj.x - (double)mj.x, (double)vj.y - (double)mj.y,
                                        (double)vj.z - (double)mj.z, ds * l3 * b1, ds * l5 * b2, fx, fy, fz);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Packed FP32 walk of the mixed form (sm_100 f32x2 arithmetic): each step
// evaluates the lane's I atom against two J atoms, whose records are staged
// pair-interleaved (x_2m, x_2m+1, y_2m, y_2m+1) so 128-bit shared loads give
// packed operands directly.  erfc(x) = t P(t) exp(-x^2) with t = 1/(1 + p x):
// the Hastings form (Abramowitz & Stegun 7.1.26) with coefficients fitted
// here to erfc on [0, 4.5] in relative error (1.1e-8 in exact arithmetic,
// 1.2e-6 at x = 4.3 evaluated in FP32), sharing exp(-x^2) with the B kernels.
// Thole damping uses 1/t precomputed per atom.
// ---------------------------------------------------------------------------
constexpr float kErfcP = 0.41f;
__constant__ float c_erfc[8] = {0.2307648634694866f,  0.23957919808529987f, 0.15874078916517892f,
                                0.3642441184340127f,  -0.29754436616944707f, 0.6117635229498828f,
                                -0.3865500288941725f, 0.0790019121010213f};

struct EwPackedTile {
    float4 p0[16], p1[16], v0[16], v1[16];   // (x,x' y,y') (z,z' q,q') (vx,vx' vy,vy') (vz,vz' t,t')
    float2 it[16];                           // 1/t of the pair
};

__device__ __forceinline__ void stage_packed(EwPackedTile& T, int lane, float4 p, float4 v) {
    const int m = lane >> 1, h = lane & 1;
    float* p0 = reinterpret_cast<float*>(&T.p0[m]);
    float* p1 = reinterpret_cast<float*>(&T.p1[m]);
    float* v0 = reinterpret_cast<float*>(&T.v0[m]);
    float* v1 = reinterpret_cast<float*>(&T.v1[m]);
    p0[h] = p.x;
    p0[2 + h] = p.y;
    p1[h] = p.z;
    p1[2 + h] = p.w;
    v0[h] = v.x;
    v0[2 + h] = v.y;
    v1[h] = v.z;
    v1[2 + h] = v.w;
    reinterpret_cast<float*>(&T.it[m])[h] = 1.0f / v.w;
}

// Whether a J atom (record offsets p in J's frame) can lie within the cutoff
// of any atom of the I tile, whose centre sits at -dc in J's frame with
// half-extents e: the distance to the I tile's box, minimum image when the
// tile pair folds, against the cutoff plus 1e-3 nm (no pair the walk would
// count is dropped by FP32 rounding).
__device__ __forceinline__ bool near_i_tile(const PairParams& P, float px, float py, float pz, const float* dc,
                                            const float* e, float rcm2, bool fold) {
    float a[3] = {px + dc[0], py + dc[1], pz + dc[2]};
    float g2 = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        if (fold) a[k] = fold_f(a[k], (float)P.box[k], (float)P.inv_box[k]);
        const float g = fmaxf(fabsf(a[k]) - e[k], 0.0f);
        g2 += g * g;
    }
    return g2 < rcm2;
}

// Minimum-image displacement of J's tile centre from I's, FP32 (mixed form).
__device__ __forceinline__ void tile_dc(const PairParams& P, double4 cA, double4 cB, float* dc) {
    dc[0] = (float)fold1(cB.x - cA.x, P.box[0], P.inv_box[0]);
    dc[1] = (float)fold1(cB.y - cA.y, P.box[1], P.inv_box[1]);
    dc[2] = (float)fold1(cB.z - cA.z, P.box[2], P.inv_box[2]);
}

template <int KIND, bool FOLD>
__device__ __forceinline__ void ew_field_walk_x2(const PairParams& P, const EwParams& E, const EwPackedTile& T,
                                                 float ox, float oy, float oz, float ti, float iti, float rc2,
                                                 float damp_r2, int nsteps, float& fx, float& fy, float& fz) {
    const f2 OX = bc2(ox), OY = bc2(oy), OZ = bc2(oz);
    const f2 ALPHA = bc2((float)E.alpha), NA2 = bc2((float)(-E.alpha * E.alpha));
    const f2 CA = bc2((float)E.ca), A2 = bc2((float)E.a2), ONE = bc2(1.0f), THREE = bc2(3.0f), NEG = bc2(-1.0f);
    const f2 PP = bc2(kErfcP), ITI = bc2(iti);
    f2 Lx = 0, Ly = 0, Lz = 0, Ix = 0, Iy = 0, Iz = 0;
    if (FOLD) {
        Lx = bc2(-(float)P.box[0]);
        Ly = bc2(-(float)P.box[1]);
        Lz = bc2(-(float)P.box[2]);
        Ix = bc2((float)P.inv_box[0]);
        Iy = bc2((float)P.inv_box[1]);
        Iz = bc2((float)P.inv_box[2]);
    }
    const f2 MAGIC = bc2(12582912.0f), NMAGIC = bc2(-12582912.0f);
    f2 FX = 0, FY = 0, FZ = 0;
#pragma unroll 2
    for (int m = 0; m < nsteps; m++) {
        const float4 a = T.p0[m], b = T.p1[m], c = T.v0[m], d = T.v1[m];
        const float2 it = T.it[m];
        f2 DX = sub2(pk2(a.x, a.y), OX), DY = sub2(pk2(a.z, a.w), OY), DZ = sub2(pk2(b.x, b.y), OZ);
        if (FOLD) {
            DX = fma2(add2(fma2(DX, Ix, MAGIC), NMAGIC), Lx, DX);
            DY = fma2(add2(fma2(DY, Iy, MAGIC), NMAGIC), Ly, DY);
            DZ = fma2(add2(fma2(DZ, Iz, MAGIC), NMAGIC), Lz, DZ);
        }
        const f2 R2 = fma2(DX, DX, fma2(DY, DY, mul2(DZ, DZ)));
        float r2a, r2b;
        un2(R2, r2a, r2b);
        const bool act_a = r2a < rc2, act_b = r2b < rc2;
        if (!__any_sync(kFull, act_a || act_b)) continue;
        r2a = act_a ? r2a : 1e30f;
        r2b = act_b ? r2b : 1e30f;
        const f2 R2S = pk2(r2a, r2b);
        const f2 RINV = pk2(rsqrtf(r2a), rsqrtf(r2b));
        const f2 RINV2 = mul2(RINV, RINV);
        const f2 R = mul2(R2S, RINV);
        const f2 X = mul2(ALPHA, R);
        float ea, eb;
        un2(mul2(NA2, R2S), ea, eb);
        const f2 EX = pk2(__expf(ea), __expf(eb));
        float da, db;
        un2(fma2(PP, X, ONE), da, db);
        const f2 TT = pk2(__fdividef(1.0f, da), __fdividef(1.0f, db));
        f2 POLY = bc2(c_erfc[7]);
#pragma unroll
        for (int k = 6; k >= 0; k--) POLY = fma2(POLY, TT, bc2(c_erfc[k]));
        const f2 B0 = mul2(mul2(mul2(POLY, TT), EX), RINV);
        const f2 G1 = mul2(CA, EX);
        f2 B1 = mul2(add2(B0, G1), RINV2);
        f2 B2 = mul2(fma2(THREE, B1, mul2(G1, A2)), RINV2);
        if (r2a < damp_r2 || r2b < damp_r2) {
            // -(1 - l3) b1 and -(1 - l5) b2 with u = r / (t_i t_j), a = min(t_i, t_j).
            const f2 U = mul2(mul2(R, ITI), pk2(it.x, it.y));
            const f2 AM = pk2(fminf(ti, d.z), fminf(ti, d.w));
            const f2 AU3 = mul2(AM, mul2(U, mul2(U, U)));
            float xa, xb;
            un2(AU3, xa, xb);
            // Per half: e^{-a u^3} and (1 + a u^3) e^{-a u^3}, zero outside the
            // damping range (a masked half has u^3 = inf, never multiplied).
            float eta = 0.0f, etb = 0.0f, wa = 0.0f, wb = 0.0f;
            if (xa < 50.0f && r2a < damp_r2) {
                eta = __expf(-xa);
                wa = (1.0f + xa) * eta;
            }
            if (xb < 50.0f && r2b < damp_r2) {
                etb = __expf(-xb);
                wb = (1.0f + xb) * etb;
            }
            const f2 BB1 = mul2(RINV, RINV2);
            B1 = sub2(B1, mul2(pk2(eta, etb), BB1));
            B2 = sub2(B2, mul2(pk2(wa, wb), mul2(mul2(THREE, BB1), RINV2)));
        }
        const f2 VX = pk2(c.x, c.y), VY = pk2(c.z, c.w), VZ = pk2(d.x, d.y);
        const f2 A = mul2(B2, fma2(VX, DX, fma2(VY, DY, mul2(VZ, DZ))));
        const f2 NB1 = mul2(B1, NEG);
        if (KIND == 0) {
            const f2 Q = pk2(b.z, b.w);
            FX = fma2(A, DX, fma2(NB1, fma2(Q, DX, VX), FX));
            FY = fma2(A, DY, fma2(NB1, fma2(Q, DY, VY), FY));
            FZ = fma2(A, DZ, fma2(NB1, fma2(Q, DZ, VZ), FZ));
        } else {
            FX = fma2(A, DX, fma2(NB1, VX, FX));
            FY = fma2(A, DY, fma2(NB1, VY, FY));
            FZ = fma2(A, DZ, fma2(NB1, VZ, FZ));
        }
    }
    float lo, hi;
    un2(FX, lo, hi);
    fx += lo + hi;
    un2(FY, lo, hi);
    fy += lo + hi;
    un2(FZ, lo, hi);
    fz += lo + hi;
}

template <class R, int KIND>
__global__ void __launch_bounds__(kEwThreads) k_ew_field(PairParams P, EwParams E,
                                                         const typename Vec4T<R>::type* __restrict__ posq_s,
                                                         const typename Vec4T<R>::type* __restrict__ src,
                                                         const double4* __restrict__ tctr,
                                                         const double4* __restrict__ text,
                                                         const double* __restrict__ pos_s,
                                                         const int* __restrict__ exs_off, const int* __restrict__ exs_j,
                                                         const double* __restrict__ exs_m,
                                                         const double* __restrict__ exs_s, const int* __restrict__ list,
                                                         const int* __restrict__ count, int n_pad,
                                                         double* __restrict__ out,
                                                         const typename Vec4T<R>::type* __restrict__ lab) {
    typedef typename Vec4T<R>::type V4;
    __shared__ V4 s_pos[kEwWarps][32], s_vec[kEwWarps][32];
    __shared__ EwPackedTile s_pk[sizeof(R) == 4 ? kEwWarps : 1];
    __shared__ double s_red[kEwWarps][3][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // One I tile per CTA; warp w takes list entries w, w + 4, ...; the four
    // partial sums are added in warp order.
    const int I = blockIdx.x;
    const int i = I * 32 + lane;
    const V4 pi = posq_s[i], vi = src[i];
    const double4 cA = tctr[I];
    const double4 eAd = text[I];
    const float eA[3] = {(float)eAd.x, (float)eAd.y, (float)eAd.z};
    const float rcm = (float)sqrt(E.rc2) + 1e-3f;
    const int e0 = i < P.n ? exs_off[i] : 0, e1 = i < P.n ? exs_off[i + 1] : 0;
    const R rc2 = (R)E.rc2, damp_r2 = (R)P.damp_r2;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    const int cnt = count[I];
    for (int t = warp; t < cnt; t += kEwWarps) {
        const int ent = list[(size_t)I * E.cap + t];
        const int J = ent & kTileMask;
        const bool fold = (ent >> 30) & 1, slow = ((unsigned)ent >> 31) & 1u;
        const double4 cB = tctr[J];
        __syncwarp();
        const V4 pj = posq_s[J * 32 + lane], vj = src[J * 32 + lane];
        int nsteps = 16;
        bool staged = false;
        if constexpr (sizeof(R) == 4) {
            if (!slow) {
                // Only the J atoms within the cutoff of the I tile's box,
                // compacted; an odd count is padded with a multipole-free copy.
                float dc[3];
                tile_dc(P, cA, cB, dc);
                const bool act = near_i_tile(P, (float)pj.x, (float)pj.y, (float)pj.z, dc, eA, rcm * rcm, fold);
                const unsigned mk = __ballot_sync(kFull, act);
                const int nact = __popc(mk), k = __popc(mk & ((1u << lane) - 1u));
                if (act) stage_packed(s_pk[warp], k, pj, vj);
                if ((nact & 1) && act && k == nact - 1)
                    stage_packed(s_pk[warp], nact, make_float4(pj.x, pj.y, pj.z, 0.0f), make_float4(0.0f, 0.0f, 0.0f, vj.w));
                nsteps = (nact + 1) >> 1;
                staged = true;
            }
        }
        if (!staged) {
            s_pos[warp][lane] = pj;
            s_vec[warp][lane] = vj;
        }
        __syncwarp();
        R ox, oy, oz;
        tile_shift<R>(P, cA, cB, pi.x, pi.y, pi.z, ox, oy, oz);
        R tx = 0, ty = 0, tz = 0;
        if constexpr (sizeof(R) == 4) {
            if (!slow) {
                const float iti = 1.0f / (float)vi.w;
                if (fold) ew_field_walk_x2<KIND, true>(P, E, s_pk[warp], ox, oy, oz, vi.w, iti, rc2, damp_r2, nsteps, tx, ty, tz);
                else ew_field_walk_x2<KIND, false>(P, E, s_pk[warp], ox, oy, oz, vi.w, iti, rc2, damp_r2, nsteps, tx, ty, tz);
                fx += (double)tx;
                fy += (double)ty;
                fz += (double)tz;
                continue;
            }
        }
        if (slow) {
            const unsigned part = partner_bits(exs_j, e0, e1, J * 32);
            if (fold) ew_field_walk<R, KIND, true, true>(P, E, s_pos[warp], s_vec[warp], i, J * 32, ox, oy, oz, vi.w, part, rc2, damp_r2, tx, ty, tz);
            else ew_field_walk<R, KIND, false, true>(P, E, s_pos[warp], s_vec[warp], i, J * 32, ox, oy, oz, vi.w, part, rc2, damp_r2, tx, ty, tz);
        } else if (fold) {
            ew_field_walk<R, KIND, true, false>(P, E, s_pos[warp], s_vec[warp], i, J * 32, ox, oy, oz, vi.w, 0u, rc2, damp_r2, tx, ty, tz);
        } else {
            ew_field_walk<R, KIND, false, false>(P, E, s_pos[warp], s_vec[warp], i, J * 32, ox, oy, oz, vi.w, 0u, rc2, damp_r2, tx, ty, tz);
        }
        fx += (double)tx;
        fy += (double)ty;
        fz += (double)tz;
    }
    s_red[warp][0][lane] = fx;
    s_red[warp][1][lane] = fy;
    s_red[warp][2][lane] = fz;
    __syncthreads();
    if (warp != 0) return;
    for (int w = 1; w < kEwWarps; w++) {
        fx += s_red[w][0][lane];
        fy += s_red[w][1][lane];
        fz += s_red[w][2][lane];
    }
    if (i < P.n)
        ew_field_exceptions<R, KIND>(P, E, pos_s, posq_s, src, exs_off, exs_j, exs_m, exs_s, i, (double)vi.w, fx, fy,
                                     fz, lab);
    else fx = fy = fz = 0.0;
    out[i] = fx;
    out[(size_t)n_pad + i] = fy;
    out[2 * (size_t)n_pad + i] = fz;
}

// ---------------------------------------------------------------------------
// Real-space energy, forces and the field acting on the permanent dipoles.
// Records: posq_s (offsets/positions, q), dipt_s (p, thole), vec_s (mu, thole).
// ---------------------------------------------------------------------------
template <class R, bool FOLD, bool SLOW>
__device__ __forceinline__ void ew_force_walk(const PairParams& P, const EwParams& E,
                                              const typename Vec4T<R>::type* __restrict__ sp,
                                              const typename Vec4T<R>::type* __restrict__ sd,
                                              const typename Vec4T<R>::type* __restrict__ su, int i, int jbase,
                                              R ox, R oy, R oz, R qi, typename Vec4T<R>::type di,
                                              typename Vec4T<R>::type ui, unsigned partners, R rc2, R damp_r2, R& en,
                                              R* f, R* g) {
    const R alpha = (R)E.alpha, ca = (R)E.ca, a2 = (R)E.a2;
    const R tix = di.x + ui.x, tiy = di.y + ui.y, tiz = di.z + ui.z;
#pragma unroll 1
    for (int s = 0; s < 32; s++) {
        const typename Vec4T<R>::type pj = sp[s], dj = sd[s], uj = su[s];
        R dx = pj.x - ox, dy = pj.y - oy, dz = pj.z - oz;
        if (FOLD) {
            dx = fold_r(dx, P.box[0], P.inv_box[0]);
            dy = fold_r(dy, P.box[1], P.inv_box[1]);
            dz = fold_r(dz, P.box[2], P.inv_box[2]);
        }
        R r2 = dx * dx + dy * dy + dz * dz;
        bool act = r2 < rc2;
        if (SLOW) {
            const int j = jbase + s;
            act = act && j != i && i < P.n && j < P.n && !((partners >> s) & 1u);
        }
        if (!__any_sync(kFull, act)) continue;
        if (!act) r2 = R(1e30);
        R rinv = rsqrt_r(r2);
        R B0, B1, B2, B3;
        erfc_kernels<R>(r2, rinv, alpha, ca, a2, B0, B1, B2, B3);
        R d1 = 0, d2 = 0, d3v = 0;
        if (r2 < damp_r2) {
            R au3;
            R et = thole_exp<R>(r2 * rinv, di.w, dj.w, au3);
            R b1 = rinv * rinv * rinv;
            R rinv2 = rinv * rinv;
            d1 = et * b1;
            d2 = (R(1) + au3) * et * R(3) * b1 * rinv2;
            d3v = (R(1) + au3 + R(0.6) * au3 * au3) * et * R(15) * b1 * rinv2 * rinv2;
        }
        R e = 0;
        // E(T,T; Be - Kd) + E(P,P; Kd)
        pair_ewald<R>(dx, dy, dz, qi, tix, tiy, tiz, pj.w, dj.x + uj.x, dj.y + uj.y, dj.z + uj.z, B0, B1 - d1, B2 - d2,
                      B3 - d3v, e, f[0], f[1], f[2], g[0], g[1], g[2]);
        if (d1 != R(0))
            pair_ewald<R>(dx, dy, dz, qi, di.x, di.y, di.z, pj.w, dj.x, dj.y, dj.z, R(0), d1, d2, d3v, e, f[0], f[1],
                          f[2], g[0], g[1], g[2]);
        en += R(0.5) * e;
    }
}

template <class R>
__device__ __forceinline__ void ew_force_exceptions(const PairParams& P, const EwParams& E,
                                                    const double* __restrict__ pos_s,
                                                    const typename Vec4T<R>::type* __restrict__ posq_s,
                                                    const typename Vec4T<R>::type* __restrict__ dipt_s,
                                                    const typename Vec4T<R>::type* __restrict__ vec_s,
                                                    const int* __restrict__ exs_off, const int* __restrict__ exs_j,
                                                    const double* __restrict__ exs_m, const double* __restrict__ exs_s,
                                                    int i, double& en, double* f, double* g) {
    const d3 pi = ld3(pos_s + 3 * i);
    const typename Vec4T<R>::type Di = dipt_s[i], Ui = vec_s[i];
    const double qi = (double)posq_s[i].w;
    const double pix = Di.x, piy = Di.y, piz = Di.z, uix = Ui.x, uiy = Ui.y, uiz = Ui.z, ti = Di.w;
    for (int e = exs_off[i]; e < exs_off[i + 1]; e++) {
        const int j = exs_j[e];
        const double m = exs_m[e], sc = exs_s[e];
        const d3 pj = ld3(pos_s + 3 * j);
        double dx = fold1(pj.x - pi.x, P.box[0], P.inv_box[0]);
        double dy = fold1(pj.y - pi.y, P.box[1], P.inv_box[1]);
        double dz = fold1(pj.z - pi.z, P.box[2], P.inv_box[2]);
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt(r2);
        double rinv2 = rinv * rinv;
        double b0 = rinv, b1 = rinv * rinv2, b2 = 3.0 * b1 * rinv2, b3 = 5.0 * b2 * rinv2;
        double B0 = 0, B1 = 0, B2 = 0, B3 = 0;
        if (r2 < E.rc2) erfc_kernels<double>(r2, rinv, E.alpha, E.ca, E.a2, B0, B1, B2, B3);
        const typename Vec4T<R>::type Dj = dipt_s[j], Uj = vec_s[j];
        const double qj = (double)posq_s[j].w;
        double au3;
        double et = thole_exp<double>(r2 * rinv, ti, (double)Dj.w, au3);
        double k1 = (1.0 - et) * b1, k2 = (1.0 - (1.0 + au3) * et) * b2,
               k3 = (1.0 - (1.0 + au3 + 0.6 * au3 * au3) * et) * b3;
        double pjx = Dj.x, pjy = Dj.y, pjz = Dj.z, ujx = Uj.x, ujy = Uj.y, ujz = Uj.z;
        double ee = 0.0;
        // E(T,T; Be - b + m Kl) + E(P,P; m b - m Kl) + E(U,U; (s - m) Kl)
        pair_ewald<double>(dx, dy, dz, qi, pix + uix, piy + uiy, piz + uiz, qj, pjx + ujx, pjy + ujy, pjz + ujz,
                           B0 - b0, B1 - b1 + m * k1, B2 - b2 + m * k2, B3 - b3 + m * k3, ee, f[0], f[1], f[2], g[0],
                           g[1], g[2]);
        pair_ewald<double>(dx, dy, dz, qi, pix, piy, piz, qj, pjx, pjy, pjz, m * b0, m * (b1 - k1), m * (b2 - k2),
                           m * (b3 - k3), ee, f[0], f[1], f[2], g[0], g[1], g[2]);
        double h[3] = {0, 0, 0};
        pair_ewald<double>(dx, dy, dz, 0.0, uix, uiy, uiz, 0.0, ujx, ujy, ujz, 0.0, (sc - m) * k1, (sc - m) * k2,
                           (sc - m) * k3, ee, f[0], f[1], f[2], h[0], h[1], h[2]);
        en += 0.5 * ee;
    }
}

// Packed J-pair records of the force walk: (x,x' y,y') (z,z' q,q')
// (px,px' py,py') (pz,pz' t,t') (ux,ux' uy,uy') (uz,uz' -,-) and 1/t.
struct EwPackedForceTile {
    float4 p0[16], p1[16], d0[16], d1[16], u0[16], u1[16];
    float2 it[16];
};

__device__ __forceinline__ void stage_packed_force(EwPackedForceTile& T, int lane, float4 p, float4 dv, float4 u) {
    const int m = lane >> 1, h = lane & 1;
    float* p0 = reinterpret_cast<float*>(&T.p0[m]);
    float* p1 = reinterpret_cast<float*>(&T.p1[m]);
    float* d0 = reinterpret_cast<float*>(&T.d0[m]);
    float* d1 = reinterpret_cast<float*>(&T.d1[m]);
    float* u0 = reinterpret_cast<float*>(&T.u0[m]);
    float* u1 = reinterpret_cast<float*>(&T.u1[m]);
    p0[h] = p.x;
    p0[2 + h] = p.y;
    p1[h] = p.z;
    p1[2 + h] = p.w;
    d0[h] = dv.x;
    d0[2 + h] = dv.y;
    d1[h] = dv.z;
    d1[2 + h] = dv.w;
    u0[h] = u.x;
    u0[2 + h] = u.y;
    u1[h] = u.z;
    u1[2 + h] = 0.0f;
    reinterpret_cast<float*>(&T.it[m])[h] = 1.0f / dv.w;
}

// pair_ewald on both halves: energy, force on i and field at i for kernels K.
__device__ __forceinline__ void pair_ewald2(f2 DX, f2 DY, f2 DZ, f2 QI, f2 IX, f2 IY, f2 IZ, f2 QJ, f2 JX, f2 JY,
                                            f2 JZ, f2 K0, f2 K1, f2 K2, f2 K3, f2& EN, f2& FX, f2& FY, f2& FZ,
                                            f2& GX, f2& GY, f2& GZ) {
    const f2 NEG = bc2(-1.0f);
    const f2 DIR = fma2(IX, DX, fma2(IY, DY, mul2(IZ, DZ)));
    const f2 DJR = fma2(JX, DX, fma2(JY, DY, mul2(JZ, DZ)));
    const f2 DIDJ = fma2(IX, JX, fma2(IY, JY, mul2(IZ, JZ)));
    const f2 G0 = mul2(QI, QJ);
    const f2 G1 = add2(fma2(QJ, DIR, mul2(mul2(QI, DJR), NEG)), DIDJ);
    const f2 G2 = mul2(mul2(DIR, DJR), NEG);
    EN = fma2(G0, K0, fma2(G1, K1, fma2(G2, K2, EN)));
    const f2 NC = mul2(fma2(G0, K1, fma2(G1, K2, mul2(G2, K3))), NEG);
    const f2 NA = mul2(mul2(DJR, K2), NEG), NB = mul2(mul2(DIR, K2), NEG);
    const f2 NQI = mul2(QI, NEG);
    // f -= d c - K1 (q_j d_i - q_i d_j) + a d_i + b d_j
    FX = fma2(DX, NC, fma2(K1, fma2(QJ, IX, mul2(NQI, JX)), fma2(NA, IX, fma2(NB, JX, FX))));
    FY = fma2(DY, NC, fma2(K1, fma2(QJ, IY, mul2(NQI, JY)), fma2(NA, IY, fma2(NB, JY, FY))));
    FZ = fma2(DZ, NC, fma2(K1, fma2(QJ, IZ, mul2(NQI, JZ)), fma2(NA, IZ, fma2(NB, JZ, FZ))));
    // field += -K1 (q_j d + d_j) + a d
    const f2 NK1 = mul2(K1, NEG), A = mul2(DJR, K2);
    GX = fma2(A, DX, fma2(NK1, fma2(QJ, DX, JX), GX));
    GY = fma2(A, DY, fma2(NK1, fma2(QJ, DY, JY), GY));
    GZ = fma2(A, DZ, fma2(NK1, fma2(QJ, DZ, JZ), GZ));
}

template <bool FOLD>
__device__ __forceinline__ void ew_force_walk_x2(const PairParams& P, const EwParams& E, const EwPackedForceTile& T,
                                                 float ox, float oy, float oz, float qi, float4 di, float4 ui,
                                                 float iti, float rc2, float damp_r2, int nsteps, float& en, float* f,
                                                 float* g) {
    const f2 OX = bc2(ox), OY = bc2(oy), OZ = bc2(oz);
    const f2 ALPHA = bc2((float)E.alpha), NA2 = bc2((float)(-E.alpha * E.alpha));
    const f2 CA = bc2((float)E.ca), A2 = bc2((float)E.a2), ONE = bc2(1.0f), THREE = bc2(3.0f),
             FIVE = bc2(5.0f), HALF = bc2(0.5f), ZERO = bc2(0.0f);
    const f2 PP = bc2(kErfcP), ITI = bc2(iti), QI = bc2(qi);
    const f2 PIX = bc2(di.x), PIY = bc2(di.y), PIZ = bc2(di.z);
    const f2 TIX = bc2(di.x + ui.x), TIY = bc2(di.y + ui.y), TIZ = bc2(di.z + ui.z);
    f2 Lx = 0, Ly = 0, Lz = 0, Ix = 0, Iy = 0, Iz = 0;
    if (FOLD) {
        Lx = bc2(-(float)P.box[0]);
        Ly = bc2(-(float)P.box[1]);
        Lz = bc2(-(float)P.box[2]);
        Ix = bc2((float)P.inv_box[0]);
        Iy = bc2((float)P.inv_box[1]);
        Iz = bc2((float)P.inv_box[2]);
    }
    const f2 MAGIC = bc2(12582912.0f), NMAGIC = bc2(-12582912.0f);
    f2 EN = 0, FX = 0, FY = 0, FZ = 0, GX = 0, GY = 0, GZ = 0;
#pragma unroll 1
    for (int m = 0; m < nsteps; m++) {
        const float4 a = T.p0[m], b = T.p1[m], c = T.d0[m], d = T.d1[m], u = T.u0[m], v = T.u1[m];
        const float2 it = T.it[m];
        f2 DX = sub2(pk2(a.x, a.y), OX), DY = sub2(pk2(a.z, a.w), OY), DZ = sub2(pk2(b.x, b.y), OZ);
        if (FOLD) {
            DX = fma2(add2(fma2(DX, Ix, MAGIC), NMAGIC), Lx, DX);
            DY = fma2(add2(fma2(DY, Iy, MAGIC), NMAGIC), Ly, DY);
            DZ = fma2(add2(fma2(DZ, Iz, MAGIC), NMAGIC), Lz, DZ);
        }
        const f2 R2 = fma2(DX, DX, fma2(DY, DY, mul2(DZ, DZ)));
        float r2a, r2b;
        un2(R2, r2a, r2b);
        const bool act_a = r2a < rc2, act_b = r2b < rc2;
        if (!__any_sync(kFull, act_a || act_b)) continue;
        r2a = act_a ? r2a : 1e30f;
        r2b = act_b ? r2b : 1e30f;
        const f2 R2S = pk2(r2a, r2b);
        const f2 RINV = pk2(rsqrtf(r2a), rsqrtf(r2b));
        const f2 RINV2 = mul2(RINV, RINV);
        const f2 R = mul2(R2S, RINV);
        const f2 X = mul2(ALPHA, R);
        float ea, eb;
        un2(mul2(NA2, R2S), ea, eb);
        const f2 EX = pk2(__expf(ea), __expf(eb));
        float da, db;
        un2(fma2(PP, X, ONE), da, db);
        const f2 TT = pk2(__fdividef(1.0f, da), __fdividef(1.0f, db));
        f2 POLY = bc2(c_erfc[7]);
#pragma unroll
        for (int k = 6; k >= 0; k--) POLY = fma2(POLY, TT, bc2(c_erfc[k]));
        const f2 B0 = mul2(mul2(mul2(POLY, TT), EX), RINV);
        f2 G1 = mul2(CA, EX);
        const f2 B1 = mul2(add2(B0, G1), RINV2);
        G1 = mul2(G1, A2);
        const f2 B2 = mul2(fma2(THREE, B1, G1), RINV2);
        G1 = mul2(G1, A2);
        const f2 B3 = mul2(fma2(FIVE, B2, G1), RINV2);
        f2 D1 = ZERO, D2 = ZERO, D3 = ZERO;
        const bool damp = r2a < damp_r2 || r2b < damp_r2;
        if (damp) {
            const f2 U = mul2(mul2(R, ITI), pk2(it.x, it.y));
            const f2 AM = pk2(fminf(di.w, d.z), fminf(di.w, d.w));
            const f2 AU3 = mul2(AM, mul2(U, mul2(U, U)));
            float xa, xb;
            un2(AU3, xa, xb);
            float e1a = 0.f, e1b = 0.f, e2a = 0.f, e2b = 0.f, e3a = 0.f, e3b = 0.f;
            if (xa < 50.0f && r2a < damp_r2) {
                e1a = __expf(-xa);
                e2a = (1.0f + xa) * e1a;
                e3a = (1.0f + xa + 0.6f * xa * xa) * e1a;
            }
            if (xb < 50.0f && r2b < damp_r2) {
                e1b = __expf(-xb);
                e2b = (1.0f + xb) * e1b;
                e3b = (1.0f + xb + 0.6f * xb * xb) * e1b;
            }
            const f2 BB1 = mul2(RINV, RINV2);
            const f2 BB2 = mul2(mul2(THREE, BB1), RINV2);
            const f2 BB3 = mul2(mul2(FIVE, BB2), RINV2);
            D1 = mul2(pk2(e1a, e1b), BB1);
            D2 = mul2(pk2(e2a, e2b), BB2);
            D3 = mul2(pk2(e3a, e3b), BB3);
        }
        const f2 QJ = pk2(b.z, b.w);
        const f2 PJX = pk2(c.x, c.y), PJY = pk2(c.z, c.w), PJZ = pk2(d.x, d.y);
        const f2 TJX = add2(PJX, pk2(u.x, u.y)), TJY = add2(PJY, pk2(u.z, u.w)), TJZ = add2(PJZ, pk2(v.x, v.y));
        // E(T,T; Be - Kd) + E(P,P; Kd)
        f2 E2 = ZERO;
        pair_ewald2(DX, DY, DZ, QI, TIX, TIY, TIZ, QJ, TJX, TJY, TJZ, B0, sub2(B1, D1), sub2(B2, D2), sub2(B3, D3), E2,
                    FX, FY, FZ, GX, GY, GZ);
        if (damp)
            pair_ewald2(DX, DY, DZ, QI, PIX, PIY, PIZ, QJ, PJX, PJY, PJZ, ZERO, D1, D2, D3, E2, FX, FY, FZ, GX, GY, GZ);
        EN = fma2(HALF, E2, EN);
    }
    float lo, hi;
    un2(EN, lo, hi);
    en += lo + hi;
    un2(FX, lo, hi);
    f[0] += lo + hi;
    un2(FY, lo, hi);
    f[1] += lo + hi;
    un2(FZ, lo, hi);
    f[2] += lo + hi;
    un2(GX, lo, hi);
    g[0] += lo + hi;
    un2(GY, lo, hi);
    g[1] += lo + hi;
    un2(GZ, lo, hi);
    g[2] += lo + hi;
}

template <class R>
__global__ void __launch_bounds__(kEwThreads) k_ew_force(PairParams P, EwParams E,
                                                         const typename Vec4T<R>::type* __restrict__ posq_s,
                                                         const typename Vec4T<R>::type* __restrict__ dipt_s,
                                                         const typename Vec4T<R>::type* __restrict__ vec_s,
                                                         const double4* __restrict__ tctr,
                                                         const double4* __restrict__ text,
                                                         const double* __restrict__ pos_s,
                                                         const int* __restrict__ exs_off, const int* __restrict__ exs_j,
                                                         const double* __restrict__ exs_m,
                                                         const double* __restrict__ exs_s, const int* __restrict__ list,
                                                         const int* __restrict__ count, int n_pad,
                                                         double* __restrict__ out, double* __restrict__ tile_energy) {
    typedef typename Vec4T<R>::type V4;
    __shared__ V4 s_pos[kEwWarps][32], s_dip[kEwWarps][32], s_ind[kEwWarps][32];
    __shared__ EwPackedForceTile s_pk[sizeof(R) == 4 ? kEwWarps : 1];
    __shared__ double s_red[kEwWarps][7][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // One I tile per CTA; warps split the neighbour list (see k_ew_field).
    const int I = blockIdx.x;
    const int i = I * 32 + lane;
    const V4 pi = posq_s[i], di = dipt_s[i], ui = vec_s[i];
    const double4 cA = tctr[I];
    const double4 eAd = text[I];
    const float eA[3] = {(float)eAd.x, (float)eAd.y, (float)eAd.z};
    const float rcm = (float)sqrt(E.rc2) + 1e-3f;
    const int e0 = i < P.n ? exs_off[i] : 0, e1 = i < P.n ? exs_off[i + 1] : 0;
    const R rc2 = (R)E.rc2, damp_r2 = (R)P.damp_r2;
    double F[3] = {0, 0, 0}, G[3] = {0, 0, 0}, en = 0.0;
    const int cnt = count[I];
    for (int t = warp; t < cnt; t += kEwWarps) {
        const int ent = list[(size_t)I * E.cap + t];
        const int J = ent & kTileMask;
        const bool fold = (ent >> 30) & 1, slow = ((unsigned)ent >> 31) & 1u;
        const double4 cB = tctr[J];
        __syncwarp();
        const V4 pj = posq_s[J * 32 + lane], dj = dipt_s[J * 32 + lane], uj = vec_s[J * 32 + lane];
        int nsteps = 16;
        bool staged = false;
        if constexpr (sizeof(R) == 4) {
            if (!slow) {
                // Only the J atoms within the cutoff of the I tile's box,
                // compacted; an odd count is padded with a multipole-free copy.
                float dc[3];
                tile_dc(P, cA, cB, dc);
                const bool act = near_i_tile(P, (float)pj.x, (float)pj.y, (float)pj.z, dc, eA, rcm * rcm, fold);
                const unsigned mk = __ballot_sync(kFull, act);
                const int nact = __popc(mk), k = __popc(mk & ((1u << lane) - 1u));
                if (act) stage_packed_force(s_pk[warp], k, pj, dj, uj);
                if ((nact & 1) && act && k == nact - 1)
                    stage_packed_force(s_pk[warp], nact, make_float4(pj.x, pj.y, pj.z, 0.0f),
                                       make_float4(0.0f, 0.0f, 0.0f, dj.w), make_float4(0.0f, 0.0f, 0.0f, 0.0f));
                nsteps = (nact + 1) >> 1;
                staged = true;
            }
        }
        if (!staged) {
            s_pos[warp][lane] = pj;
            s_dip[warp][lane] = dj;
            s_ind[warp][lane] = uj;
        }
        __syncwarp();
        R ox, oy, oz;
        tile_shift<R>(P, cA, cB, pi.x, pi.y, pi.z, ox, oy, oz);
        R f[3] = {0, 0, 0}, g[3] = {0, 0, 0}, e = 0;
        if constexpr (sizeof(R) == 4) {
            if (!slow) {
                const float iti = 1.0f / (float)di.w;
                if (fold) ew_force_walk_x2<true>(P, E, s_pk[warp], ox, oy, oz, pi.w, di, ui, iti, rc2, damp_r2, nsteps, e, f, g);
                else ew_force_walk_x2<false>(P, E, s_pk[warp], ox, oy, oz, pi.w, di, ui, iti, rc2, damp_r2, nsteps, e, f, g);
                for (int c = 0; c < 3; c++) {
                    F[c] += (double)f[c];
                    G[c] += (double)g[c];
                }
                en += (double)e;
                continue;
            }
        }
        if (slow) {
            const unsigned part = partner_bits(exs_j, e0, e1, J * 32);
            if (fold) ew_force_walk<R, true, true>(P, E, s_pos[warp], s_dip[warp], s_ind[warp], i, J * 32, ox, oy, oz, pi.w, di, ui, part, rc2, damp_r2, e, f, g);
            else ew_force_walk<R, false, true>(P, E, s_pos[warp], s_dip[warp], s_ind[warp], i, J * 32, ox, oy, oz, pi.w, di, ui, part, rc2, damp_r2, e, f, g);
        } else if (fold) {
            ew_force_walk<R, true, false>(P, E, s_pos[warp], s_dip[warp], s_ind[warp], i, J * 32, ox, oy, oz, pi.w, di, ui, 0u, rc2, damp_r2, e, f, g);
        } else {
            ew_force_walk<R, false, false>(P, E, s_pos[warp], s_dip[warp], s_ind[warp], i, J * 32, ox, oy, oz, pi.w, di, ui, 0u, rc2, damp_r2, e, f, g);
        }
        for (int c = 0; c < 3; c++) {
            F[c] += (double)f[c];
            G[c] += (double)g[c];
        }
        en += (double)e;
    }
    for (int c = 0; c < 3; c++) {
        s_red[warp][c][lane] = F[c];
        s_red[warp][3 + c][lane] = G[c];
    }
    s_red[warp][6][lane] = en;
    __syncthreads();
    if (warp != 0) return;
    for (int w = 1; w < kEwWarps; w++) {
        for (int c = 0; c < 3; c++) {
            F[c] += s_red[w][c][lane];
            G[c] += s_red[w][3 + c][lane];
        }
        en += s_red[w][6][lane];
    }
    if (i < P.n) {
        ew_force_exceptions<R>(P, E, pos_s, posq_s, dipt_s, vec_s, exs_off, exs_j, exs_m, exs_s, i, en, F, G);
    } else {
        F[0] = F[1] = F[2] = G[0] = G[1] = G[2] = en = 0.0;
    }
    for (int c = 0; c < 3; c++) {
        out[(size_t)c * n_pad + i] = F[c];
        out[(size_t)(3 + c) * n_pad + i] = G[c];
    }
    en = warp_sum(en);
    if (lane == 0) tile_energy[I] = en;
}

// ---------------------------------------------------------------------------
// PME.
// ---------------------------------------------------------------------------
// theta[j] = M5(w + j), j = 0..4 (grid point floor(u) - j), and derivatives,
// by the cardinal B-spline recursion M_k(x) = (x M_{k-1}(x) + (k - x) M_{k-1}(x - 1)) / (k - 1).
template <class R, bool SECOND>
__device__ __forceinline__ void bspline5(R w, R* th, R* d1, R* d2) {
    R m[kOrder];
    m[0] = w;
    m[1] = R(1) - w;
    m[2] = m[3] = m[4] = R(0);
    R m3[kOrder], m4[kOrder];
#pragma unroll
    for (int k = 3; k <= kOrder; k++) {
        R nw[kOrder];
        const R inv = R(1) / R(k - 1);
#pragma unroll
        for (int j = 0; j < kOrder; j++) {
            if (j >= k) {
                nw[j] = R(0);
                continue;
            }
            R a = j < k - 1 ? m[j] : R(0);
            R b = j >= 1 ? m[j - 1] : R(0);
            nw[j] = ((w + R(j)) * a + (R(k) - w - R(j)) * b) * inv;
        }
#pragma unroll
        for (int j = 0; j < kOrder; j++) m[j] = nw[j];
        if (k == 3) {
#pragma unroll
            for (int j = 0; j < kOrder; j++) m3[j] = m[j];
        }
        if (k == 4) {
#pragma unroll
            for (int j = 0; j < kOrder; j++) m4[j] = m[j];
        }
    }
#pragma unroll
    for (int j = 0; j < kOrder; j++) {
        th[j] = m[j];
        d1[j] = m4[j] - (j >= 1 ? m4[j - 1] : R(0));
        if (SECOND) d2[j] = m3[j] - R(2) * (j >= 1 ? m3[j - 1] : R(0)) + (j >= 2 ? m3[j - 2] : R(0));
    }
}

struct SplinePos {
    int base[3];
};

template <class R, bool SECOND>
__device__ __forceinline__ void atom_splines(const PmeGrid& G, const double* __restrict__ pos_s, int k, int* base,
                                             R th[3][kOrder], R d1[3][kOrder], R d2[3][kOrder]) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
        double f = pos_s[3 * k + c] * G.invL[c];
        f -= floor(f);
        double u = f * G.K[c];
        int b = (int)floor(u);
        double w = u - b;
        if (b >= G.K[c]) b -= G.K[c];
        // A non-finite position must not index outside the grid.
        if (!(b >= 0 && b < G.K[c]) || !(w >= 0.0 && w <= 1.0)) {
            b = 0;
            w = 0.0;
        }
        base[c] = b;
        bspline5<R, SECOND>((R)w, th[c], d1[c], d2[c]);
    }
}

__device__ __forceinline__ int wrap(int g, int K) { return g < 0 ? g + K : g; }

// KIND 0: (q, p) from posq_s/dipt_s; 1: (0, v) from vec_s; 2: (q, p + mu).
template <class R, int KIND>
__global__ void k_pme_spread(PmeGrid G, int n, const double* __restrict__ pos_s,
                             const typename Vec4T<R>::type* __restrict__ posq_s,
                             const typename Vec4T<R>::type* __restrict__ dipt_s,
                             const typename Vec4T<R>::type* __restrict__ vec_s,
                             unsigned long long* __restrict__ gfix, double* __restrict__ gdbl) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int base[3];
    R th[3][kOrder], d1[3][kOrder], d2[3][kOrder];
    atom_splines<R, false>(G, pos_s, k, base, th, d1, d2);
    R q = R(0), dx = R(0), dy = R(0), dz = R(0);
    if (KIND != 1) q = posq_s[k].w;
    if (KIND == 0 || KIND == 2) {
        const typename Vec4T<R>::type p = dipt_s[k];
        dx = p.x;
        dy = p.y;
        dz = p.z;
    }
    if (KIND == 1 || KIND == 2) {
        const typename Vec4T<R>::type v = vec_s[k];
        dx += v.x;
        dy += v.y;
        dz += v.z;
    }
    dx *= (R)G.sc[0];
    dy *= (R)G.sc[1];
    dz *= (R)G.sc[2];
#pragma unroll
    for (int a = 0; a < kOrder; a++) {
        const int gx = wrap(base[0] - a, G.K[0]);
#pragma unroll
        for (int b = 0; b < kOrder; b++) {
            const int gy = wrap(base[1] - b, G.K[1]);
            const R A = th[0][a] * th[1][b];
            const R S = q * A + dx * d1[0][a] * th[1][b] + dy * th[0][a] * d1[1][b];
            const R Z = dz * A;
            const size_t row = ((size_t)gx * G.K[1] + gy) * G.K[2];
#pragma unroll
            for (int c = 0; c < kOrder; c++) {
                const int gz = wrap(base[2] - c, G.K[2]);
                const R v = S * th[2][c] + Z * d1[2][c];
                if (sizeof(R) == 4)
                    atomicAdd(gfix + row + gz, (unsigned long long)__float2ll_rn((float)v * 4294967296.0f));
                else
                    atomicAdd(gdbl + row + gz, (double)v);
            }
        }
    }
}

// Fixed-point grid to G (FP32 for the solver passes, FP64 for the energy
// pass), clearing it for the next spread.
template <class G>
__global__ void k_pme_fix_to_real(size_t ng, unsigned long long* __restrict__ gfix, G* __restrict__ out) {
    size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ng) return;
    long long v = (long long)gfix[k];
    gfix[k] = 0ull;
    out[k] = (G)((double)v * kFixInv);
}

// FP32 version, four words per thread: v 2^-32 = hi + lo 2^-32 with hi the
// signed upper and lo the unsigned lower 32 bits (two 32-bit conversions).
__device__ __forceinline__ float fix_to_float(unsigned long long u) {
    const int hi = (int)(long long)(u >> 32);
    const unsigned lo = (unsigned)u;
    return __fmaf_rn((float)lo, 2.3283064365386963e-10f, (float)hi);
}
__global__ void k_pme_fix_to_f32x4(size_t ng, unsigned long long* __restrict__ gfix, float* __restrict__ out) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t k = 4 * q;
    if (k + 3 < ng) {
        ulonglong2* g2 = reinterpret_cast<ulonglong2*>(gfix + k);
        const ulonglong2 a = g2[0], b = g2[1];
        g2[0] = make_ulonglong2(0ull, 0ull);
        g2[1] = make_ulonglong2(0ull, 0ull);
        *reinterpret_cast<float4*>(out + k) =
            make_float4(fix_to_float(a.x), fix_to_float(a.y), fix_to_float(b.x), fix_to_float(b.y));
    } else {
        for (size_t j = k; j < ng; j++) {
            out[j] = fix_to_float(gfix[j]);
            gfix[j] = 0ull;
        }
    }
}

template <class R>
struct Cplx;
template <>
struct Cplx<float> {
    typedef cufftComplex type;
};
template <>
struct Cplx<double> {
    typedef cufftDoubleComplex type;
};

// F *= C; with energy, block partials of 1/2 sum_m C |F|^2 over the full
// spectrum (half-spectrum entries other than kz = 0 and kz = K3/2 count twice).
template <class R, bool ENERGY>
__global__ void k_pme_convolve(size_t nc, int kzn, int K3, const R* __restrict__ C, typename Cplx<R>::type* __restrict__ F,
                               double* __restrict__ epart) {
    __shared__ double red[40];
    size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (k < nc) {
        typename Cplx<R>::type f = F[k];
        R c = C[k];
        if (ENERGY) {
            int kz = (int)(k % kzn);
            double w = (kz == 0 || 2 * kz == K3) ? 0.5 : 1.0;
            e = w * (double)c * ((double)f.x * f.x + (double)f.y * f.y);
        }
        f.x *= c;
        f.y *= c;
        F[k] = f;
    }
    if (ENERGY) {
        e = block_sum(e, red);
        if (threadIdx.x == 0) epart[blockIdx.x] = e;
    }
}

// Influence function C(m) = exp(-pi^2 m^2/alpha^2)/(pi V m^2) |b(m)|^2 on the
// half spectrum, m_k = (i_k or i_k - K_k)/L_k.
template <class R>
__global__ void k_pme_influence(PmeGrid G, double alpha, const double* __restrict__ mx,
                                const double* __restrict__ my, const double* __restrict__ mz, R* __restrict__ C) {
    const int kzn = G.K[2] / 2 + 1;
    const size_t nc = (size_t)G.K[0] * G.K[1] * kzn;
    size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nc) return;
    int iz = (int)(k % kzn);
    int iy = (int)((k / kzn) % G.K[1]);
    int ix = (int)(k / ((size_t)kzn * G.K[1]));
    double fx = (ix <= G.K[0] / 2 ? ix : ix - G.K[0]) * G.invL[0];
    double fy = (iy <= G.K[1] / 2 ? iy : iy - G.K[1]) * G.invL[1];
    double fz = iz * G.invL[2];
    double m2 = fx * fx + fy * fy + fz * fz;
    double V = G.L[0] * G.L[1] * G.L[2];
    double c = 0.0;
    if (m2 > 0.0) c = exp(-kPi * kPi * m2 / (alpha * alpha)) / (kPi * V * m2) * mx[ix] * my[iy] * mz[iz];
    C[k] = (R)c;
}

// Field -grad phi at every atom (+ self term selfc * d) into partial slot 1;
// FORCE: force q E + (d.grad) E in components 0..2 and E in 3..5.
template <class R, class GT, int KIND, bool FORCE>
__global__ void k_pme_gather(PmeGrid G, int n, int n_pad, double selfc, const double* __restrict__ pos_s,
                             const typename Vec4T<R>::type* __restrict__ posq_s,
                             const typename Vec4T<R>::type* __restrict__ dipt_s,
                             const typename Vec4T<R>::type* __restrict__ vec_s, const GT* __restrict__ phi,
                             double* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_pad) return;
    if (k >= n) {
        for (int c = 0; c < (FORCE ? 6 : 3); c++) out[(size_t)c * n_pad + k] = 0.0;
        return;
    }
    int base[3];
    R th[3][kOrder], d1[3][kOrder], d2[3][kOrder];
    atom_splines<R, FORCE>(G, pos_s, k, base, th, d1, d2);
    R ex = 0, ey = 0, ez = 0, hxx = 0, hyy = 0, hzz = 0, hxy = 0, hxz = 0, hyz = 0;
#pragma unroll
    for (int a = 0; a < kOrder; a++) {
        const int gx = wrap(base[0] - a, G.K[0]);
#pragma unroll
        for (int b = 0; b < kOrder; b++) {
            const int gy = wrap(base[1] - b, G.K[1]);
            const size_t row = ((size_t)gx * G.K[1] + gy) * G.K[2];
            R s0 = 0, s1 = 0, s2 = 0;   // sum_c phi th_z, phi d1_z, phi d2_z
#pragma unroll
            for (int c = 0; c < kOrder; c++) {
                const R p = (R)phi[row + wrap(base[2] - c, G.K[2])];
                s0 += p * th[2][c];
                s1 += p * d1[2][c];
                if (FORCE) s2 += p * d2[2][c];
            }
            const R tx = th[0][a], ty = th[1][b], gxv = d1[0][a], gyv = d1[1][b];
            ex -= gxv * ty * s0;
            ey -= tx * gyv * s0;
            ez -= tx * ty * s1;
            if (FORCE) {
                hxx -= d2[0][a] * ty * s0;
                hyy -= tx * d2[1][b] * s0;
                hzz -= tx * ty * s2;
                hxy -= gxv * gyv * s0;
                hxz -= gxv * ty * s1;
                hyz -= tx * gyv * s1;
            }
        }
    }
    const double sx = G.sc[0], sy = G.sc[1], sz = G.sc[2];
    double E[3] = {(double)ex * sx, (double)ey * sy, (double)ez * sz};
    if (!FORCE) {
        d3 dd{0.0, 0.0, 0.0};
        if (KIND == 0) {
            const typename Vec4T<R>::type p = dipt_s[k];
            dd = {(double)p.x, (double)p.y, (double)p.z};
        } else {
            const typename Vec4T<R>::type v = vec_s[k];
            dd = {(double)v.x, (double)v.y, (double)v.z};
        }
        out[k] = E[0] + selfc * dd.x;
        out[(size_t)n_pad + k] = E[1] + selfc * dd.y;
        out[2 * (size_t)n_pad + k] = E[2] + selfc * dd.z;
    } else {
        // dE_b/dx_a = -sum phi d_a d_b Th  (hab above, scaled by sc_a sc_b)
        double H[3][3];
        H[0][0] = (double)hxx * sx * sx;
        H[1][1] = (double)hyy * sy * sy;
        H[2][2] = (double)hzz * sz * sz;
        H[0][1] = H[1][0] = (double)hxy * sx * sy;
        H[0][2] = H[2][0] = (double)hxz * sx * sz;
        H[1][2] = H[2][1] = (double)hyz * sy * sz;
        const typename Vec4T<R>::type p = dipt_s[k], v = vec_s[k];
        const double q = (double)posq_s[k].w;
        const double d[3] = {(double)p.x + (double)v.x, (double)p.y + (double)v.y, (double)p.z + (double)v.z};
        for (int a = 0; a < 3; a++) {
            double f = q * E[a];
            for (int b = 0; b < 3; b++) f += d[b] * H[a][b];
            out[(size_t)a * n_pad + k] = f;
            out[(size_t)(3 + a) * n_pad + k] = E[a];
        }
    }
}

// Induced dipoles into the sorted records (vec_s = (mu, thole)).
template <class R>
__global__ void k_ew_pack_mu(int n, const int* __restrict__ rank, const double* __restrict__ mu,
                             const double* __restrict__ thole, typename Vec4T<R>::type* __restrict__ vec_s) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    typename Vec4T<R>::type o;
    o.x = (R)mu[3 * i];
    o.y = (R)mu[3 * i + 1];
    o.z = (R)mu[3 * i + 2];
    o.w = (R)thole[i];
    vec_s[rank[i]] = o;
}

// The induced dipoles' own records (Direct polarization): charge 0 and
// permanent dipole 0, positions and Thole factors kept.
template <class R>
__global__ void k_ew_records0(int n_pad, const typename Vec4T<R>::type* __restrict__ posq_s,
                              const typename Vec4T<R>::type* __restrict__ dipt_s,
                              typename Vec4T<R>::type* __restrict__ posq0, typename Vec4T<R>::type* __restrict__ dipt0) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_pad) return;
    typename Vec4T<R>::type p = posq_s[k], t = dipt_s[k];
    p.w = R(0);
    t.x = t.y = t.z = R(0);
    posq0[k] = p;
    dipt0[k] = t;
}

// Forces and torques in index order, per-atom energy terms (self, induction).
// The self terms cancel the erf self-interaction that reciprocal space holds
// for every site, so they use the same (R-rounded) charges and dipoles the
// spread used: -alpha/sqrt(pi) q^2 - 2 alpha^3/(3 sqrt(pi)) |p + mu|^2, plus
// 1/2 |mu|^2 / alpha_i.  The torque on the permanent dipole is p x (field + selfc (p + mu)).
template <class R>
__global__ void k_ew_finish(int n, int n_pad, const int* __restrict__ rank, const double* __restrict__ partial,
                            const typename Vec4T<R>::type* __restrict__ posq_s,
                            const typename Vec4T<R>::type* __restrict__ dipt_s,
                            const typename Vec4T<R>::type* __restrict__ vec_s, const double* __restrict__ lab,
                            const double* __restrict__ pol, double alpha, double selfc, int recip,
                            double* __restrict__ fpair, double* __restrict__ torque, double* __restrict__ epart,
                            int subtract = 0) {
    __shared__ double red[40];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (i < n) {
        const int k = rank[i];
        const size_t s1 = 6 * (size_t)n_pad;
        double F[3], G[3];
        for (int c = 0; c < 3; c++) {
            F[c] = partial[(size_t)c * n_pad + k];
            G[c] = partial[(size_t)(3 + c) * n_pad + k];
            if (recip) {
                F[c] += partial[s1 + (size_t)c * n_pad + k];
                G[c] += partial[s1 + (size_t)(3 + c) * n_pad + k];
            }
        }
        const typename Vec4T<R>::type P = dipt_s[k], U = vec_s[k];
        const d3 u = {(double)U.x, (double)U.y, (double)U.z};
        const d3 t = {(double)P.x + u.x, (double)P.y + u.y, (double)P.z + u.z};
        const d3 p = ld3(lab + 3 * i);
        G[0] += selfc * t.x;
        G[1] += selfc * t.y;
        G[2] += selfc * t.z;
        const double q = (double)posq_s[k].w;
        e = -alpha / kSqrtPi * q * q - 2.0 * alpha * alpha * alpha / (3.0 * kSqrtPi) * dot(t, t);
        if (subtract) {
            // The induced dipoles' own pass: its forces come off the total;
            // nothing acts on the permanent dipoles, and no induction term.
            fpair[3 * i] -= F[0];
            fpair[3 * i + 1] -= F[1];
            fpair[3 * i + 2] -= F[2];
        } else {
            fpair[3 * i] = F[0];
            fpair[3 * i + 1] = F[1];
            fpair[3 * i + 2] = F[2];
            torque[3 * i] = p.y * G[2] - p.z * G[1];
            torque[3 * i + 1] = p.z * G[0] - p.x * G[2];
            torque[3 * i + 2] = p.x * G[1] - p.y * G[0];
            if (pol[i] > 0.0) e += 0.5 * dot(u, u) / pol[i];
        }
    }
    e = block_sum(e, red);
    if (threadIdx.x == 0) epart[blockIdx.x] = e;
}

// *out = s + plasma, or with subtract *out -= s + plasma.
__global__ void k_ew_energy_sum(int n_a, const double* __restrict__ a, int n_b, const double* __restrict__ b, int n_c,
                                const double* __restrict__ c, double plasma, double* __restrict__ out,
                                int subtract = 0) {
    __shared__ double red[40];
    double s = sum_partials(a, n_a, red);
    s += sum_partials(b, n_b, red);
    s += sum_partials(c, n_c, red);
    if (threadIdx.x == 0) *out = subtract ? *out - (s + plasma) : s + plasma;
}

inline int nblk(size_t n, int t) { return (int)((n + t - 1) / t); }

// B-spline moduli 1/|sum_{j=0}^{3} M5(j+1) exp(2 pi i m j / K)|^2; a (near) zero
// denominator (m = K/2) takes the mean of its neighbours.
std::vector<double> bspline_moduli(int K) {
    const double M[4] = {1.0 / 24.0, 11.0 / 24.0, 11.0 / 24.0, 1.0 / 24.0};
    std::vector<double> den(K);
    for (int m = 0; m < K; m++) {
        double re = 0.0, im = 0.0;
        for (int j = 0; j < 4; j++) {
            double ph = 2.0 * kPi * m * j / K;
            re += M[j] * std::cos(ph);
            im += M[j] * std::sin(ph);
        }
        den[m] = re * re + im * im;
    }
    std::vector<double> mod(den);
    for (int m = 0; m < K; m++)
        if (mod[m] < 1e-7) mod[m] = 0.5 * (mod[(m + K - 1) % K] + mod[(m + 1) % K]);
    for (int m = 0; m < K; m++) mod[m] = 1.0 / mod[m];
    return mod;
}

int smooth_size(int n) {
    for (int m = std::max(n, 1);; m++) {
        int k = m;
        for (int p : {2, 3, 5, 7})
            while (k % p == 0) k /= p;
        if (k == 1) return m;
    }
}

void check_cufft(cufftResult r, const char* what) {
    if (r != CUFFT_SUCCESS) throw TdpError{TDP_ERR_CUDA, std::string(what) + ": cuFFT error " + std::to_string((int)r)};
}

}  // namespace

// One FFT grid: real grid, half spectrum, influence function, cuFFT plans.
struct FftGrid {
    bool dbl = false;
    void* real = nullptr;
    void* cplx = nullptr;
    void* C = nullptr;
    cufftHandle fwd = 0, inv = 0;
    bool plans = false;
};

struct Ewald {
    int precision = TDP_PRECISION_MIXED;
    bool vacuum = false;   // variational NoCutoff model: real space only, alpha = 0
    std::vector<void*> owned;
    int cap = 0;
    int* list = nullptr;
    int* count = nullptr;
    int* overflow = nullptr;
    int* h_overflow = nullptr;
    double* tile_energy = nullptr;
    double* atom_epart = nullptr;
    int n_atom_blk = 1;
    // Grid (planned on the first ewald_prepare).  The solver passes run on
    // `it` (FP32 in the mixed form); the energy/force pass runs on `en64`
    // (FP64 FFT: the reciprocal energy holds every atom's erf self-interaction,
    // which the analytic self term cancels, so it needs FP64) -- in the plain
    // form both are the same FP64 grid.
    bool planned = false;
    int K[3] = {0, 0, 0};
    double alpha = 0.0, cutoff = 0.0, box[3] = {0, 0, 0};
    PmeGrid G{};
    EwParams E{};
    unsigned long long* gfix = nullptr;
    FftGrid it, en64;
    double *modx = nullptr, *mody = nullptr, *modz = nullptr;
    double* rec_epart = nullptr;
    int n_rec_blk = 1;
    int launches = 0;
    // Direct polarization: records of the induced dipoles alone (positions
    // with charge 0, then zero permanent dipoles with the Thole factors),
    // 2 * n_pad records of the form's precision.
    void* rec0 = nullptr;

    FftGrid& energy_grid() { return precision == TDP_PRECISION_DOUBLE ? it : en64; }

    ~Ewald() {
        for (FftGrid* g : {&it, &en64})
            if (g->plans) {
                cufftDestroy(g->fwd);
                cufftDestroy(g->inv);
            }
        for (void* p : owned) cudaFree(p);
        if (h_overflow) cudaFreeHost(h_overflow);
    }
};

namespace {

void make_grid(Ewald* e, FftGrid& g, bool dbl) {
    const size_t ng = (size_t)e->K[0] * e->K[1] * e->K[2];
    const size_t nc = (size_t)e->K[0] * e->K[1] * (e->K[2] / 2 + 1);
    g.dbl = dbl;
    g.real = dbl ? (void*)dalloc<double>(ng, e->owned) : (void*)dalloc<float>(ng, e->owned);
    g.cplx = dbl ? (void*)dalloc<cufftDoubleComplex>(nc, e->owned) : (void*)dalloc<cufftComplex>(nc, e->owned);
    g.C = dbl ? (void*)dalloc<double>(nc, e->owned) : (void*)dalloc<float>(nc, e->owned);
    check_cufft(cufftPlan3d(&g.fwd, e->K[0], e->K[1], e->K[2], dbl ? CUFFT_D2Z : CUFFT_R2C), "cufftPlan3d");
    if (cufftPlan3d(&g.inv, e->K[0], e->K[1], e->K[2], dbl ? CUFFT_Z2D : CUFFT_C2R) != CUFFT_SUCCESS) {
        cufftDestroy(g.fwd);
        throw TdpError{TDP_ERR_CUDA, "cufftPlan3d: inverse plan failed"};
    }
    g.plans = true;
}

void influence(Ewald* e, FftGrid& g, cudaStream_t st) {
    const size_t nc = (size_t)e->K[0] * e->K[1] * (e->K[2] / 2 + 1);
    if (g.dbl)
        k_pme_influence<double><<<nblk(nc, 256), 256, 0, st>>>(e->G, e->alpha, e->modx, e->mody, e->modz, (double*)g.C);
    else
        k_pme_influence<float><<<nblk(nc, 256), 256, 0, st>>>(e->G, e->alpha, e->modx, e->mody, e->modz, (float*)g.C);
    TDP_CUDA(cudaGetLastError());
}

}  // namespace

Ewald* ewald_create(const Dev& d, int precision, bool vacuum, bool direct) {
    Ewald* e = new Ewald();
    try {
        e->precision = precision;
        e->vacuum = vacuum;
        if (direct)
            e->rec0 = dalloc<char>(2 * (size_t)d.n_pad * (precision == TDP_PRECISION_DOUBLE ? 32 : 16), e->owned);
        const int nt = std::max(1, d.pp.n_tiles);
        e->cap = vacuum ? nt : std::min(nt, 2048);
        e->list = dalloc<int>((size_t)nt * e->cap, e->owned);
        e->count = dalloc<int>(nt, e->owned);
        e->overflow = dalloc<int>(1, e->owned);
        e->tile_energy = dalloc<double>(nt, e->owned);
        e->n_atom_blk = std::max(1, (d.n + kVecThreads - 1) / kVecThreads);
        e->atom_epart = dalloc<double>(e->n_atom_blk, e->owned);
        TDP_CUDA(cudaMallocHost(&e->h_overflow, sizeof(int)));
        *e->h_overflow = 0;
    } catch (...) {
        delete e;
        throw;
    }
    return e;
}

void ewald_destroy(Ewald* e) { delete e; }

void ewald_prepare(Ewald* e, const Dev& d, const double box[3], double cutoff, double tol, double alpha_in,
                   const int grid_in[3], cudaStream_t st) {
    if (e->vacuum) {
        e->planned = true;
        e->alpha = 0.0;
        e->E.alpha = 0.0;
        e->E.ca = 0.0;
        e->E.a2 = 0.0;
        e->E.rc2 = INFINITY;
        e->E.selfc = 0.0;
        e->E.cap = e->cap;
        e->n_rec_blk = 0;
        return;
    }
    for (int k = 0; k < 3; k++)
        if (!(box[k] > 0.0)) throw TdpError{TDP_ERR_INVALID_ARGUMENT, "the Ewald mode needs a periodic box"};
    if (!e->planned) {
        double a = alpha_in > 0.0 ? alpha_in : std::sqrt(-std::log(2.0 * tol)) / cutoff;
        for (int k = 0; k < 3; k++) {
            int g = grid_in[0] > 0 ? grid_in[k]
                                   : smooth_size(std::max(6, (int)std::ceil(2.0 * a * box[k] / (3.0 * std::pow(tol, 0.2)))));
            if (g < kOrder) throw TdpError{TDP_ERR_INVALID_ARGUMENT, "PME grid dimension below the spline order 5"};
            e->K[k] = g;
        }
        e->alpha = a;
        const size_t ng = (size_t)e->K[0] * e->K[1] * e->K[2];
        const size_t nc = (size_t)e->K[0] * e->K[1] * (e->K[2] / 2 + 1);
        const bool dbl = e->precision == TDP_PRECISION_DOUBLE;
        if (!dbl) e->gfix = dalloc<unsigned long long>(ng, e->owned);
        e->n_rec_blk = nblk(nc, kVecThreads);
        e->rec_epart = dalloc<double>(e->n_rec_blk, e->owned);
        std::vector<double> m[3];
        for (int k = 0; k < 3; k++) m[k] = bspline_moduli(e->K[k]);
        e->modx = dalloc<double>(e->K[0], e->owned);
        e->mody = dalloc<double>(e->K[1], e->owned);
        e->modz = dalloc<double>(e->K[2], e->owned);
        upload(e->modx, m[0].data(), sizeof(double) * e->K[0]);
        upload(e->mody, m[1].data(), sizeof(double) * e->K[1]);
        upload(e->modz, m[2].data(), sizeof(double) * e->K[2]);
        make_grid(e, e->it, dbl);
        if (!dbl) make_grid(e, e->en64, true);
        e->planned = true;
        e->box[0] = e->box[1] = e->box[2] = -1.0;
    }
    e->cutoff = cutoff;
    const double a = e->alpha;
    e->E.alpha = a;
    e->E.ca = 2.0 * a / kSqrtPi;
    e->E.a2 = 2.0 * a * a;
    e->E.rc2 = cutoff * cutoff;
    e->E.selfc = 4.0 * a * a * a / (3.0 * kSqrtPi);
    e->E.cap = e->cap;
    if (box[0] != e->box[0] || box[1] != e->box[1] || box[2] != e->box[2]) {
        for (int k = 0; k < 3; k++) {
            e->box[k] = box[k];
            e->G.K[k] = e->K[k];
            e->G.L[k] = box[k];
            e->G.invL[k] = 1.0 / box[k];
            e->G.sc[k] = e->K[k] / box[k];
        }
        influence(e, e->it, st);
        if (e->precision != TDP_PRECISION_DOUBLE) influence(e, e->en64, st);
    }
    (void)d;
}

void ewald_params(const Ewald* e, double* alpha, int grid[3]) {
    *alpha = e->alpha;
    for (int k = 0; k < 3; k++) grid[k] = e->K[k];
}

int ewald_list_overflow(const Ewald* e) { return *e->h_overflow; }
int pme_smooth_size(int n) { return smooth_size(n); }
int ewald_last_launches(const Ewald* e) { return e->launches; }

namespace {

// Reciprocal space of one density: spread (R arithmetic), then FFT,
// convolution and inverse FFT on grid g (element type GT).
template <class R, class GT, int KIND>
void pme_potential(Ewald* e, const Dev& d, FftGrid& g, bool energy, cudaStream_t st,
                   const typename Vec4T<R>::type* posq = nullptr, const typename Vec4T<R>::type* dipt = nullptr) {
    typedef typename Vec4T<R>::type V4;
    if (!posq) posq = (const V4*)d.posq_s;
    if (!dipt) dipt = (const V4*)d.dipt_s;
    const size_t ng = (size_t)e->K[0] * e->K[1] * e->K[2];
    const size_t nc = (size_t)e->K[0] * e->K[1] * (e->K[2] / 2 + 1);
    const bool fix = sizeof(R) == 4;   // the mixed form spreads into the fixed-point grid
    if (!fix) TDP_CUDA(cudaMemsetAsync(g.real, 0, ng * sizeof(double), st));
    k_pme_spread<R, KIND><<<nblk((size_t)d.n, 128), 128, 0, st>>>(e->G, d.n, d.pos_s, posq, dipt,
                                                                   (const V4*)d.vec_s, e->gfix,
                                                                   fix ? nullptr : (double*)g.real);
    e->launches++;
    if (fix) {
        if (sizeof(GT) == 4)
            k_pme_fix_to_f32x4<<<nblk((ng + 3) / 4, 256), 256, 0, st>>>(ng, e->gfix, (float*)g.real);
        else
            k_pme_fix_to_real<GT><<<nblk(ng, 256), 256, 0, st>>>(ng, e->gfix, (GT*)g.real);
        e->launches++;
    }
    check_cufft(cufftSetStream(g.fwd, st), "cufftSetStream");
    check_cufft(cufftSetStream(g.inv, st), "cufftSetStream");
    if (sizeof(GT) == 8) check_cufft(cufftExecD2Z(g.fwd, (double*)g.real, (cufftDoubleComplex*)g.cplx), "cufftExecD2Z");
    else check_cufft(cufftExecR2C(g.fwd, (float*)g.real, (cufftComplex*)g.cplx), "cufftExecR2C");
    const int kzn = e->K[2] / 2 + 1;
    if (energy)
        k_pme_convolve<GT, true><<<e->n_rec_blk, kVecThreads, 0, st>>>(nc, kzn, e->K[2], (const GT*)g.C,
                                                                      (typename Cplx<GT>::type*)g.cplx, e->rec_epart);
    else
        k_pme_convolve<GT, false><<<e->n_rec_blk, kVecThreads, 0, st>>>(nc, kzn, e->K[2], (const GT*)g.C,
                                                                       (typename Cplx<GT>::type*)g.cplx, e->rec_epart);
    e->launches++;
    if (sizeof(GT) == 8) check_cufft(cufftExecZ2D(g.inv, (cufftDoubleComplex*)g.cplx, (double*)g.real), "cufftExecZ2D");
    else check_cufft(cufftExecC2R(g.inv, (cufftComplex*)g.cplx, (float*)g.real), "cufftExecC2R");
}

template <class R, int KIND>
void real_field(Ewald* e, const Dev& d, const void* src, cudaStream_t st, const void* lab = nullptr) {
    typedef typename Vec4T<R>::type V4;
    const int blocks = d.pp.n_tiles;
    k_ew_field<R, KIND><<<blocks, kEwThreads, 0, st>>>(d.pp, e->E, (const V4*)d.posq_s, (const V4*)src, d.tctr_s,
                                                      d.text_s, d.pos_s, d.exs_off, d.exs_j, d.exs_m, d.exs_s, e->list, e->count,
                                                      d.n_pad, d.partial, (const V4*)lab);
    e->launches++;
}

}  // namespace

void ewald_build_list(Ewald* e, const Dev& d, cudaStream_t st) {
    TDP_CUDA(cudaMemsetAsync(e->overflow, 0, sizeof(int), st));
    k_ew_tiles<<<(d.pp.n_tiles + kEwWarps - 1) / kEwWarps, kEwThreads, 0, st>>>(d.pp, e->E, d.tctr_s, d.text_s,
                                                                              d.exs_tiles, e->list, e->count,
                                                                              e->overflow);
    TDP_CUDA(cudaMemcpyAsync(e->h_overflow, e->overflow, sizeof(int), cudaMemcpyDeviceToHost, st));
    e->launches++;
}

template <class R>
void ewald_fixed_field(Ewald* e, const Dev& d, cudaStream_t st, const void* operand) {
    typedef typename Vec4T<R>::type V4;
    // The dipole records: the lab-frame permanent dipoles, or (fused start)
    // the operand P = m + mu0, whose field is E + T mu0.
    const V4* dip = operand ? (const V4*)operand : (const V4*)d.dipt_s;
    e->launches = 0;
    ewald_build_list(e, d, st);
    real_field<R, 0>(e, d, dip, st, operand ? d.dipt_s : nullptr);
    TDP_CUDA(cudaGetLastError());
    if (e->vacuum) return;
    pme_potential<R, R, 0>(e, d, e->it, false, st, nullptr, dip);
    k_pme_gather<R, R, 0, false><<<nblk((size_t)d.n_pad, 128), 128, 0, st>>>(
        e->G, d.n, d.n_pad, e->E.selfc, d.pos_s, (const V4*)d.posq_s, dip, (const V4*)d.vec_s,
        (const R*)e->it.real, d.partial + 3 * (size_t)d.n_pad);
    e->launches++;
    TDP_CUDA(cudaGetLastError());
}

template <class R>
void ewald_matvec(Ewald* e, const Dev& d, cudaStream_t st) {
    typedef typename Vec4T<R>::type V4;
    e->launches = 0;
    real_field<R, 1>(e, d, d.vec_s, st);
    TDP_CUDA(cudaGetLastError());
    if (e->vacuum) return;
    pme_potential<R, R, 1>(e, d, e->it, false, st);
    k_pme_gather<R, R, 1, false><<<nblk((size_t)d.n_pad, 128), 128, 0, st>>>(
        e->G, d.n, d.n_pad, e->E.selfc, d.pos_s, (const V4*)d.posq_s, (const V4*)d.dipt_s, (const V4*)d.vec_s,
        (const R*)e->it.real, d.partial + 3 * (size_t)d.n_pad);
    e->launches++;
    TDP_CUDA(cudaGetLastError());
}

namespace {

// One energy/force pass over the records (posq, dipt) and the induced dipoles
// in vec_s.  subtract = 0: forces, torques and the energy are written;
// subtract = 1: the pass's forces and energy come off them (no torques).
template <class R>
void energy_pass(Ewald* e, const Dev& d, const typename Vec4T<R>::type* posq, const typename Vec4T<R>::type* dipt,
                 double plasma, int subtract, cudaStream_t st) {
    typedef typename Vec4T<R>::type V4;
    k_ew_force<R><<<d.pp.n_tiles, kEwThreads, 0, st>>>(d.pp, e->E, posq, dipt, (const V4*)d.vec_s, d.tctr_s,
                                                       d.text_s, d.pos_s, d.exs_off, d.exs_j, d.exs_m, d.exs_s,
                                                       e->list, e->count, d.n_pad, d.partial, e->tile_energy);
    if (!e->vacuum) {
        FftGrid& g = e->energy_grid();
        pme_potential<R, double, 2>(e, d, g, true, st, posq, dipt);
        k_pme_gather<R, double, 2, true><<<nblk((size_t)d.n_pad, 128), 128, 0, st>>>(
            e->G, d.n, d.n_pad, e->E.selfc, d.pos_s, posq, dipt, (const V4*)d.vec_s, (const double*)g.real,
            d.partial + 6 * (size_t)d.n_pad);
    }
    k_ew_finish<R><<<e->n_atom_blk, kVecThreads, 0, st>>>(d.n, d.n_pad, d.rank, d.partial, posq, dipt,
                                                          (const V4*)d.vec_s, d.lab, d.alpha, e->alpha, e->E.selfc,
                                                          e->vacuum ? 0 : 1, d.fpair, d.torque, e->atom_epart,
                                                          subtract);
    k_ew_energy_sum<<<1, kVecThreads, 0, st>>>(d.pp.n_tiles, e->tile_energy, e->n_rec_blk, e->rec_epart,
                                               e->n_atom_blk, e->atom_epart, plasma, d.energy, subtract);
    e->launches += e->vacuum ? 3 : 4;
}

}  // namespace

template <class R>
void ewald_energy(Ewald* e, const Dev& d, double total_charge, cudaStream_t st, bool direct) {
    typedef typename Vec4T<R>::type V4;
    e->launches = 0;
    k_ew_pack_mu<R><<<nblk((size_t)d.n, kVecThreads), kVecThreads, 0, st>>>(d.n, d.rank, d.mu, d.thole, (V4*)d.vec_s);
    e->launches++;
    const double V = e->box[0] * e->box[1] * e->box[2];
    const double plasma =
        e->vacuum ? 0.0 : -kPi * total_charge * total_charge / (2.0 * V * e->alpha * e->alpha);
    energy_pass<R>(e, d, (const V4*)d.posq_s, (const V4*)d.dipt_s, plasma, 0, st);
    if (direct) {
        // Direct polarization: its functional U_perm - mu.E_M + 1/2 mu alpha^-1 mu
        // is the Mutual one minus U(0, mu), the induced dipoles' own Ewald
        // energy (-1/2 mu.T mu), so energy and forces are the Mutual pass's
        // minus those of a pass over the induced dipoles alone.
        if (!e->rec0) throw TdpError{TDP_ERR_CUDA, "Ewald mode: Direct records were not allocated"};
        V4* posq0 = (V4*)e->rec0;
        V4* dipt0 = posq0 + d.n_pad;
        k_ew_records0<R><<<nblk((size_t)d.n_pad, kVecThreads), kVecThreads, 0, st>>>(
            d.n_pad, (const V4*)d.posq_s, (const V4*)d.dipt_s, posq0, dipt0);
        e->launches++;
        energy_pass<R>(e, d, posq0, dipt0, 0.0, 1, st);
    }
    TDP_CUDA(cudaGetLastError());
}

template void ewald_fixed_field<float>(Ewald*, const Dev&, cudaStream_t, const void*);
template void ewald_fixed_field<double>(Ewald*, const Dev&, cudaStream_t, const void*);
template void ewald_matvec<float>(Ewald*, const Dev&, cudaStream_t);
template void ewald_matvec<double>(Ewald*, const Dev&, cudaStream_t);
template void ewald_energy<float>(Ewald*, const Dev&, double, cudaStream_t, bool);
template void ewald_energy<double>(Ewald*, const Dev&, double, cudaStream_t, bool);

}  // namespace tdp
