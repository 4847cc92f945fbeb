// tdp_adjoint.cu -- hand-written reverse mode of the TholeDipoleForce
// evaluation (reference semantics, FP64) for tdp_adjoint.
//
// Forward chain (aehogan/tholedipoleplugin ReferenceTholeDipoleForce.cpp,
// "RTDF.cpp"):  mu_lab = R(S mu_mol) (rotation :477-571, S = chirality sign);
// E = Efix(q, mu_lab, t) (:678-733);  A mu = E with A = alpha^-1 - T(t)
// (fixed point of :820-851);  (F_pair, tau) = Pair(q, mu_lab, mu, t)
// (:129-393);  F = F_pair + M tau (:915-1115).  Given g = dL/dF and
// gE = dL/dE:
//   g_tau = M^T g                                   (k_torque_vjp)
//   a     = d/d(q, mu_lab, mu, t) of  gE*E_pair + g.F_pair + g_tau.tau
//                                                   (k_pair_vjp)
//   A lambda = a_mu                                 (one CG solve, same system)
//   b     = d/d(q, mu_lab, t) of lambda . Efix      (k_fixed_vjp)
//   c_t   = d/dt of lambda^T T(t) mu                (k_matvec_t_vjp)
//   dL/dalpha_i = (a_mu + T lambda)_i . (E + T mu)_i   (= lambda_i.mu_i/alpha_i^2)
//   dL/dq = a_q + b_q,  dL/dt = a_t + b_t + c_t,
//   dL/dmu_mol = S R^T (a_mu_lab + b_mu_lab).
// Extrapolated polarization (:853-909: mu_0 = alpha E, mu_k = alpha (E + T
// mu_(k-1)), mu = sum_k c_k mu_k) has no solve; its adjoint runs the
// recursion backwards: gbar_(K-1) = c_(K-1) a_mu, gbar_k = c_k a_mu +
// T (alpha gbar_(k+1)); then lambda = sum_k alpha gbar_k takes the place of
// the adjoint solution in b, dL/dalpha = sum_k gbar_k . (E + T mu_(k-1)) and
// c_t = sum_(k>=1) d/dt of (alpha gbar_k)^T T mu_(k-1).
// For fixed geometry and damping the pair routine's energy, forces and
// torques are bilinear in the two atoms' multipoles (every term is one
// quantity of atom I times one of atom K), so the derivative with respect to
// one atom's multipoles is the pair function evaluated with those multipoles
// set to unit vectors; the Thole-factor derivative flows through the damping
// factors and is taken with a one-direction dual number.  Damping terms are
// recomputed in every pass rather than stored.  Pairs beyond the damping
// range with unit scales (nearly all of a box) take the closed-form lab-frame
// VJP (pair_vjp_lab), a few times cheaper.  Every pair is visited from both
// atoms (each atom owns kLanes threads), so no atomics are needed.
#include "tholedipole_b200.h"
#include <algorithm>
#include "tdp_adjoint.cuh"

namespace tdp {
namespace adj {

// The per-atom reductions below give each atom kLanes consecutive threads:
// lane l visits partners j = l, l + kLanes, ..., and the lanes' sums are
// combined by a fixed xor-shuffle tree, so results do not depend on timing.
constexpr int kLanes = 8;

__device__ __forceinline__ double lane_sum(double v) {
#pragma unroll
    for (int o = kLanes / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, kLanes);
    return v;
}

// a = d/d(q, lab, mu, t) of gE*E_pair + g.F_pair + gT.tau, per atom.  out: n*8.
__global__ void k_pair_vjp(PairParams P, AtomData A, const double* __restrict__ g, const double* __restrict__ gT,
                           double gE, const int* __restrict__ exc_off, const int* __restrict__ exc_j,
                           const double* __restrict__ exc_m, const double* __restrict__ exc_s, double* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int me = t / kLanes, l = t % kLanes;
    const bool act = me < P.n;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (act) {
        for (int j = l; j < P.n; j += kLanes)
            if (j != me) visit_pair(P, A, g, gT, gE, me, j, 1.0, 1.0, acc);
        // Covalent scales: the pair function is linear in (mScale, iScale).
        for (int e = exc_off[me] + l; e < exc_off[me + 1]; e += kLanes)
            visit_pair(P, A, g, gT, gE, me, exc_j[e], exc_m[e] - 1.0, exc_s[e] - 1.0, acc);
    }
    for (int k = 0; k < 8; k++) acc[k] = lane_sum(acc[k]);
    if (act && l == 0)
        for (int k = 0; k < 8; k++) out[8 * me + k] = acc[k];
}

// k_pair_vjp in two passes, for rInvVec[4] = 0 (the default; the closed form
// assumes it).
// Pass 1 (k_pair_vjp_fast): one thread per atom, J atoms staged in shared
// memory 32 at a time; every pair beyond the damping range whose frame row is
// regular takes the closed-form lab-frame VJP in the arithmetic T (FP32 in
// the mixed form, FP64 in the plain form) from a displacement formed in FP64
// with the minimum image and rounded once; per-tile sums are added in FP64.
// The other pairs (damped or degenerate, ~0.6 % of a box) are listed in the
// atom's row of `slow`, in index order (beyond kSlowCap they are evaluated in
// place).  Pass 2 (k_pair_vjp_slow): one warp per atom runs the FP64 routine
// over the listed pairs and the covalent corrections, lane l taking entries
// l, l + 32, ..., and adds the warp's sums, reduced by a fixed shuffle tree.
// Small systems split the J range over blockIdx.y (at most kVjpSplit
// splits) to fill the GPU: split s keeps its own sums and slow rows, and
// pass 2 adds the splits in order.  Both passes are deterministic.
constexpr int kVjpTile = 32;
constexpr int kSlowCap = 192;
// k_pair_vjp_fast at 12 blocks per SM (168 registers, 48 B of spills):
// 7.3 ms per 12,288-atom adjoint against 7.9 ms at 215 registers and 8.2 ms
// at 128 (mixed form).
constexpr int kVjpSplit = 8;
// The FP64 routine out of line, so that the rare overflow of a slow row does
// not set the fast pass's register budget.
__device__ __noinline__ void visit_pair_call(const PairParams& P, const AtomData& A, const double* g,
                                             const double* gT, double gE, int me, int j, double* acc) {
    visit_pair(P, A, g, gT, gE, me, j, 1.0, 1.0, acc);
}
template <class T>
__global__ void __launch_bounds__(kVjpTile, 12) k_pair_vjp_fast(PairParams P, AtomData A, const double* __restrict__ g,
                                                           const double* __restrict__ gT, double gE,
                                                           int* __restrict__ slow, int* __restrict__ nslow,
                                                           double* __restrict__ part_out) {
    typedef V3T<T> W;
    __shared__ double s_pos[3][kVjpTile];
    __shared__ double2 s_yz[kVjpTile];
    __shared__ T s_q[kVjpTile];
    __shared__ T s_v[12][kVjpTile];   // lab, mu, g, gT
    const int me = blockIdx.x * kVjpTile + threadIdx.x;
    const bool act = me < P.n;
    const int mi = act ? me : 0;
    const double px = A.pos[3 * mi], py = A.pos[3 * mi + 1], pz = A.pos[3 * mi + 2];
    const double2 myz = A.yz ? A.yz[mi] : make_double2(py, pz);
    const T q0 = (T)A.q[mi];
    const W m0 = {(T)A.lab[3 * mi], (T)A.lab[3 * mi + 1], (T)A.lab[3 * mi + 2]};
    const W u0 = {(T)A.mu[3 * mi], (T)A.mu[3 * mi + 1], (T)A.mu[3 * mi + 2]};
    const W g0 = {(T)g[3 * mi], (T)g[3 * mi + 1], (T)g[3 * mi + 2]};
    const W t0 = {(T)gT[3 * mi], (T)gT[3 * mi + 1], (T)gT[3 * mi + 2]};
    const T kap = P.mutual ? T(1) : T(-1), tgE = (T)gE;
    const double damp_r2 = P.damp_r2 == 0.0f ? 0.0 : (double)P.damp_r2;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int ns = 0;
    const size_t sm = (size_t)blockIdx.y * P.n + mi;   // (split, atom)
    int* row = slow + sm * kSlowCap;
    const int ntile = (P.n + kVjpTile - 1) / kVjpTile;
    const int tb = (int)(((long)ntile * blockIdx.y) / gridDim.y), te = (int)(((long)ntile * (blockIdx.y + 1)) / gridDim.y);
    for (int base = tb * kVjpTile; base < te * kVjpTile && base < P.n; base += kVjpTile) {
        __syncwarp();
        const int js = base + threadIdx.x;
        if (js < P.n) {
            for (int c = 0; c < 3; c++) {
                s_pos[c][threadIdx.x] = A.pos[3 * js + c];
                s_v[c][threadIdx.x] = (T)A.lab[3 * js + c];
                s_v[3 + c][threadIdx.x] = (T)A.mu[3 * js + c];
                s_v[6 + c][threadIdx.x] = (T)g[3 * js + c];
                s_v[9 + c][threadIdx.x] = (T)gT[3 * js + c];
            }
            s_yz[threadIdx.x] = A.yz ? A.yz[js] : make_double2(A.pos[3 * js + 1], A.pos[3 * js + 2]);
            s_q[threadIdx.x] = (T)A.q[js];
        }
        __syncwarp();
        if (!act) continue;
        const int cnt = min(kVjpTile, P.n - base);
        T part[7] = {0, 0, 0, 0, 0, 0, 0};
        for (int jj = 0; jj < cnt; jj++) {
            const int j = base + jj;
            if (j == me) continue;
            const bool meI = me < j;
            // d = p_K - p_I with I the lower index.
            V3 d = min_image(P, {s_pos[0][jj] - px, s_pos[1][jj] - py, s_pos[2][jj] - pz});
            if (!meI) d = {-d.x, -d.y, -d.z};
            const double2 yj = s_yz[jj];
            const bool yzd = (myz.x != yj.x) || (myz.y != yj.y);
            const double r2 = d.x * d.x + d.y * d.y + d.z * d.z;
            if (!(r2 < damp_r2) && yzd && d.y * d.y + d.z * d.z > 0.0) {
                const W dj = {(T)d.x, (T)d.y, (T)d.z};
                const W mj = {s_v[0][jj], s_v[1][jj], s_v[2][jj]}, uj = {s_v[3][jj], s_v[4][jj], s_v[5][jj]};
                const W gj = {s_v[6][jj], s_v[7][jj], s_v[8][jj]}, tj = {s_v[9][jj], s_v[10][jj], s_v[11][jj]};
                const T qj = s_q[jj];
                T o[7];
                if (meI) pair_vjp_lab<T>(dj, q0, m0, u0, qj, mj, uj, kap, tgE, g0, gj, t0, tj, true, o);
                else pair_vjp_lab<T>(dj, qj, mj, uj, q0, m0, u0, kap, tgE, gj, g0, tj, t0, false, o);
                for (int a = 0; a < 7; a++) part[a] += o[a];
            } else {
                // The count goes on past the row (the list users then scan all
                // partners of this atom).
                if (ns < kSlowCap) row[ns] = j;
                else visit_pair_call(P, A, g, gT, gE, me, j, acc);
                ns++;
            }
        }
        for (int a = 0; a < 7; a++) acc[a] += (double)part[a];
    }
    if (!act) return;
    nslow[sm] = ns;
    for (int k = 0; k < 8; k++) part_out[8 * sm + k] = acc[k];
}

__global__ void k_pair_vjp_slow(PairParams P, AtomData A, const double* __restrict__ g, const double* __restrict__ gT,
                                double gE, int nsplit, const int* __restrict__ slow, const int* __restrict__ nslow,
                                const double* __restrict__ part, const int* __restrict__ exc_off,
                                const int* __restrict__ exc_j, const double* __restrict__ exc_m,
                                const double* __restrict__ exc_s, double* __restrict__ out) {
    const int me = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, l = threadIdx.x & 31;
    if (me >= P.n) return;   // whole warps leave together
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int sp = 0; sp < nsplit; sp++) {
        const size_t sm = (size_t)sp * P.n + me;
        const int* row = slow + sm * kSlowCap;
        for (int e = l; e < min(nslow[sm], kSlowCap); e += 32) visit_pair(P, A, g, gT, gE, me, row[e], 1.0, 1.0, acc);
    }
    // Covalent scales: the pair function is linear in (mScale, iScale).
    for (int e = exc_off[me] + l; e < exc_off[me + 1]; e += 32)
        visit_pair(P, A, g, gT, gE, me, exc_j[e], exc_m[e] - 1.0, exc_s[e] - 1.0, acc);
    for (int k = 0; k < 8; k++) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        acc[k] = v;
    }
    if (l == 0)
        for (int k = 0; k < 8; k++) {
            double v = 0.0;
            for (int sp = 0; sp < nsplit; sp++) v += part[8 * ((size_t)sp * P.n + me) + k];
            out[8 * me + k] = v + acc[k];
        }
}

// b = d/d(q, lab, t) of lambda . Efix, per atom (out: n*5).  Field at i due to
// k (RTDF.cpp:698-704): f_ik = -m [d (rr3 q_k - rr5 lab_k.d) + lab_k rr3],
// d = p_k - p_i.
// with_dual = 0: the unit-scale pairs' Thole-factor term is left to
// k_fixed_dual_list (the covalent corrections keep theirs here).
__global__ void k_fixed_vjp(PairParams P, AtomData A, const double* __restrict__ lam, const int* __restrict__ exc_off,
                            const int* __restrict__ exc_j, const double* __restrict__ exc_m, double* __restrict__ out,
                            int with_dual) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = t / kLanes, l = t % kLanes;
    const bool act = k < P.n;
    double acc[5] = {0, 0, 0, 0, 0};
    if (act) {
        for (int i = l; i < P.n; i += kLanes)
            if (i != k) fixed_vjp_visit(P, A, lam, k, i, 1.0, acc, with_dual != 0);
        for (int e = exc_off[k] + l; e < exc_off[k + 1]; e += kLanes)
            fixed_vjp_visit(P, A, lam, k, exc_j[e], exc_m[e] - 1.0, acc);
    }
    for (int c = 0; c < 5; c++) acc[c] = lane_sum(acc[c]);
    if (act && l == 0)
        for (int c = 0; c < 5; c++) out[5 * k + c] = acc[c];
}

// c_t = d/dt_k of lambda^T T(t) mu (RTDF.cpp:766-818), per atom.
__global__ void k_matvec_t_vjp(PairParams P, AtomData A, const double* __restrict__ lam,
                               const int* __restrict__ exc_off, const int* __restrict__ exc_j,
                               const double* __restrict__ exc_s, double* __restrict__ out, int accumulate) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = t / kLanes, l = t % kLanes;
    const bool act = k < P.n;
    double acc = 0.0;
    if (act) {
        for (int j = l; j < P.n; j += kLanes)
            if (j != k) acc += matvec_t_visit(P, A, lam, k, j, 1.0);
        for (int e = exc_off[k] + l; e < exc_off[k + 1]; e += kLanes)
            acc += matvec_t_visit(P, A, lam, k, exc_j[e], exc_s[e] - 1.0);
    }
    acc = lane_sum(acc);
    if (act && l == 0) out[k] = accumulate ? out[k] + acc : acc;
}

// k_fixed_vjp without the Thole-factor term, over shared-memory J tiles, one
// thread per atom: undamped pairs in the arithmetic T (FP32 in the mixed
// form) from an FP64 minimum-image displacement, damped pairs in FP64; the
// covalent corrections (with their Thole term) in FP64 at the end.  The
// J range is split over blockIdx.y as in k_pair_vjp_fast; split s writes
// part + s * n * 5 and k_sum_splits5 adds the splits in order.
template <class T>
__global__ void __launch_bounds__(kVjpTile) k_fixed_vjp_fast(PairParams P, AtomData A, const double* __restrict__ lam,
                                                            const int* __restrict__ exc_off,
                                                            const int* __restrict__ exc_j,
                                                            const double* __restrict__ exc_m,
                                                            double* __restrict__ part) {
    __shared__ double s_pos[3][kVjpTile];
    __shared__ T s_l[3][kVjpTile];
    const int k = blockIdx.x * kVjpTile + threadIdx.x;
    const bool act = k < P.n;
    const int kk = act ? k : 0;
    const double px = A.pos[3 * kk], py = A.pos[3 * kk + 1], pz = A.pos[3 * kk + 2];
    const double damp_r2 = (double)P.damp_r2;
    double acc[5] = {0, 0, 0, 0, 0};
    const int ntile = (P.n + kVjpTile - 1) / kVjpTile;
    const int tb = (int)(((long)ntile * blockIdx.y) / gridDim.y), te = (int)(((long)ntile * (blockIdx.y + 1)) / gridDim.y);
    for (int base = tb * kVjpTile; base < te * kVjpTile && base < P.n; base += kVjpTile) {
        __syncwarp();
        const int js = base + threadIdx.x;
        if (js < P.n)
            for (int c = 0; c < 3; c++) {
                s_pos[c][threadIdx.x] = A.pos[3 * js + c];
                s_l[c][threadIdx.x] = (T)lam[3 * js + c];
            }
        __syncwarp();
        if (!act) continue;
        const int cnt = min(kVjpTile, P.n - base);
        T a0 = 0, a1 = 0, a2 = 0, a3 = 0;
        for (int jj = 0; jj < cnt; jj++) {
            const int i = base + jj;
            if (i == k) continue;
            // d = p_k - p_i
            const V3 d = min_image(P, {px - s_pos[0][jj], py - s_pos[1][jj], pz - s_pos[2][jj]});
            const double r2 = d.x * d.x + d.y * d.y + d.z * d.z;
            if (r2 < damp_r2) {
                fixed_vjp_visit(P, A, lam, k, i, 1.0, acc, false);
                continue;
            }
            const T dx = (T)d.x, dy = (T)d.y, dz = (T)d.z;
            const T ri = div_sqrt(T(1), (T)r2), ri2 = ri * ri, rr3 = ri * ri2, rr5 = T(3) * rr3 * ri2;
            const T lx = s_l[0][jj], ly = s_l[1][jj], lz = s_l[2][jj];
            const T ldd = lx * dx + ly * dy + lz * dz;
            a0 -= rr3 * ldd;
            a1 += rr5 * ldd * dx - rr3 * lx;
            a2 += rr5 * ldd * dy - rr3 * ly;
            a3 += rr5 * ldd * dz - rr3 * lz;
        }
        acc[0] += (double)a0;
        acc[1] += (double)a1;
        acc[2] += (double)a2;
        acc[3] += (double)a3;
    }
    if (!act) return;
    if (blockIdx.y == 0)
        for (int e = exc_off[k]; e < exc_off[k + 1]; e++) fixed_vjp_visit(P, A, lam, k, exc_j[e], exc_m[e] - 1.0, acc);
    double* o = part + 5 * ((size_t)blockIdx.y * P.n + k);
    for (int c = 0; c < 5; c++) o[c] = acc[c];
}

// out[k] = sum over splits s of part[s * m + k], in split order.
__global__ void k_sum_splits(int m, int nsplit, const double* __restrict__ part, double* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    double v = 0.0;
    for (int s = 0; s < nsplit; s++) v += part[(size_t)s * m + k];
    out[k] = v;
}

// Warp-per-atom passes over the damped-partner lists of the pair VJP (the
// same pairs, within the damping range, are the only ones whose Thole factors
// matter).  An atom whose list overflowed its row falls back to a scan of all
// partners.  Lanes take entries l, l + 32, ... in split order; a fixed
// shuffle tree adds them.
__device__ __forceinline__ double warp_sum_fixed(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ bool list_overflow(const AdjPairList& L, int n, int k) {
    for (int sp = 0; sp < L.nsplit; sp++)
        if (L.nslow[(size_t)sp * n + k] > L.cap) return true;
    return false;
}

// out[5 k + 4] += d/dt_k of lambda . Efix over the unit-scale damped pairs.
__global__ void k_fixed_dual_list(PairParams P, AtomData A, const double* __restrict__ lam, AdjPairList L,
                                  double* __restrict__ out) {
    const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, l = threadIdx.x & 31;
    if (k >= P.n) return;   // whole warps leave together
    double acc = 0.0;
    if (list_overflow(L, P.n, k)) {
        for (int i = l; i < P.n; i += 32)
            if (i != k) acc += fixed_vjp_dual(P, A, lam, k, i, 1.0);
    } else {
        for (int sp = 0; sp < L.nsplit; sp++) {
            const size_t sk = (size_t)sp * P.n + k;
            const int* row = L.slow + sk * L.cap;
            for (int e = l; e < L.nslow[sk]; e += 32) acc += fixed_vjp_dual(P, A, lam, k, row[e], 1.0);
        }
    }
    acc = warp_sum_fixed(acc);
    if (l == 0) out[5 * k + 4] += acc;
}

// k_matvec_t_vjp over the damped-partner lists.
__global__ void k_matvec_t_list(PairParams P, AtomData A, const double* __restrict__ lam, AdjPairList L,
                                const int* __restrict__ exc_off, const int* __restrict__ exc_j,
                                const double* __restrict__ exc_s, double* __restrict__ out, int accumulate) {
    const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, l = threadIdx.x & 31;
    if (k >= P.n) return;
    double acc = 0.0;
    if (list_overflow(L, P.n, k)) {
        for (int j = l; j < P.n; j += 32)
            if (j != k) acc += matvec_t_visit(P, A, lam, k, j, 1.0);
    } else {
        for (int sp = 0; sp < L.nsplit; sp++) {
            const size_t sk = (size_t)sp * P.n + k;
            const int* row = L.slow + sk * L.cap;
            for (int e = l; e < L.nslow[sk]; e += 32) acc += matvec_t_visit(P, A, lam, k, row[e], 1.0);
        }
    }
    for (int e = exc_off[k] + l; e < exc_off[k + 1]; e += 32)
        acc += matvec_t_visit(P, A, lam, k, exc_j[e], exc_s[e] - 1.0);
    acc = warp_sum_fixed(acc);
    if (l == 0) out[k] = accumulate ? out[k] + acc : acc;
}

}  // namespace adj

// ---------------------------------------------------------------------------
// Frame part: g_tau = M^T g and the rotation transpose.
// ---------------------------------------------------------------------------
// g_tau_i = sum over the frame roles of atom i of J_role^T g_atom(role), where
// J_role tau = the force the role receives (linear in tau).
__global__ void k_torque_vjp(int n, const double* __restrict__ pos, const int4* __restrict__ axis,
                             const double* __restrict__ g, double* __restrict__ gt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int4 ax = axis[i];
    double out[3] = {0.0, 0.0, 0.0};
    if (ax.x != 5) {
        int atoms[4] = {i, ax.y, ax.z, ax.w};
        for (int role = 0; role < 4; role++) {
            int a = atoms[role];
            if (a < 0) continue;
            if (role == 2 && ax.x == 4) continue;                          // ZOnly: X receives nothing
            if (role == 3 && !(ax.x == 2 || ax.x == 3)) continue;          // W only for ZBisect / ThreeFold
            for (int c = 0; c < 3; c++) {
                d3 e = {c == 0 ? 1.0 : 0.0, c == 1 ? 1.0 : 0.0, c == 2 ? 1.0 : 0.0};
                d3 f = torque_role_force(pos, ax, i, role, e);
                out[c] += f.x * g[3 * a] + f.y * g[3 * a + 1] + f.z * g[3 * a + 2];
            }
        }
    }
    gt[3 * i] = out[0];
    gt[3 * i + 1] = out[1];
    gt[3 * i + 2] = out[2];
}

// dL/dmu_mol_i = S R_i^T dL/dlab_i (rotation of applyRotationMatrixToParticle,
// RTDF.cpp:477-546, lab = sum_j d_j R[j]); S flips y when the chirality check
// flipped the dipole (:432-452).
__global__ void k_rotation_vjp(int n, const double* __restrict__ pos, const int4* __restrict__ axis,
                               const double* __restrict__ glab, double* __restrict__ gmol) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double R[3][3], sy;
    frame_rows(pos, axis[i], i, R, sy);
    for (int j = 0; j < 3; j++) {
        double v = R[j][0] * glab[3 * i] + R[j][1] * glab[3 * i + 1] + R[j][2] * glab[3 * i + 2];
        gmol[3 * i + j] = j == 1 ? sy * v : v;
    }
}

// Assemble per-atom gradients: q, alpha, t, mu_mol (3) = 6 per atom.
__global__ void k_adjoint_assemble(int n, const double* __restrict__ a8, const double* __restrict__ b5,
                                   const double* __restrict__ ct, const double* __restrict__ amu_tlam,
                                   const double* __restrict__ e_tmu, const double* __restrict__ gmol,
                                   double* __restrict__ out, const double* __restrict__ galpha) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[6 * i] = a8[8 * i] + b5[5 * i];
    double ga = 0.0;
    if (galpha) ga = galpha[i];
    else
        for (int c = 0; c < 3; c++) ga += amu_tlam[3 * i + c] * e_tmu[3 * i + c];
    out[6 * i + 1] = ga;
    out[6 * i + 2] = a8[8 * i + 7] + b5[5 * i + 4] + ct[i];
    for (int c = 0; c < 3; c++) out[6 * i + 3 + c] = gmol[3 * i + c];
}

// glab = a_lab + b_lab; a_mu extracted; (rhs + T x) for the alpha gradient.
__global__ void k_adjoint_split(int n, const double* __restrict__ a8, const double* __restrict__ b5,
                                double* __restrict__ amu, double* __restrict__ glab) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int c = 0; c < 3; c++) {
        amu[3 * i + c] = a8[8 * i + 4 + c];
        if (b5) glab[3 * i + c] = a8[8 * i + 1 + c] + b5[5 * i + 1 + c];
    }
}

// out = base + (sum of field partials at slot rank[i]) (e.g. a_mu + T lambda).
__global__ void k_add_field(int n, const int* __restrict__ rank, int nsplit, int n_pad,
                            const double* __restrict__ partial, const double* __restrict__ base,
                            double* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int k = rank[i];
    for (int c = 0; c < 3; c++) {
        double t = 0.0;
        for (int s = 0; s < nsplit; s++) t += partial[((size_t)s * 3 + c) * n_pad + k];
        out[3 * i + c] = base[3 * i + c] + t;
    }
}

// Right-hand side of an adjoint solve: E := rhs, mu := alpha rhs,
// y := sqrt(alpha) rhs, operand := mu (the start of solve_cg).
template <class R>
__global__ void k_rhs_init(int n, const int* __restrict__ rank, const double* __restrict__ rhs,
                           const double* __restrict__ alpha, const double* __restrict__ salpha,
                           const double* __restrict__ thole, double* __restrict__ E, double* __restrict__ mu,
                           double* __restrict__ y, typename Vec4T<R>::type* __restrict__ vec) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int c = 0; c < 3; c++) {
        double v = rhs[3 * i + c];
        E[3 * i + c] = v;
        mu[3 * i + c] = alpha[i] * v;
        y[3 * i + c] = salpha[i] * v;
    }
    typename Vec4T<R>::type v;
    v.x = (R)mu[3 * i];
    v.y = (R)mu[3 * i + 1];
    v.z = (R)mu[3 * i + 2];
    v.w = (R)thole[i];
    vec[rank[i]] = v;
}

// Operand := x (for a plain T x matvec).
template <class R>
__global__ void k_set_operand(int n, const int* __restrict__ rank, const double* __restrict__ x,
                              const double* __restrict__ thole, typename Vec4T<R>::type* __restrict__ vec) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    typename Vec4T<R>::type v;
    v.x = (R)x[3 * i];
    v.y = (R)x[3 * i + 1];
    v.z = (R)x[3 * i + 2];
    v.w = (R)thole[i];
    vec[rank[i]] = v;
}

// ---------------------------------------------------------------------------
// Launchers.
// ---------------------------------------------------------------------------
static inline int nb(int n) { return (n + 127) / 128; }

// Scratch of the two-pass pair VJP, per (split, atom): 8 FP64 sums, the
// slow-pair row and its count.
// Splits of the J range of the tiled passes: about 16 warps per SM (148 SMs)
// in total, at most kVjpSplit.
static int vjp_splits(int n) {
    const int blocks = (std::max(n, 1) + adj::kVjpTile - 1) / adj::kVjpTile;
    return std::min(adj::kVjpSplit, std::max(1, (16 * 148 + blocks - 1) / blocks));
}

size_t adjoint_pair_scratch(int n) {
    const size_t m = (size_t)vjp_splits(n) * (size_t)std::max(n, 1);
    return 8 * m + (m * (adj::kSlowCap + 1) * sizeof(int) + sizeof(double) - 1) / sizeof(double);
}

size_t adjoint_fixed_scratch(int n) { return 5 * (size_t)vjp_splits(n) * (size_t)std::max(n, 1); }

void launch_adjoint_pair(const Dev& d, const double* g, const double* gT, double gE, double* a8, int precision,
                         double* scratch, AdjPairList* list, cudaStream_t st) {
    if (list) *list = AdjPairList{};
    if (d.n <= 0) return;
    adj::AtomData A{d.pos, d.charge, d.lab, d.mu, d.thole, d.yz};
    if (d.pp.rinv4_power != 0.0f || d.pp.rinv4_fill != 0.0f) {
        adj::k_pair_vjp<<<nb(d.n * adj::kLanes), 128, 0, st>>>(d.pp, A, g, gT, gE, d.exc_off, d.exc_j, d.exc_m,
                                                                d.exc_s, a8);
        return;
    }
    const int blocks = (d.n + adj::kVjpTile - 1) / adj::kVjpTile;
    const int nsplit = vjp_splits(d.n);
    const size_t m = (size_t)nsplit * d.n;
    double* part = scratch;
    int* slow = reinterpret_cast<int*>(scratch + 8 * m);
    int* nslow = slow + m * adj::kSlowCap;
    const dim3 grid(blocks, nsplit);
    if (precision == TDP_PRECISION_MIXED)
        adj::k_pair_vjp_fast<float><<<grid, adj::kVjpTile, 0, st>>>(d.pp, A, g, gT, gE, slow, nslow, part);
    else
        adj::k_pair_vjp_fast<double><<<grid, adj::kVjpTile, 0, st>>>(d.pp, A, g, gT, gE, slow, nslow, part);
    adj::k_pair_vjp_slow<<<nb(32 * d.n), 128, 0, st>>>(d.pp, A, g, gT, gE, nsplit, slow, nslow, part, d.exc_off,
                                                        d.exc_j, d.exc_m, d.exc_s, a8);
    if (list) *list = AdjPairList{nsplit, adj::kSlowCap, slow, nslow};
}
void launch_adjoint_fixed(const Dev& d, const double* lam, double* b5, const AdjPairList& list, int precision,
                          double* scratch, cudaStream_t st) {
    if (d.n <= 0) return;
    adj::AtomData A{d.pos, d.charge, d.lab, d.mu, d.thole, d.yz};
    if (list.nsplit <= 0 || !scratch) {
        adj::k_fixed_vjp<<<nb(d.n * adj::kLanes), 128, 0, st>>>(d.pp, A, lam, d.exc_off, d.exc_j, d.exc_m, b5, 1);
        return;
    }
    const int blocks = (d.n + adj::kVjpTile - 1) / adj::kVjpTile;
    const int nsplit = vjp_splits(d.n);
    const dim3 grid(blocks, nsplit);
    if (precision == TDP_PRECISION_MIXED)
        adj::k_fixed_vjp_fast<float><<<grid, adj::kVjpTile, 0, st>>>(d.pp, A, lam, d.exc_off, d.exc_j, d.exc_m, scratch);
    else
        adj::k_fixed_vjp_fast<double><<<grid, adj::kVjpTile, 0, st>>>(d.pp, A, lam, d.exc_off, d.exc_j, d.exc_m, scratch);
    adj::k_sum_splits<<<nb(5 * d.n), 128, 0, st>>>(5 * d.n, nsplit, scratch, b5);
    adj::k_fixed_dual_list<<<nb(32 * d.n), 128, 0, st>>>(d.pp, A, lam, list, b5);
}
void launch_adjoint_matvec_t(const Dev& d, const double* lam, double* ct, const AdjPairList& list, cudaStream_t st) {
    launch_adjoint_matvec_t_mu(d, lam, d.mu, ct, false, list, st);
}
void launch_adjoint_matvec_t_mu(const Dev& d, const double* lam, const double* mu, double* ct, bool accumulate,
                                const AdjPairList& list, cudaStream_t st) {
    if (d.n <= 0) return;
    adj::AtomData A{d.pos, d.charge, d.lab, mu, d.thole, d.yz};
    if (list.nsplit > 0)
        adj::k_matvec_t_list<<<nb(32 * d.n), 128, 0, st>>>(d.pp, A, lam, list, d.exc_off, d.exc_j, d.exc_s, ct,
                                                            accumulate ? 1 : 0);
    else
        adj::k_matvec_t_vjp<<<nb(d.n * adj::kLanes), 128, 0, st>>>(d.pp, A, lam, d.exc_off, d.exc_j, d.exc_s, ct,
                                                                    accumulate ? 1 : 0);
}

__global__ void k_lincomb(int n3, double ca, const double* __restrict__ a, double cb, const double* __restrict__ b,
                          double* __restrict__ out) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n3) out[k] = ca * a[k] + (b ? cb * b[k] : 0.0);
}
__global__ void k_dot3_acc(int n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ acc) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) acc[i] += a[3 * i] * b[3 * i] + a[3 * i + 1] * b[3 * i + 1] + a[3 * i + 2] * b[3 * i + 2];
}
__global__ void k_alpha_mul(int n, const double* __restrict__ alpha, const double* __restrict__ v,
                            double* __restrict__ out) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < 3 * n) out[k] = alpha[k / 3] * v[k];
}
void launch_lincomb(int n, double ca, const double* a, double cb, const double* b, double* out, cudaStream_t st) {
    k_lincomb<<<nb(3 * n), 128, 0, st>>>(3 * n, ca, a, cb, b, out);
}
void launch_dot3_acc(int n, const double* a, const double* b, double* acc, cudaStream_t st) {
    k_dot3_acc<<<nb(n), 128, 0, st>>>(n, a, b, acc);
}
void launch_alpha_scale(const Dev& d, const double* v, double* out, cudaStream_t st) {
    k_alpha_mul<<<nb(3 * d.n), 128, 0, st>>>(d.n, d.alpha, v, out);
}
void launch_torque_vjp(const Dev& d, const double* g, double* gt, cudaStream_t st) {
    k_torque_vjp<<<nb(d.n), 128, 0, st>>>(d.n, d.pos, d.axis, g, gt);
}
void launch_rotation_vjp(const Dev& d, const double* glab, double* gmol, cudaStream_t st) {
    k_rotation_vjp<<<nb(d.n), 128, 0, st>>>(d.n, d.pos, d.axis, glab, gmol);
}
void launch_adjoint_split(const Dev& d, const double* a8, const double* b5, double* amu, double* glab,
                          cudaStream_t st) {
    k_adjoint_split<<<nb(d.n), 128, 0, st>>>(d.n, a8, b5, amu, glab);
}
void launch_add_field(const Dev& d, const double* base, double* out, cudaStream_t st) {
    k_add_field<<<nb(d.n), 128, 0, st>>>(d.n, d.rank, d.nsplit, d.n_pad, d.partial, base, out);
}
template <class R>
void launch_rhs_init(const Dev& d, const double* rhs, cudaStream_t st) {
    k_rhs_init<R><<<nb(d.n), 128, 0, st>>>(d.n, d.rank, rhs, d.alpha, d.salpha, d.thole, d.E, d.mu, d.y,
                                           (typename Vec4T<R>::type*)d.vec_s);
}
template <class R>
void launch_set_operand(const Dev& d, const double* x, cudaStream_t st) {
    k_set_operand<R><<<nb(d.n), 128, 0, st>>>(d.n, d.rank, x, d.thole, (typename Vec4T<R>::type*)d.vec_s);
}
template void launch_rhs_init<float>(const Dev&, const double*, cudaStream_t);
template void launch_rhs_init<double>(const Dev&, const double*, cudaStream_t);
template void launch_set_operand<float>(const Dev&, const double*, cudaStream_t);
template void launch_set_operand<double>(const Dev&, const double*, cudaStream_t);
void launch_adjoint_assemble(const Dev& d, const double* a8, const double* b5, const double* ct,
                             const double* amu_tlam, const double* e_tmu, const double* gmol, double* out,
                             cudaStream_t st, const double* galpha) {
    k_adjoint_assemble<<<nb(d.n), 128, 0, st>>>(d.n, a8, b5, ct, amu_tlam, e_tmu, gmol, out, galpha);
}

}  // namespace tdp
