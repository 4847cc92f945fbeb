// tdp_kernels.cu -- sm_100a kernels of the TholeDipoleForce hot path in the
// reference's semantics (aehogan/tholedipoleplugin,
// platforms/reference/src/ReferenceTholeDipoleForce.cpp, "RTDF.cpp"): packing
// of the tile records, lab-frame rotation, the O(N) kernels of the solvers,
// the torque gather and the queries.  The all-pairs kernels (permanent field,
// mutual-field matvec, energy/force/torque) are in tdp_sym.cu; they leave
// per-band partial sums that the consumers here reduce in a fixed order.
//
// Mixed form: positions are FP32 offsets from FP64 32-atom tile centres, so
// near pairs keep full FP32 precision wherever they are in the box.
#include "tdp_frames.cuh"
#include "tdp_kernels.cuh"
#include "tdp_pairs.cuh"

#include <math.h>

namespace tdp {

// ---------------------------------------------------------------------------
// Packing: tile centres/extents and per-atom position records.
// ---------------------------------------------------------------------------
template <class R>
__global__ void k_pack(int n, int n_tiles_pad, const double* __restrict__ pos, const double* __restrict__ charge,
                       double4* __restrict__ tctr, double4* __restrict__ text,
                       typename Vec4T<R>::type* __restrict__ posq, double2* __restrict__ yz) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (warp >= n_tiles_pad) return;
    int i = warp * kTile + lane;
    bool valid = i < n;
    double x = valid ? pos[3 * i] : 0.0, y = valid ? pos[3 * i + 1] : 0.0, z = valid ? pos[3 * i + 2] : 0.0;
    int cnt = __popc(__ballot_sync(0xffffffffu, valid));
    double cx = warp_sum(x), cy = warp_sum(y), cz = warp_sum(z);
    if (cnt > 0) {
        cx /= cnt;
        cy /= cnt;
        cz /= cnt;
    }
    double ex = valid ? fabs(x - cx) : 0.0, ey = valid ? fabs(y - cy) : 0.0, ez = valid ? fabs(z - cz) : 0.0;
    ex = warp_max(ex);
    ey = warp_max(ey);
    ez = warp_max(ez);
    if (lane == 0) {
        tctr[warp] = make_double4(cx, cy, cz, 0.0);
        text[warp] = make_double4(ex, ey, ez, 0.0);
    }
    double q = valid ? charge[i] : 0.0;
    typename Vec4T<R>::type p;
    if (sizeof(R) == 4) {
        p.x = (R)(valid ? x - cx : 0.0);
        p.y = (R)(valid ? y - cy : 0.0);
        p.z = (R)(valid ? z - cz : 0.0);
    } else {
        p.x = (R)(valid ? x : cx);
        p.y = (R)(valid ? y : cy);
        p.z = (R)(valid ? z : cz);
    }
    p.w = (R)q;
    posq[i] = p;
    yz[i] = make_double2(y, z);
}

// Same records in the spatially sorted order of the field kernels: slot k
// holds atom order[k]; also the FP64 positions by slot.
template <class R>
__global__ void k_pack_sorted(int n_tiles_pad, const int* __restrict__ order, const double* __restrict__ pos,
                              const double* __restrict__ charge, double4* __restrict__ tctr,
                              double4* __restrict__ text, typename Vec4T<R>::type* __restrict__ posq,
                              double* __restrict__ pos_s) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (warp >= n_tiles_pad) return;
    int k = warp * kTile + lane;
    int i = order[k];
    bool valid = i >= 0;
    double x = valid ? pos[3 * i] : 0.0, y = valid ? pos[3 * i + 1] : 0.0, z = valid ? pos[3 * i + 2] : 0.0;
    int cnt = __popc(__ballot_sync(0xffffffffu, valid));
    double cx = warp_sum(x), cy = warp_sum(y), cz = warp_sum(z);
    if (cnt > 0) {
        cx /= cnt;
        cy /= cnt;
        cz /= cnt;
    }
    double ex = valid ? fabs(x - cx) : 0.0, ey = valid ? fabs(y - cy) : 0.0, ez = valid ? fabs(z - cz) : 0.0;
    ex = warp_max(ex);
    ey = warp_max(ey);
    ez = warp_max(ez);
    if (lane == 0) {
        tctr[warp] = make_double4(cx, cy, cz, 0.0);
        text[warp] = make_double4(ex, ey, ez, 0.0);
    }
    typename Vec4T<R>::type p;
    if (sizeof(R) == 4) {
        p.x = (R)(valid ? x - cx : 0.0);
        p.y = (R)(valid ? y - cy : 0.0);
        p.z = (R)(valid ? z - cz : 0.0);
    } else {
        p.x = (R)(valid ? x : cx);
        p.y = (R)(valid ? y : cy);
        p.z = (R)(valid ? z : cz);
    }
    p.w = (R)(valid ? charge[i] : 0.0);
    posq[k] = p;
    pos_s[3 * k] = valid ? x : cx;
    pos_s[3 * k + 1] = valid ? y : cy;
    pos_s[3 * k + 2] = valid ? z : cz;
}

// ---------------------------------------------------------------------------
// Local -> lab frame of the permanent dipoles: checkChiral (RTDF.cpp:432-467)
// then applyRotationMatrixToParticle (RTDF.cpp:477-571), FP64.
// ---------------------------------------------------------------------------
template <class R>
__global__ void k_rotate(int n, const double* __restrict__ pos, const double* __restrict__ dip_mol,
                         const int4* __restrict__ axis, const double* __restrict__ thole, double* __restrict__ lab,
                         typename Vec4T<R>::type* __restrict__ dipt, const int* __restrict__ rank,
                         typename Vec4T<R>::type* __restrict__ dipt_s) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double Rm[3][3], sy;
    frame_rows(pos, axis[i], i, Rm, sy);
    double d0 = dip_mol[3 * i], d1 = sy * dip_mol[3 * i + 1], d2 = dip_mol[3 * i + 2];
    d3 d;
    d.x = 0.0 + d0 * Rm[0][0] + d1 * Rm[1][0] + d2 * Rm[2][0];
    d.y = 0.0 + d0 * Rm[0][1] + d1 * Rm[1][1] + d2 * Rm[2][1];
    d.z = 0.0 + d0 * Rm[0][2] + d1 * Rm[1][2] + d2 * Rm[2][2];
    lab[3 * i] = d.x;
    lab[3 * i + 1] = d.y;
    lab[3 * i + 2] = d.z;
    typename Vec4T<R>::type v;
    v.x = (R)d.x;
    v.y = (R)d.y;
    v.z = (R)d.z;
    v.w = (R)thole[i];
    dipt[i] = v;
    dipt_s[rank[i]] = v;
}

// forces_out = pair forces + torque-mapped forces (FP64, deterministic).
__global__ void k_torque_gather(int n, const double* __restrict__ pos, const int4* __restrict__ axis,
                                const double* __restrict__ torque, const int* __restrict__ users_off,
                                const int2* __restrict__ users, const double* __restrict__ fpair,
                                double* __restrict__ fout) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    d3 f = ld3(fpair + 3 * a);
    for (int k = users_off[a]; k < users_off[a + 1]; k++) {
        int2 u = users[k];  // (frame atom i, role)
        d3 T = ld3(torque + 3 * u.x);
        f = f + torque_role_force(pos, axis[u.x], u.x, u.y, T);
    }
    fout[3 * a] = f.x;
    fout[3 * a + 1] = f.y;
    fout[3 * a + 2] = f.z;
}

// ---------------------------------------------------------------------------
// O(N) vector kernels of the solvers (FP64 vectors, deterministic reductions).
// ---------------------------------------------------------------------------
// Sum of the j-split partials of the field kernels for slot k.
__device__ __forceinline__ d3 sum_partial3(const double* __restrict__ partial, int nsplit, int n_pad, int i) {
    d3 t = {0.0, 0.0, 0.0};
    for (int s = 0; s < nsplit; s++) {
        size_t b = (size_t)s * 3 * n_pad;
        t.x += partial[b + i];
        t.y += partial[b + n_pad + i];
        t.z += partial[b + 2 * (size_t)n_pad + i];
    }
    return t;
}

template <class R>
__device__ __forceinline__ void store_vec(typename Vec4T<R>::type* v, int i, d3 a, double t) {
    typename Vec4T<R>::type o;
    o.x = (R)a.x;
    o.y = (R)a.y;
    o.z = (R)a.z;
    o.w = (R)t;
    v[i] = o;
}

// E = sum of permanent-field partials; mu = alpha*E (RTDF.cpp:743-746);
// packs mu as the next matvec operand; CG start y = sqrt(alpha)*E.
template <class R>
__global__ void k_fixed_done(int n, const int* __restrict__ rank, int nsplit, int n_pad, const double* __restrict__ partial,
                             const double* __restrict__ alpha, const double* __restrict__ salpha,
                             const double* __restrict__ thole, double* __restrict__ E, double* __restrict__ mu,
                             double* __restrict__ y, typename Vec4T<R>::type* __restrict__ vec) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    d3 e = sum_partial3(partial, nsplit, n_pad, rank[i]);
    E[3 * i] = e.x;
    E[3 * i + 1] = e.y;
    E[3 * i + 2] = e.z;
    d3 m = e * alpha[i];
    mu[3 * i] = m.x;
    mu[3 * i + 1] = m.y;
    mu[3 * i + 2] = m.z;
    d3 yy = e * salpha[i];
    y[3 * i] = yy.x;
    y[3 * i + 1] = yy.y;
    y[3 * i + 2] = yy.z;
    store_vec<R>(vec, rank[i], m, thole[i]);
}

// Warm start: y = mu / sqrt(alpha) (0 where alpha = 0); packs mu.
template <class R>
__global__ void k_warm_start(int n, const int* __restrict__ rank, const double* __restrict__ salpha, const double* __restrict__ thole,
                             const double* __restrict__ mu, double* __restrict__ y,
                             typename Vec4T<R>::type* __restrict__ vec) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    d3 m = ld3(mu + 3 * i);
    double s = salpha[i];
    d3 yy = s > 0.0 ? m * (1.0 / s) : d3{0.0, 0.0, 0.0};
    y[3 * i] = yy.x;
    y[3 * i + 1] = yy.y;
    y[3 * i + 2] = yy.z;
    store_vec<R>(vec, rank[i], m, thole[i]);
}

// Starting point extrapolated from the last two solutions: mu = 2 mu1 - mu2.
__global__ void k_predict(size_t n3, int nh, const double* __restrict__ h0, const double* __restrict__ h1,
                          const double* __restrict__ h2, const double* __restrict__ h3, double c0, double c1,
                          double c2, double c3, double* __restrict__ mu) {
    const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (k >= n3) return;
    double v = c0 * h0[k];
    if (nh > 1) v += c1 * h1[k];
    if (nh > 2) v += c2 * h2[k];
    if (nh > 3) v += c3 * h3[k];
    mu[k] = v;
}

// Start of a fused warm start: the operand records carry m + mu0 (mu0 in mu),
// so one permanent-field walk gives E + T mu0 for unit-scale pairs.
template <class R>
__global__ void k_pack_total(int n, const int* __restrict__ rank, const double* __restrict__ lab,
                             const double* __restrict__ mu, const double* __restrict__ thole,
                             typename Vec4T<R>::type* __restrict__ vec) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    store_vec<R>(vec, rank[i], ld3(lab + 3 * i) + ld3(mu + 3 * i), thole[i]);
}

// E := E_fixed + T mu0 (the fused walk's partial sums); y = mu0 / sqrt(alpha).
__global__ void k_fused_done(int n, const int* __restrict__ rank, int nsplit, int n_pad,
                             const double* __restrict__ partial, const double* __restrict__ salpha,
                             const double* __restrict__ mu, double* __restrict__ E, double* __restrict__ y) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    d3 e = sum_partial3(partial, nsplit, n_pad, rank[i]);
    E[3 * i] = e.x;
    E[3 * i + 1] = e.y;
    E[3 * i + 2] = e.z;
    d3 m = ld3(mu + 3 * i);
    double s = salpha[i];
    d3 yy = s > 0.0 ? m * (1.0 / s) : d3{0.0, 0.0, 0.0};
    y[3 * i] = yy.x;
    y[3 * i + 1] = yy.y;
    y[3 * i + 2] = yy.z;
}

// True residual in y-space: r = sqrt(alpha)*(E + T mu) - y, with mu = sqrt(alpha)*y.
// p = r, packs sqrt(alpha)*p; block partials of r.r and sum alpha|r|^2.
// use_partial = 0: the field term is already included in E.
template <class R>
__global__ void k_cg_residual(int n, const int* __restrict__ rank, int nsplit, int n_pad, const double* __restrict__ partial,
                              const double* __restrict__ E, const double* __restrict__ salpha,
                              const double* __restrict__ thole, const double* __restrict__ y, double* __restrict__ r,
                              double* __restrict__ p, typename Vec4T<R>::type* __restrict__ vec,
                              double* __restrict__ rr_part, double* __restrict__ eps_part, int use_partial) {
    __shared__ double red[40];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double rr = 0.0, ee = 0.0;
    if (i < n) {
        d3 t = use_partial ? sum_partial3(partial, nsplit, n_pad, rank[i]) : d3{0.0, 0.0, 0.0};
        double s = salpha[i];
        d3 rv = (ld3(E + 3 * i) + t) * s - ld3(y + 3 * i);
        r[3 * i] = rv.x;
        r[3 * i + 1] = rv.y;
        r[3 * i + 2] = rv.z;
        p[3 * i] = rv.x;
        p[3 * i + 1] = rv.y;
        p[3 * i + 2] = rv.z;
        store_vec<R>(vec, rank[i], rv * s, thole[i]);
        rr = dot(rv, rv);
        ee = s * s * rr;
    }
    rr = block_sum(rr, red);
    ee = block_sum(ee, red);
    if (threadIdx.x == 0) {
        rr_part[blockIdx.x] = rr;
        eps_part[blockIdx.x] = ee;
    }
}

// q = p - sqrt(alpha) * (T sqrt(alpha) p); block partials of p.q.
__global__ void k_cg_q(int n, const int* __restrict__ rank, int nsplit, int n_pad, const double* __restrict__ partial,
                       const double* __restrict__ salpha, const double* __restrict__ p, double* __restrict__ q,
                       double* __restrict__ pq_part) {
    __shared__ double red[40];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double pq = 0.0;
    if (i < n) {
        d3 t = sum_partial3(partial, nsplit, n_pad, rank[i]);
        d3 pv = ld3(p + 3 * i);
        d3 qv = pv - t * salpha[i];
        q[3 * i] = qv.x;
        q[3 * i + 1] = qv.y;
        q[3 * i + 2] = qv.z;
        pq = dot(pv, qv);
    }
    pq = block_sum(pq, red);
    if (threadIdx.x == 0) pq_part[blockIdx.x] = pq;
}

// a = rr/pq; y += a p; r -= a q; block partials of r.r and sum alpha|r|^2.
// scal_a (may be NULL) keeps a for the flexible beta of a preconditioned solve.
__global__ void k_cg_update(int n, int nblk, const double* __restrict__ scal_rr, int slot,
                            const double* __restrict__ pq_part, const double* __restrict__ salpha,
                            const double* __restrict__ p, const double* __restrict__ q, double* __restrict__ y,
                            double* __restrict__ r, double* __restrict__ rr_part, double* __restrict__ eps_part,
                            double* __restrict__ scal_a) {
    __shared__ double red[40];
    double pq = sum_partials(pq_part, nblk, red);
    double a = scal_rr[slot] / pq;
    if (scal_a && blockIdx.x == 0 && threadIdx.x == 0) scal_a[slot] = a;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double rr = 0.0, ee = 0.0;
    if (i < n) {
        d3 yv = ld3(y + 3 * i) + ld3(p + 3 * i) * a;
        d3 rv = ld3(r + 3 * i) - ld3(q + 3 * i) * a;
        y[3 * i] = yv.x;
        y[3 * i + 1] = yv.y;
        y[3 * i + 2] = yv.z;
        r[3 * i] = rv.x;
        r[3 * i + 1] = rv.y;
        r[3 * i + 2] = rv.z;
        double s = salpha[i];
        rr = dot(rv, rv);
        ee = s * s * rr;
    }
    rr = block_sum(rr, red);
    ee = block_sum(ee, red);
    if (threadIdx.x == 0) {
        rr_part[blockIdx.x] = rr;
        eps_part[blockIdx.x] = ee;
    }
}

// rr' = sum(rr_part) -> scal_rr[slot]; eps -> scal_eps[slot].  With prev >= 0
// also p = r + (rr'/scal_rr[prev]) p and packs sqrt(alpha)*p for the next
// matvec.
template <class R>
__global__ void k_cg_p(int n, const int* __restrict__ rank, int nblk, int prev, int slot, double* __restrict__ scal_rr,
                       double* __restrict__ scal_eps, const double* __restrict__ rr_part,
                       const double* __restrict__ eps_part, const double* __restrict__ salpha,
                       const double* __restrict__ thole, const double* __restrict__ r, double* __restrict__ p,
                       typename Vec4T<R>::type* __restrict__ vec) {
    __shared__ double red[40];
    double rr = sum_partials(rr_part, nblk, red);
    double ee = sum_partials(eps_part, nblk, red);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        scal_rr[slot] = rr;
        scal_eps[slot] = sqrt(ee / (double)n);
    }
    if (prev < 0) return;
    double beta = rr / scal_rr[prev];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        d3 pv = ld3(r + 3 * i) + ld3(p + 3 * i) * beta;
        p[3 * i] = pv.x;
        p[3 * i + 1] = pv.y;
        p[3 * i + 2] = pv.z;
        store_vec<R>(vec, rank[i], pv * salpha[i], thole[i]);
    }
}

// mu = sqrt(alpha) y; packs mu (mu - mu0 when mu0 is given).
template <class R>
__global__ void k_cg_mu(int n, const int* __restrict__ rank, const double* __restrict__ salpha, const double* __restrict__ thole,
                        const double* __restrict__ y, double* __restrict__ mu,
                        typename Vec4T<R>::type* __restrict__ vec, const double* __restrict__ mu0) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    d3 m = ld3(y + 3 * i) * salpha[i];
    mu[3 * i] = m.x;
    mu[3 * i + 1] = m.y;
    mu[3 * i + 2] = m.z;
    store_vec<R>(vec, rank[i], mu0 ? m - ld3(mu0 + 3 * i) : m, thole[i]);
}

// One Jacobi sweep of convergeInducedDipolesByDIIS (RTDF.cpp:838-846):
// mu' = alpha (E + T mu); block partials of |mu' - mu|^2; packs mu'.
template <class R>
__global__ void k_jacobi(int n, const int* __restrict__ rank, int nsplit, int n_pad, const double* __restrict__ partial,
                         const double* __restrict__ E, const double* __restrict__ alpha,
                         const double* __restrict__ thole, double* __restrict__ mu,
                         typename Vec4T<R>::type* __restrict__ vec, double* __restrict__ eps_part) {
    __shared__ double red[40];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double ee = 0.0;
    if (i < n) {
        d3 t = sum_partial3(partial, nsplit, n_pad, rank[i]);
        d3 nw = (ld3(E + 3 * i) + t) * alpha[i];
        d3 dl = nw - ld3(mu + 3 * i);
        ee = dot(dl, dl);
        mu[3 * i] = nw.x;
        mu[3 * i + 1] = nw.y;
        mu[3 * i + 2] = nw.z;
        store_vec<R>(vec, rank[i], nw, thole[i]);
    }
    ee = block_sum(ee, red);
    if (threadIdx.x == 0) eps_part[blockIdx.x] = ee;
}

// Extrapolation (RTDF.cpp:876-887): mu = alpha (E + T mu), stored as order k.
template <class R>
__global__ void k_extrap_step(int n, const int* __restrict__ rank, int nsplit, int n_pad, const double* __restrict__ partial,
                              const double* __restrict__ E, const double* __restrict__ alpha,
                              const double* __restrict__ thole, double* __restrict__ mu, double* __restrict__ hist_k,
                              typename Vec4T<R>::type* __restrict__ vec) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    d3 t = sum_partial3(partial, nsplit, n_pad, rank[i]);
    d3 nw = (ld3(E + 3 * i) + t) * alpha[i];
    mu[3 * i] = nw.x;
    mu[3 * i + 1] = nw.y;
    mu[3 * i + 2] = nw.z;
    hist_k[3 * i] = nw.x;
    hist_k[3 * i + 1] = nw.y;
    hist_k[3 * i + 2] = nw.z;
    store_vec<R>(vec, rank[i], nw, thole[i]);
}

// mu = sum_k c_k mu_k (RTDF.cpp:890-895); packs mu.
template <class R>
__global__ void k_extrap_combine(int n, const int* __restrict__ rank, int korder, const double* __restrict__ coef, const double* __restrict__ hist,
                                 const double* __restrict__ thole, double* __restrict__ mu,
                                 typename Vec4T<R>::type* __restrict__ vec) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    d3 m = {0.0, 0.0, 0.0};
    for (int k = 0; k < korder; k++) m = m + ld3(hist + (size_t)k * 3 * n + 3 * i) * coef[k];
    mu[3 * i] = m.x;
    mu[3 * i + 1] = m.y;
    mu[3 * i + 2] = m.z;
    store_vec<R>(vec, rank[i], m, thole[i]);
}

// Block partials of |alpha (E + T mu) - mu|^2 (RTDF.cpp:898-906).
__global__ void k_step_eps(int n, const int* __restrict__ rank, int nsplit, int n_pad, const double* __restrict__ partial,
                           const double* __restrict__ E, const double* __restrict__ alpha,
                           const double* __restrict__ mu, double* __restrict__ eps_part) {
    __shared__ double red[40];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double ee = 0.0;
    if (i < n) {
        d3 t = sum_partial3(partial, nsplit, n_pad, rank[i]);
        d3 dl = (ld3(E + 3 * i) + t) * alpha[i] - ld3(mu + 3 * i);
        ee = dot(dl, dl);
    }
    ee = block_sum(ee, red);
    if (threadIdx.x == 0) eps_part[blockIdx.x] = ee;
}

// scal[slot] = sqrt(sum(eps_part)/n).
__global__ void k_eps_scalar(int n, int nblk, const double* __restrict__ eps_part, double* __restrict__ scal,
                             int slot) {
    __shared__ double red[40];
    double ee = sum_partials(eps_part, nblk, red);
    if (threadIdx.x == 0) scal[slot] = sqrt(ee / (double)n);
}

// Induced dipoles packed for the energy kernel.
template <class R>
__global__ void k_pack_ind(int n, const double* __restrict__ mu, typename Vec4T<R>::type* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    store_vec<R>(out, i, ld3(mu + 3 * i), 0.0);
}

// Pair forces/torques and the total energy from the energy-kernel partials.
__global__ void k_energy_done(int n, int nsplit, int n_pad, int n_eblk, const double* __restrict__ partial,
                              const double* __restrict__ energy_partial, double* __restrict__ fpair,
                              double* __restrict__ torque, double* __restrict__ energy_out) {
    __shared__ double red[40];
    if (blockIdx.x == 0) {
        double e = sum_partials(energy_partial, n_eblk, red);
        if (threadIdx.x == 0) *energy_out = e;
    }
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double f[6] = {0, 0, 0, 0, 0, 0};
    for (int s = 0; s < nsplit; s++) {
        size_t b = (size_t)s * 6 * n_pad;
        for (int c = 0; c < 6; c++) f[c] += partial[b + (size_t)c * n_pad + i];
    }
    fpair[3 * i] = f[0];
    fpair[3 * i + 1] = f[1];
    fpair[3 * i + 2] = f[2];
    torque[3 * i] = f[3];
    torque[3 * i + 1] = f[4];
    torque[3 * i + 2] = f[5];
}

// accum += forces (device accumulator of either element type).
__global__ void k_add_forces(int n3, const double* __restrict__ f, double* __restrict__ acc64,
                             float* __restrict__ acc32) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n3) return;
    if (acc64) acc64[k] += f[k];
    else acc32[k] += (float)f[k];
}

// Positions of either element type into the FP64 working copy.
__global__ void k_positions_in(int n3, const void* __restrict__ src, int is_f32, double* __restrict__ dst) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n3) return;
    dst[k] = is_f32 ? (double)((const float*)src)[k] : ((const double*)src)[k];
}

// OpenMM CUDA-platform coordinates: slot k of posq (float4 or double4, x y z q)
// holds atom atom_index[k].
__global__ void k_posq_in(int n, const void* __restrict__ posq, int is_double, const int* __restrict__ atom_index,
                          double* __restrict__ dst) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int a = atom_index[k];
    if (a < 0 || a >= n) return;
    double x, y, z;
    if (is_double) {
        const double4 p = ((const double4*)posq)[k];
        x = p.x;
        y = p.y;
        z = p.z;
    } else {
        const float4 p = ((const float4*)posq)[k];
        x = p.x;
        y = p.y;
        z = p.z;
    }
    dst[3 * a] = x;
    dst[3 * a + 1] = y;
    dst[3 * a + 2] = z;
}

// Forces added to OpenMM's 64-bit fixed-point accumulator (2^32 units per
// force unit, component c of slot k at k + c * padded, truncated toward zero
// as the platform converts).
__global__ void k_forces_out_fixed(int n, const double* __restrict__ f, const int* __restrict__ atom_index,
                                   int padded, unsigned long long* __restrict__ acc) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int a = atom_index[k];
    if (a < 0 || a >= n) return;
    for (int c = 0; c < 3; c++)
        acc[k + (size_t)c * padded] += (unsigned long long)__double2ll_rz(f[3 * a + c] * 4294967296.0);
}

// Electrostatic potential at grid points, calculateElectrostaticPotential-
// ForParticleGridPoint (RTDF.cpp:1348-1372), FP64.
__global__ void k_potential(int n, int ng, PairParams P, const double* __restrict__ pos,
                            const double* __restrict__ charge, const double* __restrict__ lab,
                            const double* __restrict__ mu, const double* __restrict__ grid, double* __restrict__ out) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ng) return;
    d3 gp = ld3(grid + 3 * g);
    double pot = 0.0;
    for (int i = 0; i < n; i++) {
        d3 dr = ld3(pos + 3 * i) - gp;
        if (P.periodic) {
            dr.x = fold_d(dr.x, P.box[0], P.inv_box[0]);
            dr.y = fold_d(dr.y, P.box[1], P.inv_box[1]);
            dr.z = fold_d(dr.z, P.box[2], P.inv_box[2]);
        }
        double r = sqrt(dot(dr, dr));
        double rr1 = 1.0 / r, rr2 = rr1 * rr1, rr3 = rr1 * rr2;
        double p = charge[i] * rr1;
        double scd = dot(ld3(lab + 3 * i), dr);
        double scu = dot(ld3(mu + 3 * i), dr);
        p -= (scd + scu) * rr3;
        pot += p;
    }
    out[g] = pot;
}

// Block partial sums for the system multipole moments
// (RTDF.cpp:1243-1283): 0 mass, 1-3 mass-weighted position.
__global__ void k_com_partials(int n, const double* __restrict__ pos, const double* __restrict__ mass,
                               double* __restrict__ part) {
    __shared__ double red[40];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[4] = {0, 0, 0, 0};
    if (i < n) {
        double m = mass[i];
        v[0] = m;
        v[1] = pos[3 * i] * m;
        v[2] = pos[3 * i + 1] * m;
        v[3] = pos[3 * i + 2] * m;
    }
    for (int c = 0; c < 4; c++) {
        double s = block_sum(v[c], red);
        if (threadIdx.x == 0) part[(size_t)c * gridDim.x + blockIdx.x] = s;
    }
}

// 0 netchg, 1-3 dpl, 4 xx, 5 xy, 6 xz, 7 yy, 8 yz, 9 zz.
__global__ void k_moment_partials(int n, int ncomblk, const double* __restrict__ com_part,
                                  const double* __restrict__ pos, const double* __restrict__ charge,
                                  const double* __restrict__ lab, const double* __restrict__ mu,
                                  double* __restrict__ part) {
    __shared__ double red[40];
    double tm = sum_partials(com_part, ncomblk, red);
    d3 com = {sum_partials(com_part + ncomblk, ncomblk, red), sum_partials(com_part + 2 * ncomblk, ncomblk, red),
              sum_partials(com_part + 3 * ncomblk, ncomblk, red)};
    if (tm > 0.0) com = com * (1.0 / tm);
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (i < n) {
        double q = charge[i];
        d3 p = ld3(pos + 3 * i) - com;
        d3 nd = ld3(lab + 3 * i) + ld3(mu + 3 * i);
        v[0] = q;
        d3 dp = p * q + nd;
        v[1] = dp.x;
        v[2] = dp.y;
        v[3] = dp.z;
        v[4] = p.x * p.x * q + 2.0 * p.x * nd.x;
        v[5] = p.x * p.y * q + p.x * nd.y + p.y * nd.x;
        v[6] = p.x * p.z * q + p.x * nd.z + p.z * nd.x;
        v[7] = p.y * p.y * q + 2.0 * p.y * nd.y;
        v[8] = p.y * p.z * q + p.y * nd.z + p.z * nd.y;
        v[9] = p.z * p.z * q + 2.0 * p.z * nd.z;
    }
    for (int c = 0; c < 10; c++) {
        double s = block_sum(v[c], red);
        if (threadIdx.x == 0) part[(size_t)c * gridDim.x + blockIdx.x] = s;
    }
}

__global__ void k_moment_final(int nblk, const double* __restrict__ part, double* __restrict__ out13) {
    __shared__ double red[40];
    double s[10];
    for (int c = 0; c < 10; c++) s[c] = sum_partials(part + (size_t)c * nblk, nblk, red);
    if (threadIdx.x != 0) return;
    double xx = s[4], xy = s[5], xz = s[6], yy = s[7], yz = s[8], zz = s[9];
    double qave = (xx + yy + zz) / 3.0;
    double o[13];
    o[4] = 0.5 * (xx - qave);
    o[5] = 0.5 * xy;
    o[6] = 0.5 * xz;
    o[8] = 0.5 * (yy - qave);
    o[9] = 0.5 * yz;
    o[12] = 0.5 * (zz - qave);
    o[7] = o[5];
    o[10] = o[6];
    o[11] = o[9];
    double debye = 4.80321;
    o[0] = s[0];
    o[1] = s[1] * (10.0 * debye);
    o[2] = s[2] * (10.0 * debye);
    o[3] = s[3] * (10.0 * debye);
    debye *= 3.0;
    for (int k = 4; k < 13; k++) o[k] *= 100.0 * debye;
    for (int k = 0; k < 13; k++) out13[k] = o[k];
}

// ---------------------------------------------------------------------------
// Launchers.
// ---------------------------------------------------------------------------
static inline int nblk(int n, int t) { return (n + t - 1) / t; }

template <class R>
void launch_pack(const Dev& d, cudaStream_t st) {
    int threads = 128;
    int warps = d.n_pad / kTile;
    k_pack<R><<<nblk(warps * 32, threads), threads, 0, st>>>(
        d.n, warps, d.pos, d.charge, d.tctr, d.text, (typename Vec4T<R>::type*)d.posq, d.yz);
    k_pack_sorted<R><<<nblk(warps * 32, threads), threads, 0, st>>>(
        warps, d.order, d.pos, d.charge, d.tctr_s, d.text_s, (typename Vec4T<R>::type*)d.posq_s, d.pos_s);
}

template <class R>
void launch_rotate(const Dev& d, cudaStream_t st) {
    k_rotate<R><<<nblk(d.n, kVecThreads), kVecThreads, 0, st>>>(d.n, d.pos, d.dip_mol, d.axis, d.thole, d.lab,
                                                                 (typename Vec4T<R>::type*)d.dipt, d.rank,
                                                                 (typename Vec4T<R>::type*)d.dipt_s);
}

#define TDP_INSTANTIATE(R)                                                                                  \
    template void launch_pack<R>(const Dev&, cudaStream_t);                                                 \
    template void launch_rotate<R>(const Dev&, cudaStream_t);

TDP_INSTANTIATE(float)
TDP_INSTANTIATE(double)

template <class R>
void launch_fixed_done(const Dev& d, cudaStream_t st) {
    k_fixed_done<R><<<nblk(d.n, kVecThreads), kVecThreads, 0, st>>>(d.n, d.rank, d.nsplit, d.n_pad, d.partial, d.alpha,
                                                                     d.salpha, d.thole, d.E, d.mu, d.y,
                                                                     (typename Vec4T<R>::type*)d.vec_s);
}
void launch_predict(const Dev& d, int nh, const double* c, cudaStream_t st) {
    const size_t n3 = 3 * (size_t)d.n;
    k_predict<<<nblk(n3, kVecThreads), kVecThreads, 0, st>>>(n3, nh, d.mu_hist[0], d.mu_hist[1], d.mu_hist[2],
                                                              d.mu_hist[3], c[0], c[1], c[2], c[3], d.mu);
}
template <class R>
void launch_warm_start(const Dev& d, cudaStream_t st) {
    k_warm_start<R><<<nblk(d.n, kVecThreads), kVecThreads, 0, st>>>(d.n, d.rank, d.salpha, d.thole, d.mu, d.y,
                                                                     (typename Vec4T<R>::type*)d.vec_s);
}
template <class R>
void launch_cg_residual(const Dev& d, cudaStream_t st, bool use_partial) {
    k_cg_residual<R><<<d.nvb, kVecThreads, 0, st>>>(d.n, d.rank, d.nsplit, d.n_pad, d.partial, d.E, d.salpha, d.thole, d.y,
                                                    d.r, d.p, (typename Vec4T<R>::type*)d.vec_s, d.rr_part, d.eps_part,
                                                    use_partial ? 1 : 0);
}
template <class R>
void launch_pack_total(const Dev& d, cudaStream_t st) {
    k_pack_total<R><<<nblk(d.n, kVecThreads), kVecThreads, 0, st>>>(d.n, d.rank, d.lab, d.mu, d.thole,
                                                                     (typename Vec4T<R>::type*)d.vec_s);
}
template <class R>
void launch_fused_done(const Dev& d, cudaStream_t st) {
    k_fused_done<<<nblk(d.n, kVecThreads), kVecThreads, 0, st>>>(d.n, d.rank, d.nsplit, d.n_pad, d.partial, d.salpha,
                                                                 d.mu, d.E, d.y);
}
void launch_cg_q(const Dev& d, cudaStream_t st) {
    k_cg_q<<<d.nvb, kVecThreads, 0, st>>>(d.n, d.rank, d.nsplit, d.n_pad, d.partial, d.salpha, d.p, d.q, d.pq_part);
}
void launch_cg_update(const Dev& d, int slot, cudaStream_t st) {
    k_cg_update<<<d.nvb, kVecThreads, 0, st>>>(d.n, d.nvb, d.scal_rr, slot, d.pq_part, d.salpha, d.p, d.q, d.y, d.r,
                                               d.rr_part, d.eps_part, d.scal_a);
}
template <class R>
void launch_cg_p(const Dev& d, int prev, int slot, cudaStream_t st) {
    k_cg_p<R><<<d.nvb, kVecThreads, 0, st>>>(d.n, d.rank, d.nvb, prev, slot, d.scal_rr, d.scal_eps, d.rr_part, d.eps_part, d.salpha,
                                             d.thole, d.r, d.p, (typename Vec4T<R>::type*)d.vec_s);
}
template <class R>
void launch_cg_mu(const Dev& d, cudaStream_t st, const double* mu0) {
    k_cg_mu<R><<<d.nvb, kVecThreads, 0, st>>>(d.n, d.rank, d.salpha, d.thole, d.y, d.mu, (typename Vec4T<R>::type*)d.vec_s,
                                              mu0);
}
template <class R>
void launch_jacobi(const Dev& d, cudaStream_t st) {
    k_jacobi<R><<<d.nvb, kVecThreads, 0, st>>>(d.n, d.rank, d.nsplit, d.n_pad, d.partial, d.E, d.alpha, d.thole, d.mu,
                                               (typename Vec4T<R>::type*)d.vec_s, d.eps_part);
}
template <class R>
void launch_extrap_step(const Dev& d, int k, cudaStream_t st) {
    k_extrap_step<R><<<d.nvb, kVecThreads, 0, st>>>(d.n, d.rank, d.nsplit, d.n_pad, d.partial, d.E, d.alpha, d.thole, d.mu,
                                                    d.hist + (size_t)k * 3 * d.n, (typename Vec4T<R>::type*)d.vec_s);
}
template <class R>
void launch_extrap_combine(const Dev& d, int korder, const double* coef, cudaStream_t st) {
    k_extrap_combine<R><<<d.nvb, kVecThreads, 0, st>>>(d.n, d.rank, korder, coef, d.hist, d.thole, d.mu,
                                                       (typename Vec4T<R>::type*)d.vec_s);
}
void launch_step_eps(const Dev& d, cudaStream_t st) {
    k_step_eps<<<d.nvb, kVecThreads, 0, st>>>(d.n, d.rank, d.nsplit, d.n_pad, d.partial, d.E, d.alpha, d.mu, d.eps_part);
}
void launch_eps_scalar(const Dev& d, int slot, cudaStream_t st) {
    k_eps_scalar<<<1, kVecThreads, 0, st>>>(d.n, d.nvb, d.eps_part, d.scal_eps, slot);
}
template <class R>
void launch_pack_ind(const Dev& d, cudaStream_t st) {
    k_pack_ind<R><<<d.nvb, kVecThreads, 0, st>>>(d.n, d.mu, (typename Vec4T<R>::type*)d.ind);
}
void launch_energy_done(const Dev& d, cudaStream_t st) {
    k_energy_done<<<d.nvb, kVecThreads, 0, st>>>(d.n, d.nsplit, d.n_pad, d.n_eblk, d.partial, d.energy_partial,
                                                 d.fpair, d.torque, d.energy);
}
void launch_torque_gather(const Dev& d, cudaStream_t st) {
    k_torque_gather<<<d.nvb, kVecThreads, 0, st>>>(d.n, d.pos, d.axis, d.torque, d.users_off, d.users, d.fpair,
                                                   d.ftotal);
}
void launch_add_forces(const Dev& d, void* acc, int is_f32, cudaStream_t st) {
    int n3 = 3 * d.n;
    k_add_forces<<<nblk(n3, kVecThreads), kVecThreads, 0, st>>>(n3, d.ftotal, is_f32 ? nullptr : (double*)acc,
                                                                 is_f32 ? (float*)acc : nullptr);
}
void launch_positions_in(const Dev& d, const void* src, int is_f32, cudaStream_t st) {
    int n3 = 3 * d.n;
    k_positions_in<<<nblk(n3, kVecThreads), kVecThreads, 0, st>>>(n3, src, is_f32, d.pos);
}
void launch_posq_in(const Dev& d, const void* posq, int is_double, const int* atom_index, cudaStream_t st) {
    k_posq_in<<<nblk(d.n, kVecThreads), kVecThreads, 0, st>>>(d.n, posq, is_double, atom_index, d.pos);
}
void launch_forces_out_fixed(const Dev& d, const int* atom_index, int padded, long long* acc, cudaStream_t st) {
    k_forces_out_fixed<<<nblk(d.n, kVecThreads), kVecThreads, 0, st>>>(d.n, d.ftotal, atom_index, padded,
                                                                        (unsigned long long*)acc);
}
void launch_potential(const Dev& d, const double* grid, int ng, double* out, cudaStream_t st) {
    k_potential<<<nblk(ng, 128), 128, 0, st>>>(d.n, ng, d.pp, d.pos, d.charge, d.lab, d.mu, grid, out);
}
void launch_moments(const Dev& d, const double* mass, double* scratch, double* out13, cudaStream_t st) {
    int nb = d.nvb;
    k_com_partials<<<nb, kVecThreads, 0, st>>>(d.n, d.pos, mass, scratch);
    k_moment_partials<<<nb, kVecThreads, 0, st>>>(d.n, nb, scratch, d.pos, d.charge, d.lab, d.mu, scratch + 4 * nb);
    k_moment_final<<<1, kVecThreads, 0, st>>>(nb, scratch + 4 * nb, out13);
}

#define TDP_INSTANTIATE2(R)                                                         \
    template void launch_fixed_done<R>(const Dev&, cudaStream_t);                   \
    template void launch_warm_start<R>(const Dev&, cudaStream_t);                   \
    template void launch_cg_residual<R>(const Dev&, cudaStream_t, bool);            \
    template void launch_pack_total<R>(const Dev&, cudaStream_t);                   \
    template void launch_fused_done<R>(const Dev&, cudaStream_t);                   \
    template void launch_cg_p<R>(const Dev&, int, int, cudaStream_t);               \
    template void launch_cg_mu<R>(const Dev&, cudaStream_t, const double*);         \
    template void launch_jacobi<R>(const Dev&, cudaStream_t);                       \
    template void launch_extrap_step<R>(const Dev&, int, cudaStream_t);             \
    template void launch_extrap_combine<R>(const Dev&, int, const double*, cudaStream_t); \
    template void launch_pack_ind<R>(const Dev&, cudaStream_t);

TDP_INSTANTIATE2(float)
TDP_INSTANTIATE2(double)

}  // namespace tdp
