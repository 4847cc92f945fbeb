// tdp_precond.cu -- Ewald-operator preconditioner of the minimum-image CG
// solve (tdp_precond.cuh describes the method).
//
// Every vector here is FP64 (n*3, atom order); B's matvec is the Ewald mode's
// (tdp_ewald.cu) in the form's arithmetic, reading the packed operand in
// vec_s and leaving real space in partial slot 0 and reciprocal space plus
// self term in slot 1.  Reductions are block partials summed in a fixed order
// by the next kernel, so an application is deterministic.
#include "tdp_ewald.cuh"
#include "tdp_frames.cuh"
#include "tdp_host.h"
#include "tdp_precond.cuh"

#include <math.h>

#include <algorithm>
#include <vector>

namespace tdp {

namespace {

constexpr double kPi = 3.1415926535897932385;
constexpr int kMaxInner = 8;
// Block-partial regions (each nvb doubles): r.r of the inner residual, by the
// parity of the inner iteration; the three components of M = sum sqrt(alpha) p;
// p.q; and for the outer beta r.z and z.q.
enum { kRR0 = 0, kRR1 = 1, kMx = 2, kMy = 3, kMz = 4, kPQ = 5, kRZ = 6, kZQ = 7, kRegions = 8 };
// Scalars: [0] the scale sigma of the residual, [1 + j] the inner r.r of
// iteration j.
constexpr int kScal = 2 + kMaxInner;

__device__ __forceinline__ void st3(double* v, int i, d3 a) {
    v[3 * i] = a.x;
    v[3 * i + 1] = a.y;
    v[3 * i + 2] = a.z;
}

template <class R>
__device__ __forceinline__ void pack_vec(typename Vec4T<R>::type* v, int slot, d3 a, double t) {
    typename Vec4T<R>::type o;
    o.x = (R)a.x;
    o.y = (R)a.y;
    o.z = (R)a.z;
    o.w = (R)t;
    v[slot] = o;
}

// Inner start: v = sigma r with sigma = 1 / RMS(r) per atom; rin = pin = v;
// packs sqrt(alpha) v; partials of v.v (kRR0) and of M (kMx..kMz).
template <class R>
__global__ void k_pc_start(int n, const int* __restrict__ rank, int nvb, const double* __restrict__ rr_part,
                           const double* __restrict__ salpha, const double* __restrict__ thole,
                           const double* __restrict__ r, double* __restrict__ rin, double* __restrict__ pin,
                           typename Vec4T<R>::type* __restrict__ vec, double* __restrict__ part,
                           double* __restrict__ scal) {
    __shared__ double red[40];
    const double rr = sum_partials(rr_part, nvb, red);
    const double sig = rr > 0.0 ? sqrt((double)n / rr) : 1.0;
    if (blockIdx.x == 0 && threadIdx.x == 0) scal[0] = sig;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double vv = 0.0;
    d3 m = {0.0, 0.0, 0.0};
    if (i < n) {
        const d3 v = ld3(r + 3 * i) * sig;
        st3(rin, i, v);
        st3(pin, i, v);
        m = v * salpha[i];
        pack_vec<R>(vec, rank[i], m, thole[i]);
        vv = dot(v, v);
    }
    vv = block_sum(vv, red);
    m.x = block_sum(m.x, red);
    m.y = block_sum(m.y, red);
    m.z = block_sum(m.z, red);
    if (threadIdx.x == 0) {
        part[(size_t)kRR0 * nvb + blockIdx.x] = vv;
        part[(size_t)kMx * nvb + blockIdx.x] = m.x;
        part[(size_t)kMy * nvb + blockIdx.x] = m.y;
        part[(size_t)kMz * nvb + blockIdx.x] = m.z;
    }
}

// q = p - sqrt(alpha) (T_B sqrt(alpha) p - csurf M); partials of p.q.
__global__ void k_pc_q(int n, const int* __restrict__ rank, int n_pad, const double* __restrict__ partial, int nvb,
                       double csurf, const double* __restrict__ salpha, const double* __restrict__ pin,
                       double* __restrict__ qin, double* __restrict__ part) {
    __shared__ double red[40];
    const d3 M = {sum_partials(part + (size_t)kMx * nvb, nvb, red), sum_partials(part + (size_t)kMy * nvb, nvb, red),
                  sum_partials(part + (size_t)kMz * nvb, nvb, red)};
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double pq = 0.0;
    if (i < n) {
        const int k = rank[i];
        d3 f;
        f.x = partial[k] + partial[3 * (size_t)n_pad + k];
        f.y = partial[(size_t)n_pad + k] + partial[4 * (size_t)n_pad + k];
        f.z = partial[2 * (size_t)n_pad + k] + partial[5 * (size_t)n_pad + k];
        f = f - M * csurf;
        const d3 p = ld3(pin + 3 * i);
        const d3 q = p - f * salpha[i];
        st3(qin, i, q);
        pq = dot(p, q);
    }
    pq = block_sum(pq, red);
    if (threadIdx.x == 0) part[(size_t)kPQ * nvb + blockIdx.x] = pq;
}

// a = rr_j / p.q; x += a p (x = a p at j = 0).  Not last: rin -= a q and
// partials of the new rin.rin.  Last: z = x / sigma and the outer partials
// r.z and (not first) z.q_outer.
__global__ void k_pc_update(int n, int nvb, int j, int last, int first, double* __restrict__ part,
                            double* __restrict__ scal, const double* __restrict__ pin, const double* __restrict__ qin,
                            double* __restrict__ rin, double* __restrict__ x, const double* __restrict__ r,
                            const double* __restrict__ q_outer) {
    __shared__ double red[40];
    const double rr = sum_partials(part + (size_t)(j & 1) * nvb, nvb, red);
    const double pq = sum_partials(part + (size_t)kPQ * nvb, nvb, red);
    const double a = pq != 0.0 ? rr / pq : 0.0;
    if (blockIdx.x == 0 && threadIdx.x == 0) scal[1 + j] = rr;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double s0 = 0.0, s1 = 0.0;
    if (i < n) {
        const d3 p = ld3(pin + 3 * i);
        const d3 xv = (j == 0 ? d3{0.0, 0.0, 0.0} : ld3(x + 3 * i)) + p * a;
        if (!last) {
            const d3 rv = ld3(rin + 3 * i) - ld3(qin + 3 * i) * a;
            st3(rin, i, rv);
            st3(x, i, xv);
            s0 = dot(rv, rv);
        } else {
            const d3 z = xv * (1.0 / scal[0]);
            st3(x, i, z);
            s0 = dot(ld3(r + 3 * i), z);
            if (!first) s1 = dot(z, ld3(q_outer + 3 * i));
        }
    }
    s0 = block_sum(s0, red);
    s1 = block_sum(s1, red);
    if (threadIdx.x == 0) {
        if (!last) {
            part[(size_t)((j + 1) & 1) * nvb + blockIdx.x] = s0;
        } else {
            part[(size_t)kRZ * nvb + blockIdx.x] = s0;
            part[(size_t)kZQ * nvb + blockIdx.x] = s1;
        }
    }
}

// Inner direction of iteration j >= 1: beta = rr_j / rr_(j-1);
// p = rin + beta p; packs sqrt(alpha) p; partials of M.
template <class R>
__global__ void k_pc_p(int n, const int* __restrict__ rank, int nvb, int j, double* __restrict__ part,
                       const double* __restrict__ scal, const double* __restrict__ salpha,
                       const double* __restrict__ thole, const double* __restrict__ rin, double* __restrict__ pin,
                       typename Vec4T<R>::type* __restrict__ vec) {
    __shared__ double red[40];
    const double rr = sum_partials(part + (size_t)(j & 1) * nvb, nvb, red);
    const double prev = scal[j];
    const double beta = prev != 0.0 ? rr / prev : 0.0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    d3 m = {0.0, 0.0, 0.0};
    if (i < n) {
        const d3 p = ld3(rin + 3 * i) + ld3(pin + 3 * i) * beta;
        st3(pin, i, p);
        m = p * salpha[i];
        pack_vec<R>(vec, rank[i], m, thole[i]);
    }
    m.x = block_sum(m.x, red);
    m.y = block_sum(m.y, red);
    m.z = block_sum(m.z, red);
    if (threadIdx.x == 0) {
        part[(size_t)kMx * nvb + blockIdx.x] = m.x;
        part[(size_t)kMy * nvb + blockIdx.x] = m.y;
        part[(size_t)kMz * nvb + blockIdx.x] = m.z;
    }
}

// Outer direction: scal_rr[slot] = r.z; p = z (first) or z + beta p with
// beta = -a_(slot-1) z.q / (r.z)_(slot-1); packs sqrt(alpha) p.
template <class R>
__global__ void k_pcg_p(int n, const int* __restrict__ rank, int nvb, int slot, int first,
                        const double* __restrict__ part, double* __restrict__ scal_rr,
                        const double* __restrict__ scal_a, const double* __restrict__ salpha,
                        const double* __restrict__ thole, const double* __restrict__ z, double* __restrict__ p,
                        typename Vec4T<R>::type* __restrict__ vec) {
    __shared__ double red[40];
    const double rz = sum_partials(part + (size_t)kRZ * nvb, nvb, red);
    double beta = 0.0;
    if (!first) {
        const double zq = sum_partials(part + (size_t)kZQ * nvb, nvb, red);
        const double prev = scal_rr[slot - 1];
        beta = prev != 0.0 ? -scal_a[slot - 1] * zq / prev : 0.0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) scal_rr[slot] = rz;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const d3 zv = ld3(z + 3 * i);
    const d3 pv = first ? zv : zv + ld3(p + 3 * i) * beta;
    st3(p, i, pv);
    pack_vec<R>(vec, rank[i], pv * salpha[i], thole[i]);
}

// Cold start, first half: r = b = sqrt(alpha) E (the residual of y = 0) and
// block partials of r.r for the scale of the inner solve.
__global__ void k_pc_rhs(int n, const double* __restrict__ salpha, const double* __restrict__ E,
                         double* __restrict__ r, double* __restrict__ rr_part) {
    __shared__ double red[40];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double rr = 0.0;
    if (i < n) {
        const d3 b = ld3(E + 3 * i) * salpha[i];
        st3(r, i, b);
        rr = dot(b, b);
    }
    rr = block_sum(rr, red);
    if (threadIdx.x == 0) rr_part[blockIdx.x] = rr;
}

// Cold start, second half: y = z = M(b); mu = sqrt(alpha) y packed as the
// operand of the residual's matvec.
template <class R>
__global__ void k_pc_take(int n, const int* __restrict__ rank, const double* __restrict__ salpha,
                          const double* __restrict__ thole, const double* __restrict__ z, double* __restrict__ y,
                          double* __restrict__ mu, typename Vec4T<R>::type* __restrict__ vec) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const d3 zv = ld3(z + 3 * i);
    st3(y, i, zv);
    const d3 m = zv * salpha[i];
    st3(mu, i, m);
    pack_vec<R>(vec, rank[i], m, thole[i]);
}

}  // namespace

struct Precond {
    Ewald* ew = nullptr;
    std::vector<void*> owned;
    double cutoff = 0.6, tol = 1e-3;
    int inner = 3;
    double csurf = 0.0;
    double* z = nullptr;
    double* rin = nullptr;
    double* pin = nullptr;
    double* qin = nullptr;
    double* part = nullptr;
    double* scal = nullptr;
    int launches = 0;

    ~Precond() {
        if (ew) ewald_destroy(ew);
        for (void* p : owned) cudaFree(p);
    }
};

Precond* precond_create(const Dev& d, int precision, double cutoff, double tol, int inner) {
    Precond* p = new Precond();
    try {
        p->cutoff = cutoff;
        p->tol = tol;
        p->inner = std::min(std::max(inner, 1), kMaxInner);
        p->ew = ewald_create(d, precision, false, false);
        const size_t n3 = 3 * (size_t)std::max(d.n, 1);
        p->z = dalloc<double>(n3, p->owned);
        p->rin = dalloc<double>(n3, p->owned);
        p->pin = dalloc<double>(n3, p->owned);
        p->qin = dalloc<double>(n3, p->owned);
        p->part = dalloc<double>((size_t)kRegions * d.nvb, p->owned);
        p->scal = dalloc<double>(kScal, p->owned);
    } catch (...) {
        delete p;
        throw;
    }
    return p;
}

void precond_destroy(Precond* p) { delete p; }

double precond_cutoff(const Precond* p) { return p->cutoff; }

void precond_prepare(Precond* p, const Dev& d, const double box[3], cudaStream_t st) {
    const int grid0[3] = {0, 0, 0};
    ewald_prepare(p->ew, d, box, p->cutoff, p->tol, 0.0, grid0, st);
    p->csurf = 4.0 * kPi / (3.0 * box[0] * box[1] * box[2]);
    ewald_build_list(p->ew, d, st);
}

namespace {

// z = M(r) from d.r (r.r block partials in d.rr_part); with first = false
// also the partials of z.q for the flexible beta.  Returns the launches.
template <class R>
int inner_solve(Precond* p, const Dev& d, bool first, cudaStream_t st) {
    typedef typename Vec4T<R>::type V4;
    const int nvb = d.nvb;
    V4* vec = (V4*)d.vec_s;
    int launches = 0;
    k_pc_start<R><<<nvb, kVecThreads, 0, st>>>(d.n, d.rank, nvb, d.rr_part, d.salpha, d.thole, d.r, p->rin, p->pin,
                                               vec, p->part, p->scal);
    launches++;
    for (int j = 0; j < p->inner; j++) {
        const bool last = j == p->inner - 1;
        ewald_matvec<R>(p->ew, d, st);
        launches += ewald_last_launches(p->ew);
        k_pc_q<<<nvb, kVecThreads, 0, st>>>(d.n, d.rank, d.n_pad, d.partial, nvb, p->csurf, d.salpha, p->pin, p->qin,
                                            p->part);
        k_pc_update<<<nvb, kVecThreads, 0, st>>>(d.n, nvb, j, last ? 1 : 0, first ? 1 : 0, p->part, p->scal, p->pin,
                                                 p->qin, p->rin, p->z, d.r, d.q);
        launches += 2;
        if (!last) {
            k_pc_p<R><<<nvb, kVecThreads, 0, st>>>(d.n, d.rank, nvb, j + 1, p->part, p->scal, d.salpha, d.thole,
                                                   p->rin, p->pin, vec);
            launches++;
        }
    }
    return launches;
}

}  // namespace

template <class R>
void precond_apply(Precond* p, const Dev& d, int slot, bool first, cudaStream_t st) {
    typedef typename Vec4T<R>::type V4;
    int launches = inner_solve<R>(p, d, first, st);
    k_pcg_p<R><<<d.nvb, kVecThreads, 0, st>>>(d.n, d.rank, d.nvb, slot, first ? 1 : 0, p->part, d.scal_rr, d.scal_a,
                                              d.salpha, d.thole, p->z, d.p, (V4*)d.vec_s);
    launches++;
    TDP_CUDA(cudaGetLastError());
    p->launches = launches;
}

template <class R>
void precond_cold_start(Precond* p, const Dev& d, cudaStream_t st) {
    typedef typename Vec4T<R>::type V4;
    k_pc_rhs<<<d.nvb, kVecThreads, 0, st>>>(d.n, d.salpha, d.E, d.r, d.rr_part);
    int launches = 1 + inner_solve<R>(p, d, true, st);
    k_pc_take<R><<<d.nvb, kVecThreads, 0, st>>>(d.n, d.rank, d.salpha, d.thole, p->z, d.y, d.mu, (V4*)d.vec_s);
    launches++;
    TDP_CUDA(cudaGetLastError());
    p->launches = launches;
}

int precond_last_launches(const Precond* p) { return p->launches; }
int precond_list_overflow(const Precond* p) { return ewald_list_overflow(p->ew); }

template void precond_apply<float>(Precond*, const Dev&, int, bool, cudaStream_t);
template void precond_apply<double>(Precond*, const Dev&, int, bool, cudaStream_t);
template void precond_cold_start<float>(Precond*, const Dev&, cudaStream_t);
template void precond_cold_start<double>(Precond*, const Dev&, cudaStream_t);

}  // namespace tdp
