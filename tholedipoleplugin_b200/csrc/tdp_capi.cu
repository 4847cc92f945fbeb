// tdp_capi.cu -- C ABI (include/tholedipole_b200.h) over the sm_100a kernels:
// validation, the covalent scale tables, device buffers and the per-call
// orchestration of rotation -> permanent field -> induced-dipole solve ->
// energy/force/torque -> torque mapping, in the reference's semantics
// (aehogan/tholedipoleplugin, platforms/reference/src/ReferenceTholeDipoleForce.cpp,
// driven as ReferenceCalcTholeDipoleForceKernel does in
// platforms/reference/src/ReferenceTholeDipoleKernels.cpp).
#include "tholedipole_b200.h"
#include "tdp_ewald.cuh"
#include "tdp_precond.cuh"
#include "tdp_host.h"
#include "tdp_kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

using namespace tdp;

namespace tdp {
const char* noalloc_error_message();
void noalloc_clear_error();
}  // namespace tdp

namespace {

thread_local std::string g_create_error;

}  // namespace

struct tdp_handle {
    int n = 0;
    int method = TDP_NO_CUTOFF;
    int polarization = TDP_MUTUAL;
    int precision = TDP_PRECISION_MIXED;
    int solver = TDP_SOLVER_CG;
    uint32_t flags = 0;
    double cutoff = 1.0, ewald_tol = 1e-4, pme_alpha = 0.0;
    int pme_grid[3] = {0, 0, 0};
    double target_eps = 1e-5;
    int max_iter = 60;
    std::vector<double> extrap;
    double box[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    bool have_box = false;

    // Host copies of the per-particle parameters.
    std::vector<double> charge, dip, alpha, thole;
    std::vector<int> axis;  // n*4
    // Covalent scale exceptions by atom: (partner, M scale, I scale).
    std::vector<std::vector<std::tuple<int, double, double>>> exc_user;
    size_t n_exc = 0;
    // Molecules (connected by covalent lists and axis atoms), CSR in index order;
    // the field kernels order molecules along a Morton curve.
    std::vector<int> comp_off, comp_atoms;
    bool sorted = false;
    int since_sort = 0;
    int resort_interval = 1000;
    std::vector<double> hpos;

    Dev d;
    std::vector<void*> owned;
    cudaStream_t stream = nullptr;
    double* h_scal = nullptr;   // pinned scalar readback
    int* h_fixerr = nullptr;    // pinned copy of the accumulator range flag
    double* h_forces = nullptr; // pinned n*3
    double* d_stage = nullptr;  // device staging for host FP32 positions / query inputs
    size_t stage_bytes = 0;
    int n_hist = 0;         // valid entries of d.mu_hist
    int predictor = 3;      // history points the warm-start predictor uses (1-4, TDP_PREDICTOR)
    // Warm-started Mutual solves start with one walk that gives E + T mu0
    // (TDP_FUSED_START=0 keeps the separate permanent-field walk and matvec).
    bool fused_start = true;
    // TDP_TRUE_RESIDUAL=1: confirm every CG solve on the true residual, even
    // when the drift bound makes the check redundant (see solve_cg).
    bool always_true_residual = false;
    bool e_shifted = false;   // the last solve started fused: d.E holds E + T mu0, d.mu0 holds mu0
    bool have_results = false;

    int iterations = 0;
    double epsilon = 1.0e50;
    int converged = 0;
    int status = TDP_STATUS_CONVERGED;
    int matvecs = 0;
    size_t nscal = 0;  // capacity of the per-iteration scalar arrays
    int eps_slots = 0; // stopping quantities the last CG / Jacobi solve left in d.scal_eps

    bool timing = false;
    cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    std::vector<cudaEvent_t> kev;  // event pairs around matvec / energy kernels
    std::vector<int> kev_kind;     // 0 matvec, 1 energy, 2 fused start, 3 preconditioner, per pair
    size_t kev_used = 0;
    double stage_ms[TDP_NUM_STAGE_TIMES] = {};
    long launches = 0;

    // Ewald mode (TDP_FLAG_EWALD): neighbour list, PME grid and plans.
    Ewald* ew = nullptr;
    // Minimum-image Mutual CG: the Ewald-operator preconditioner
    // (tdp_precond.cuh), used whenever the box holds twice its cutoff.
    Precond* pre = nullptr;
    int pre_applications = 0;   // B matvecs of the last evaluation
    double total_charge = 0.0;

    // Device scratch of the device-side parameter update and the adjoint's
    // right-hand-side scale (allocated on first use).
    double* d_pstat = nullptr;

    // Adjoint work buffers (allocated on first use).
    double* adj = nullptr;
    double adj_eps = 0.0;
    int adj_iterations = 0;

    std::string err;
};

namespace {

int fail(tdp_handle* h, const TdpError& e) {
    if (h) {
        h->err = e.msg;
    } else {
        g_create_error = e.msg;
        noalloc_clear_error();
    }
    return e.code;
}

// Per-particle parameters and everything derived from them.
void upload_params(tdp_handle* h) {
    int n = h->n;
    Dev& d = h->d;
    std::vector<double> sal(n);
    for (int i = 0; i < n; i++) sal[i] = h->alpha[i] > 0.0 ? std::sqrt(h->alpha[i]) : 0.0;
    upload(d.charge, h->charge.data(), sizeof(double) * n);
    // Net charge for the neutralising-plasma term, from the charges as the pair
    // records hold them (FP32 in the mixed form), which reciprocal space sums.
    h->total_charge = 0.0;
    for (int i = 0; i < n; i++)
        h->total_charge += h->precision == TDP_PRECISION_DOUBLE ? h->charge[i] : (double)(float)h->charge[i];
    upload(d.dip_mol, h->dip.data(), sizeof(double) * 3 * n);
    upload(d.alpha, h->alpha.data(), sizeof(double) * n);
    upload(d.salpha, sal.data(), sizeof(double) * n);
    upload(d.thole, h->thole.data(), sizeof(double) * n);
    upload(d.axis, h->axis.data(), sizeof(int) * 4 * n);
    d.pp.damp_r2 = (float)damp_radius2(h->thole);

    // Torque-mapping users: which atoms receive force from the frame of atom
    // i, and in which role.
    std::vector<int> off;
    std::vector<int2> flat;
    torque_users(n, h->axis, off, flat);
    if (d.users) {
        cudaFree(d.users);
        h->owned.erase(std::find(h->owned.begin(), h->owned.end(), (void*)d.users));
    }
    d.users = dalloc<int2>(flat.size(), h->owned);
    upload(d.users_off, off.data(), sizeof(int) * (n + 1));
    upload(d.users, flat.data(), sizeof(int2) * flat.size());
}

// Per-particle parameters given on the device: sqrt(alpha), and in one CTA
// (fixed summation order) the largest Thole factor, whether any is negative or
// not a number, and the net charge as the pair records hold it.
__global__ void k_param_stats(int n, int f32_charges, const double* __restrict__ alpha,
                              const double* __restrict__ thole, const double* __restrict__ charge,
                              double* __restrict__ salpha, double* __restrict__ out) {
    __shared__ double s_max[1024], s_q[1024];
    __shared__ int s_bad[1024];
    double tmax = 0.0, qsum = 0.0;
    int bad = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double a = alpha[i];
        salpha[i] = a > 0.0 ? sqrt(a) : 0.0;
        const double t = thole[i];
        if (t < 0.0 || isnan(t)) bad = 1;
        else tmax = fmax(tmax, t);
        qsum += f32_charges ? (double)(float)charge[i] : charge[i];
    }
    s_max[threadIdx.x] = tmax;
    s_q[threadIdx.x] = qsum;
    s_bad[threadIdx.x] = bad;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (unsigned k = 1; k < blockDim.x; k++) {
            tmax = fmax(tmax, s_max[k]);
            qsum += s_q[k];
            bad |= s_bad[k];
        }
        out[0] = tmax;
        out[1] = bad;
        out[2] = qsum;
    }
}

// s2 = sum_i |alpha_i v_i|^2 over n*3 values, one CTA, fixed order.
__global__ void k_alpha_norm2(int n, const double* __restrict__ alpha, const double* __restrict__ v,
                              double* __restrict__ out) {
    __shared__ double s[1024];
    double acc = 0.0;
    for (int k = threadIdx.x; k < 3 * n; k += blockDim.x) {
        const double x = alpha[k / 3] * v[k];
        acc += x * x;
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (unsigned k = 1; k < blockDim.x; k++) acc += s[k];
        out[0] = acc;
    }
}

// out = alpha v (n*3).
__global__ void k_alpha_scale(int n, const double* __restrict__ alpha, const double* __restrict__ v,
                              double* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < 3 * n) out[k] = alpha[k / 3] * v[k];
}

double* pstat(tdp_handle* h) {
    if (!h->d_pstat) h->d_pstat = dalloc<double>(4, h->owned);
    return h->d_pstat;
}

void refresh_box(tdp_handle* h) {
    PairParams& P = h->d.pp;
    P.periodic = h->method == TDP_PME ? 1 : 0;
    for (int k = 0; k < 3; k++) {
        double L = h->box[4 * k];
        if (!P.periodic || !(L > 0.0)) {
            // getPeriodicDelta skips a zero box dimension (RTDF.cpp:1419).
            P.box[k] = 0.0;
            P.inv_box[k] = 0.0;
            P.half_box_tol[k] = INFINITY;
        } else {
            P.box[k] = L;
            P.inv_box[k] = 1.0 / L;
            // Pairs whose FP32 displacement lies within 16 ulp of half a box are
            // re-derived in FP64.
            int ex;
            std::frexp(L, &ex);
            double ulp = std::ldexp(1.0, ex - 24);
            P.half_box_tol[k] = 0.5 * L - 16.0 * ulp;
        }
    }
}

// Union-find molecules over the covalent lists and axis atoms.
void build_components(tdp_handle* h, const tdp_system_desc* desc) {
    int n = h->n;
    std::vector<int> parent(n);
    for (int i = 0; i < n; i++) parent[i] = i;
    auto find = [&](int a) {
        while (parent[a] != a) a = parent[a] = parent[parent[a]];
        return a;
    };
    auto unite = [&](int a, int b) {
        if (a < 0 || b < 0 || a >= n || b >= n) return;
        a = find(a);
        b = find(b);
        if (a != b) parent[std::max(a, b)] = std::min(a, b);
    };
    for (int i = 0; i < n; i++) {
        unite(i, h->axis[4 * i + 1]);
        unite(i, h->axis[4 * i + 2]);
        unite(i, h->axis[4 * i + 3]);
        for (int list = 0; list < 2; list++) {
            const int32_t* off = list == 0 ? desc->covalent12_offsets : desc->covalent13_offsets;
            const int32_t* atoms = list == 0 ? desc->covalent12_atoms : desc->covalent13_atoms;
            if (!off) continue;
            for (int p = off[i]; p < off[i + 1]; p++) unite(i, atoms[p]);
        }
    }
    std::vector<int> root(n), count(n, 0);
    for (int i = 0; i < n; i++) count[root[i] = find(i)]++;
    std::vector<int> cid(n, -1);
    int nc = 0;
    for (int i = 0; i < n; i++)
        if (root[i] == i) cid[i] = nc++;
    h->comp_off.assign(nc + 1, 0);
    for (int i = 0; i < n; i++) h->comp_off[cid[root[i]] + 1]++;
    for (int c = 0; c < nc; c++) h->comp_off[c + 1] += h->comp_off[c];
    std::vector<int> fill(h->comp_off.begin(), h->comp_off.end() - 1);
    h->comp_atoms.assign(n, 0);
    for (int i = 0; i < n; i++) h->comp_atoms[fill[cid[root[i]]]++] = i;
}

static inline uint64_t spread21(uint64_t v) {
    v &= 0x1fffff;
    v = (v | v << 32) & 0x1f00000000ffffull;
    v = (v | v << 16) & 0x1f0000ff0000ffull;
    v = (v | v << 8) & 0x100f00f00f00f00full;
    v = (v | v << 4) & 0x10c30c30c30c30c3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
}

// Orders molecules along a Morton curve of their centroids (wrapped into the
// box when periodic) and uploads order/rank plus the slot-indexed exception
// tables.  Only the field kernels' memory layout changes; results are the
// same up to summation order.
void sort_atoms(tdp_handle* h) {
    int n = h->n;
    Dev& d = h->d;
    h->hpos.resize(3 * (size_t)n);
    TDP_CUDA(cudaMemcpyAsync(h->hpos.data(), d.pos, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, h->stream));
    TDP_CUDA(cudaStreamSynchronize(h->stream));
    int nc = (int)h->comp_off.size() - 1;
    std::vector<double> cen(3 * (size_t)nc, 0.0);
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int c = 0; c < nc; c++) {
        int a0 = h->comp_off[c], a1 = h->comp_off[c + 1];
        for (int k = 0; k < 3; k++) {
            double sum = 0.0;
            for (int a = a0; a < a1; a++) sum += h->hpos[3 * (size_t)h->comp_atoms[a] + k];
            double v = sum / (a1 - a0);
            double L = d.pp.box[k];
            if (d.pp.periodic && L > 0.0) v -= L * std::floor(v / L);
            if (!std::isfinite(v)) v = 0.0;
            cen[3 * (size_t)c + k] = v;
            lo[k] = std::min(lo[k], v);
            hi[k] = std::max(hi[k], v);
        }
    }
    std::vector<std::pair<uint64_t, int>> keys(nc);
    for (int c = 0; c < nc; c++) {
        uint64_t key = 0;
        for (int k = 0; k < 3; k++) {
            double span = hi[k] - lo[k];
            double f = span > 0.0 ? (cen[3 * (size_t)c + k] - lo[k]) / span : 0.0;
            uint64_t q = (uint64_t)std::min(std::max(f, 0.0) * 2097151.0, 2097151.0);
            key |= spread21(q) << k;
        }
        keys[c] = {key, c};
    }
    std::stable_sort(keys.begin(), keys.end());
    std::vector<int> order(d.n_pad, -1), rank(n);
    int k = 0;
    for (auto& kc : keys)
        for (int a = h->comp_off[kc.second]; a < h->comp_off[kc.second + 1]; a++) {
            int i = h->comp_atoms[a];
            order[k] = i;
            rank[i] = k++;
        }
    std::vector<int> off(n + 1, 0), ej;
    std::vector<double> em, es;
    std::vector<int2> etiles(d.n_pad / kTile, make_int2(1 << 30, -1));
    for (int slot = 0; slot < n; slot++) {
        for (auto& t : h->exc_user[order[slot]]) {
            int js = rank[std::get<0>(t)];
            ej.push_back(js);
            em.push_back(std::get<1>(t));
            es.push_back(std::get<2>(t));
            int2& r = etiles[slot / kTile];
            r.x = std::min(r.x, js / kTile);
            r.y = std::max(r.y, js / kTile);
        }
        off[slot + 1] = (int)ej.size();
    }
    upload(d.order, order.data(), sizeof(int) * order.size());
    upload(d.rank, rank.data(), sizeof(int) * n);
    upload(d.exs_off, off.data(), sizeof(int) * (n + 1));
    upload(d.exs_j, ej.data(), sizeof(int) * ej.size());
    upload(d.exs_m, em.data(), sizeof(double) * em.size());
    upload(d.exs_s, es.data(), sizeof(double) * es.size());
    upload(d.exs_tiles, etiles.data(), sizeof(int2) * etiles.size());
    h->sorted = true;
    h->since_sort = 0;
}

template <class R>
void setup_and_solve(tdp_handle* h);

template <class R>
void run_energy(tdp_handle* h);

void stage_positions(tdp_handle* h, const void* positions, int dtype, int on_device) {
    Dev& d = h->d;
    size_t n3 = 3 * (size_t)h->n;
    if (dtype != TDP_F64 && dtype != TDP_F32) throw TdpError{TDP_ERR_INVALID_ARGUMENT, "unknown position dtype"};
    if (!positions) throw TdpError{TDP_ERR_INVALID_ARGUMENT, "positions is NULL"};
    if (on_device) {
        if (dtype == TDP_F64)
            TDP_CUDA(cudaMemcpyAsync(d.pos, positions, n3 * 8, cudaMemcpyDeviceToDevice, h->stream));
        else
            launch_positions_in(d, positions, 1, h->stream);
    } else {
        // Host coordinates are checked here, before any device work; device
        // coordinates that are not finite surface as a non-finite solve or sum.
        bool finite = true;
        if (dtype == TDP_F64) {
            const double* p = static_cast<const double*>(positions);
            for (size_t k = 0; k < n3; k++) finite &= std::isfinite(p[k]);
        } else {
            const float* p = static_cast<const float*>(positions);
            for (size_t k = 0; k < n3; k++) finite &= std::isfinite(p[k]);
        }
        if (!finite) throw TdpError{TDP_ERR_NON_FINITE, "a particle coordinate is not finite"};
        if (dtype == TDP_F64) {
            TDP_CUDA(cudaMemcpyAsync(d.pos, positions, n3 * 8, cudaMemcpyHostToDevice, h->stream));
        } else {
            TDP_CUDA(cudaMemcpyAsync(h->d_stage, positions, n3 * 4, cudaMemcpyHostToDevice, h->stream));
            launch_positions_in(d, h->d_stage, 1, h->stream);
        }
    }
}

void check_box(tdp_handle* h) {
    if (h->method != TDP_PME) return;
    double minAllowed = 1.999999 * h->cutoff;
    if (!h->have_box || h->box[0] < minAllowed || h->box[4] < minAllowed || h->box[8] < minAllowed)
        throw TdpError{TDP_ERR_BOX_TOO_SMALL, "The periodic box size has decreased to less than twice the nonbonded cutoff."};
    if (h->ew && (h->box[1] != 0.0 || h->box[2] != 0.0 || h->box[3] != 0.0 || h->box[5] != 0.0 || h->box[6] != 0.0 ||
                  h->box[7] != 0.0))
        throw TdpError{TDP_ERR_UNSUPPORTED, "the Ewald mode supports orthorhombic boxes only"};
}

double read_scalar(tdp_handle* h, const double* dptr) {
    TDP_CUDA(cudaMemcpyAsync(h->h_scal, dptr, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    TDP_CUDA(cudaStreamSynchronize(h->stream));
    return *h->h_scal;
}

void record(tdp_handle* h, int k) {
    if (h->timing) TDP_CUDA(cudaEventRecord(h->ev[k], h->stream));
}

// Event pair around one pair-kernel launch (kind 0: matvec, 1: energy, 2:
// fused start, 3: one preconditioner application).
size_t kernel_begin(tdp_handle* h, int kind) {
    if (!h->timing) return 0;
    size_t k = h->kev_used++;
    if (2 * k + 2 > h->kev.size()) {
        cudaEvent_t a, b;
        TDP_CUDA(cudaEventCreate(&a));
        TDP_CUDA(cudaEventCreate(&b));
        h->kev.push_back(a);
        h->kev.push_back(b);
        h->kev_kind.push_back(kind);
    }
    h->kev_kind[k] = kind;
    TDP_CUDA(cudaEventRecord(h->kev[2 * k], h->stream));
    return k;
}
void kernel_end(tdp_handle* h, size_t k) {
    if (h->timing) TDP_CUDA(cudaEventRecord(h->kev[2 * k + 1], h->stream));
}

// One mutual-field matvec (pair kernel), timed and counted.
template <class R>
void matvec(tdp_handle* h) {
    size_t k = kernel_begin(h, 0);
    if (h->ew) {
        ewald_matvec<R>(h->ew, h->d, h->stream);
        h->launches += ewald_last_launches(h->ew);
    } else {
        launch_field<R>(h->d, 1, h->stream);
        h->launches++;
    }
    kernel_end(h, k);
    h->matvecs++;
}

// Mutual polarization by conjugate gradients in y = mu / sqrt(alpha):
// (I - S T S) y = S E with S = diag(sqrt(alpha)), whose fixed point is the
// reference's Jacobi fixed point mu = alpha (E + T mu).  The stopping test is
// the reference's epsilon: the RMS change a Jacobi step would make,
// sqrt(sum alpha |r|^2 / N), confirmed on the true residual before returning.
//
// fused: the start of a warm-started solve whose single field walk left
// E' = E + T mu0 in d.E (mu0 in d.mu0).  The starting residual then needs no
// matvec, and the final check's matvec runs on mu - mu0:
// E + T mu = E' + T (mu - mu0).
//
// The true-residual check guards against the recursive residual drifting
// from the true one (FP32 matvecs).  That drift is bounded by a multiple of
// the residual norms the recursion has stepped through: kDriftPerStep times
// their sum (measured ratio on the 98,304-atom box, mixed form: 4e-10 from a
// cold start, 1.5e-10 warm).  When that bound is below the margin between the
// target and the recursive residual, the check could not change the outcome
// and is skipped (always the case for warm-started MD steps, which then save
// one matvec); TDP_TRUE_RESIDUAL=1 at create keeps it on every solve.
constexpr double kDriftPerStep = 1e-5;
template <class R>
void solve_pcg(tdp_handle* h, bool fused, bool cold);
// cold: the solve starts from y = sqrt(alpha) E (no warm start), which the
// preconditioned form replaces by y = M(sqrt(alpha) E).
template <class R>
void solve_cg(tdp_handle* h, bool fused = false, bool cold = true) {
    Dev& d = h->d;
    cudaStream_t st = h->stream;
    if (h->pre) {
        const double L[3] = {h->box[0], h->box[4], h->box[8]};
        const double rc2 = 2.0 * precond_cutoff(h->pre);
        if (L[0] >= rc2 && L[1] >= rc2 && L[2] >= rc2) {
            precond_prepare(h->pre, d, L, st);
            h->launches += 1;
            solve_pcg<R>(h, fused, cold && !fused);
            return;
        }
    }
    const int cap = h->max_iter;
    int slot = 0;
    // Residual of the starting point (mu = alpha E, or the previous solution).
    if (fused) {
        launch_cg_residual<R>(d, st, false);
    } else {
        matvec<R>(h);
        launch_cg_residual<R>(d, st);
    }
    launch_cg_p<R>(d, -1, slot, st);
    h->launches += 2;
    double eps = read_scalar(h, d.scal_eps + slot);
    double eps_sum = eps;   // residual norms stepped through since the last true residual
    bool is_true = true;
    int it = 0;
    h->status = TDP_STATUS_MAX_ITERATIONS;
    while (true) {
        if (!std::isfinite(eps)) {
            h->status = TDP_STATUS_NON_FINITE;
            break;
        }
        if (eps <= h->target_eps || it >= cap || (size_t)slot + 3 >= h->nscal) {
            const bool drift_ok = eps <= h->target_eps && !h->always_true_residual &&
                                  kDriftPerStep * eps_sum <= h->target_eps - eps;
            if (!is_true && !drift_ok) {
                launch_cg_mu<R>(d, st, fused ? d.mu0 : nullptr);
                matvec<R>(h);
                launch_cg_residual<R>(d, st);
                launch_cg_p<R>(d, -1, ++slot, st);
                h->launches += 3;
                eps = read_scalar(h, d.scal_eps + slot);
                eps_sum = eps;
                is_true = true;
                continue;
            }
            if (eps <= h->target_eps) h->status = TDP_STATUS_CONVERGED;
            break;
        }
        matvec<R>(h);
        launch_cg_q(d, st);
        launch_cg_update(d, slot, st);
        launch_cg_p<R>(d, slot, slot + 1, st);
        h->launches += 3;
        slot++;
        it++;
        eps = read_scalar(h, d.scal_eps + slot);
        eps_sum += eps;
        is_true = false;
    }
    launch_cg_mu<R>(d, st);
    h->launches += 1;
    h->eps_slots = slot + 1;
    h->iterations = it;
    h->epsilon = eps;
    h->converged = (h->status == TDP_STATUS_CONVERGED) ? 1 : 0;
}

// solve_cg preconditioned by the Ewald operator of the same box
// (tdp_precond.cuh): the same start, stopping test, drift bound and
// true-residual check; every iteration first applies z = M(r) and steps along
// the flexible direction p = z + beta p.  The residual r and its stopping
// quantity are the unpreconditioned ones, so the converged dipoles are the
// same fixed point.  A cold solve starts from y = M(b), b = sqrt(alpha) E,
// instead of y = b: that costs one preconditioner application and saves about
// one outer iteration.
template <class R>
void solve_pcg(tdp_handle* h, bool fused, bool cold) {
    Dev& d = h->d;
    cudaStream_t st = h->stream;
    const int cap = h->max_iter;
    int slot = 0;
    if (fused) {
        launch_cg_residual<R>(d, st, false);
    } else {
        if (cold) {
            size_t k = kernel_begin(h, 3);
            precond_cold_start<R>(h->pre, d, st);
            kernel_end(h, k);
            h->launches += precond_last_launches(h->pre);
            h->pre_applications++;
        }
        matvec<R>(h);
        launch_cg_residual<R>(d, st);
    }
    launch_cg_p<R>(d, -1, slot, st);
    h->launches += 2;
    double eps = read_scalar(h, d.scal_eps + slot);
    double eps_sum = eps;
    bool is_true = true, first = true;
    int it = 0;
    h->status = TDP_STATUS_MAX_ITERATIONS;
    while (true) {
        if (!std::isfinite(eps)) {
            h->status = TDP_STATUS_NON_FINITE;
            break;
        }
        if (eps <= h->target_eps || it >= cap || (size_t)slot + 3 >= h->nscal) {
            const bool drift_ok = eps <= h->target_eps && !h->always_true_residual &&
                                  kDriftPerStep * eps_sum <= h->target_eps - eps;
            if (!is_true && !drift_ok) {
                launch_cg_mu<R>(d, st, fused ? d.mu0 : nullptr);
                matvec<R>(h);
                launch_cg_residual<R>(d, st);
                launch_cg_p<R>(d, -1, ++slot, st);
                h->launches += 3;
                eps = read_scalar(h, d.scal_eps + slot);
                eps_sum = eps;
                is_true = true;
                first = true;   // restart the directions from the true residual
                continue;
            }
            if (eps <= h->target_eps) h->status = TDP_STATUS_CONVERGED;
            break;
        }
        size_t k = kernel_begin(h, 3);
        precond_apply<R>(h->pre, d, slot, first, st);
        kernel_end(h, k);
        h->launches += precond_last_launches(h->pre);
        h->pre_applications++;
        matvec<R>(h);
        launch_cg_q(d, st);
        launch_cg_update(d, slot, st);
        launch_cg_p<R>(d, -1, slot + 1, st);
        h->launches += 3;
        slot++;
        it++;
        first = false;
        eps = read_scalar(h, d.scal_eps + slot);
        eps_sum += eps;
        is_true = false;
    }
    launch_cg_mu<R>(d, st);
    h->launches += 1;
    h->eps_slots = slot + 1;
    h->iterations = it;
    h->epsilon = eps;
    h->converged = (h->status == TDP_STATUS_CONVERGED) ? 1 : 0;
}

// The reference's own Jacobi loop (RTDF.cpp:820-851), sweep for sweep.
template <class R>
void solve_jacobi(tdp_handle* h) {
    Dev& d = h->d;
    cudaStream_t st = h->stream;
    double eps = 1.0;
    int it = 0;
    for (; it < h->max_iter && eps > h->target_eps; it++) {
        matvec<R>(h);
        launch_jacobi<R>(d, st);
        launch_eps_scalar(d, it, st);
        h->launches += 2;
        eps = read_scalar(h, d.scal_eps + it);
        if (!std::isfinite(eps)) break;
    }
    h->iterations = it;
    h->eps_slots = it;
    h->epsilon = eps;
    h->converged = eps < h->target_eps ? 1 : 0;
    h->status = std::isfinite(eps) ? (h->converged ? TDP_STATUS_CONVERGED : TDP_STATUS_MAX_ITERATIONS)
                                   : TDP_STATUS_NON_FINITE;
}

// Perturbation-theory extrapolation (RTDF.cpp:853-909).
template <class R>
void solve_extrapolated(tdp_handle* h) {
    Dev& d = h->d;
    cudaStream_t st = h->stream;
    int k = (int)h->extrap.size();
    TDP_CUDA(cudaMemcpyAsync(d.hist, d.mu, sizeof(double) * 3 * h->n, cudaMemcpyDeviceToDevice, st));
    for (int o = 1; o < k; o++) {
        matvec<R>(h);
        launch_extrap_step<R>(d, o, st);
        h->launches++;
    }
    launch_extrap_combine<R>(d, k, d.coef, st);
    matvec<R>(h);
    launch_step_eps(d, st);
    launch_eps_scalar(d, 0, st);
    h->launches += 3;
    h->epsilon = read_scalar(h, d.scal_eps);
    h->iterations = k;
    h->converged = 1;
    h->status = std::isfinite(h->epsilon) ? TDP_STATUS_CONVERGED : TDP_STATUS_NON_FINITE;
}

// Warm-start predictor weights, newest solution first: the polynomial of
// degree nh - 1 through the last nh solutions, evaluated one step ahead
// (binomial weights (-1)^(k) C(nh, k + 1)).
constexpr double kPredictor[kMuHist][kMuHist] = {
    {1.0, 0.0, 0.0, 0.0}, {2.0, -1.0, 0.0, 0.0}, {3.0, -3.0, 1.0, 0.0}, {4.0, -6.0, 4.0, -1.0}};

// setup (RTDF.cpp:1117-1155): rotation, permanent field, induced dipoles.
template <class R>
void setup_and_solve(tdp_handle* h) {
    Dev& d = h->d;
    cudaStream_t st = h->stream;
    h->matvecs = 0;
    h->launches = 0;
    h->kev_used = 0;
    h->pre_applications = 0;
    h->eps_slots = 0;
    if (d.fix_err) TDP_CUDA(cudaMemsetAsync(d.fix_err, 0, sizeof(int), st));
    record(h, 0);
    launch_pack<R>(d, st);
    launch_rotate<R>(d, st);
    record(h, 1);
    // A warm-started Mutual CG solve takes the fused start: one walk with the
    // operand m + mu0 gives E + T mu0 (see solve_cg).
    const bool fused = h->polarization == TDP_MUTUAL && h->solver == TDP_SOLVER_CG &&
                       (h->flags & TDP_FLAG_WARM_START) && h->n_hist > 0 && h->fused_start && d.mu0;
    h->e_shifted = false;
    if (h->ew) {
        const double L[3] = {h->box[0], h->box[4], h->box[8]};
        ewald_prepare(h->ew, d, L, h->cutoff, h->ewald_tol, h->pme_alpha, h->pme_grid, st);
        if (!fused) {
            ewald_fixed_field<R>(h->ew, d, st);
            h->launches += 3 + ewald_last_launches(h->ew);
        }
    } else if (!fused) {
        launch_field<R>(d, 0, st);
        h->launches += 4;
    }
    if (!fused) launch_fixed_done<R>(d, st);
    record(h, 2);
    if (h->polarization == TDP_DIRECT) {
        h->iterations = 0;
        h->epsilon = 1.0e50;
        h->converged = 1;
        h->status = TDP_STATUS_CONVERGED;
    } else if (h->polarization == TDP_MUTUAL) {
        if (h->solver == TDP_SOLVER_JACOBI) {
            solve_jacobi<R>(h);
        } else {
            if ((h->flags & TDP_FLAG_WARM_START) && h->n_hist > 0) {
                // Polynomial extrapolation through the last nh solutions (exact
                // for a trajectory of degree nh - 1 in time).
                const int nh = std::min(h->n_hist, h->predictor);
                launch_predict(d, nh, kPredictor[nh - 1], st);
                if (fused) {
                    TDP_CUDA(cudaMemcpyAsync(d.mu0, d.mu, sizeof(double) * 3 * h->n, cudaMemcpyDeviceToDevice, st));
                    launch_pack_total<R>(d, st);
                    size_t k = kernel_begin(h, 2);
                    if (h->ew) {
                        ewald_fixed_field<R>(h->ew, d, st, d.vec_s);
                        h->launches += ewald_last_launches(h->ew);
                    } else {
                        launch_field<R>(d, 2, st);
                        h->launches += 1 + (sizeof(R) == 4 ? 1 : 0);
                    }
                    kernel_end(h, k);
                    launch_fused_done<R>(d, st);
                    h->launches += 3;
                    h->e_shifted = true;
                } else {
                    launch_warm_start<R>(d, st);
                }
                h->launches += 1;
            }
            solve_cg<R>(h, fused, !((h->flags & TDP_FLAG_WARM_START) && h->n_hist > 0));
        }
        const bool ok = h->status == TDP_STATUS_CONVERGED;
        // The oldest buffer takes this solution and moves to the front.
        double* oldest = d.mu_hist[kMuHist - 1];
        for (int k = kMuHist - 1; k > 0; k--) d.mu_hist[k] = d.mu_hist[k - 1];
        d.mu_hist[0] = oldest;
        TDP_CUDA(cudaMemcpyAsync(d.mu_hist[0], d.mu, sizeof(double) * 3 * h->n, cudaMemcpyDeviceToDevice, st));
        h->n_hist = ok ? std::min(h->n_hist + 1, kMuHist) : 0;
    } else {
        solve_extrapolated<R>(h);
    }
    record(h, 3);
}

// calculateElectrostatic + mapTorqueToForce (RTDF.cpp:117-124).
template <class R>
void run_energy(tdp_handle* h) {
    Dev& d = h->d;
    cudaStream_t st = h->stream;
    if (h->ew) {
        size_t k = kernel_begin(h, 1);
        ewald_energy<R>(h->ew, d, h->total_charge, st, h->polarization == TDP_DIRECT);
        kernel_end(h, k);
        h->launches += ewald_last_launches(h->ew);
        record(h, 4);
        launch_torque_gather(d, st);
        record(h, 5);
        h->launches += 1;
        return;
    }
    launch_pack_ind<R>(d, st);
    size_t k = kernel_begin(h, 1);
    launch_energy<R>(d, st);
    kernel_end(h, k);
    launch_energy_done(d, st);
    record(h, 4);
    launch_torque_gather(d, st);
    record(h, 5);
    h->launches += 4;
}

void finish_timing(tdp_handle* h) {
    if (!h->timing) return;
    TDP_CUDA(cudaEventSynchronize(h->ev[5]));
    float ms;
    for (int k = 0; k < 5; k++) {
        TDP_CUDA(cudaEventElapsedTime(&ms, h->ev[k], h->ev[k + 1]));
        h->stage_ms[k] = ms;
    }
    TDP_CUDA(cudaEventElapsedTime(&ms, h->ev[0], h->ev[5]));
    h->stage_ms[5] = ms;
    h->stage_ms[6] = h->matvecs;
    double mv = 0.0, en = 0.0, fu = 0.0, pc = 0.0;
    int nfu = 0;
    for (size_t k = 0; k < h->kev_used; k++) {
        TDP_CUDA(cudaEventElapsedTime(&ms, h->kev[2 * k], h->kev[2 * k + 1]));
        if (h->kev_kind[k] == 0) mv += ms;
        else if (h->kev_kind[k] == 1) en += ms;
        else if (h->kev_kind[k] == 3) pc += ms;
        else {
            fu += ms;
            nfu++;
        }
    }
    h->stage_ms[12] = h->pre_applications;
    h->stage_ms[13] = pc;
    h->stage_ms[7] = mv;
    h->stage_ms[8] = en;
    h->stage_ms[9] = (double)h->launches;
    h->stage_ms[10] = nfu;
    h->stage_ms[11] = fu;
}

// Device-side failure flags of the last evaluation: enqueue their readback
// before the stream is synchronised, check them after.
void enqueue_flags(tdp_handle* h) {
    if (h->d.fix_err)
        TDP_CUDA(cudaMemcpyAsync(h->h_fixerr, h->d.fix_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
}
void check_flags(tdp_handle* h) {
    if (h->ew && ewald_list_overflow(h->ew))
        throw TdpError{TDP_ERR_CUDA, "Ewald mode: a neighbour-tile list row overflowed its capacity"};
    if (h->pre && precond_list_overflow(h->pre))
        throw TdpError{TDP_ERR_CUDA, "CG preconditioner: a neighbour-tile list row overflowed its capacity"};
    if (h->d.fix_err && *h->h_fixerr)
        throw TdpError{TDP_ERR_NON_FINITE,
                       "a field or force sum is not finite or exceeds the fixed-point accumulator range "
                       "(2^23 per band sum; near-coincident particles?)"};
}

// positions == &kStaged: the coordinates are already in d.pos.
const char kStaged = 0;

void solve_at(tdp_handle* h, const void* positions, int dtype, int on_device) {
    if (positions) {
        check_box(h);
        if (positions != &kStaged) stage_positions(h, positions, dtype, on_device);
        if (!h->sorted || ++h->since_sort >= h->resort_interval) sort_atoms(h);
        if (h->precision == TDP_PRECISION_DOUBLE) setup_and_solve<double>(h);
        else setup_and_solve<float>(h);
        h->have_results = true;
    } else if (!h->have_results) {
        throw TdpError{TDP_ERR_INVALID_ARGUMENT, "no positions given and no previous evaluation"};
    }
}

// Reverse mode of one evaluation (tdp_adjoint.cu has the kernels and the
// derivation).  Needs the state of the last evaluation (positions, lab-frame
// and induced dipoles, permanent field); leaves it as it was.
template <class R>
void run_adjoint(tdp_handle* h, const double* g_in, double gE, double* out_dst, bool on_device) {
    Dev& d = h->d;
    cudaStream_t st = h->stream;
    const int n = h->n;
    const size_t n3 = 3 * (size_t)n;
    if (!h->adj) h->adj = dalloc<double>(n3 * 11 + 8 * (size_t)n + 5 * (size_t)n + 2 * (size_t)n + 6 * (size_t)n +
                                             adjoint_pair_scratch(n) + adjoint_fixed_scratch(n),
                                         h->owned);
    double* g = h->adj;
    double* gt = g + n3;
    double* amu = gt + n3;
    double* lam = amu + n3;
    double* glab = lam + n3;
    double* gmol = glab + n3;
    double* mu_fwd = gmol + n3;
    double* E_fwd = mu_fwd + n3;
    double* amu_tlam = E_fwd + n3;
    double* e_tmu = amu_tlam + n3;
    double* a8 = e_tmu + n3;
    double* b5 = a8 + 8 * (size_t)n;
    double* ct = b5 + 5 * (size_t)n;
    double* out = ct + n;
    double* ext_v = out + 6 * (size_t)n;   // Extrapolated: E + T mu_(k-1)
    double* galpha = ext_v + n3;           // Extrapolated: polarizability gradient
    double* pair_scratch = galpha + n;     // split sums and damped-partner lists of the pair VJP
    double* fixed_scratch = pair_scratch + adjoint_pair_scratch(n);   // split sums of the fixed-field VJP
    if (g_in)
        TDP_CUDA(cudaMemcpyAsync(g, g_in, n3 * 8, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    else
        TDP_CUDA(cudaMemsetAsync(g, 0, n3 * 8, st));
    TDP_CUDA(cudaMemcpyAsync(mu_fwd, d.mu, n3 * 8, cudaMemcpyDeviceToDevice, st));
    TDP_CUDA(cudaMemcpyAsync(E_fwd, d.E, n3 * 8, cudaMemcpyDeviceToDevice, st));
    launch_torque_vjp(d, g, gt, st);
    AdjPairList plist;
    launch_adjoint_pair(d, g, gt, gE, a8, h->precision, pair_scratch, &plist, st);
    launch_adjoint_split(d, a8, nullptr, amu, nullptr, st);
    if (h->polarization == TDP_MUTUAL) {
        // One solve of the same symmetric system: A lambda = a_mu.  Target:
        // 1e-12 (FP64 form) or 1e-6 (mixed form, whose true residual is
        // itself limited by the FP32 matvec near 1e-7) of the RMS of
        // alpha * a_mu (the solver's Jacobi-step units).
        double* ps = pstat(h);
        k_alpha_norm2<<<1, 1024, 0, st>>>(n, d.alpha, amu, ps);
        const double s2 = read_scalar(h, ps);
        double rms = std::sqrt(s2 / std::max(n, 1));
        int it0 = h->iterations, conv0 = h->converged, st0 = h->status, mv0 = h->matvecs;
        double eps0 = h->epsilon, tgt0 = h->target_eps;
        int cap0 = h->max_iter;
        h->target_eps = std::max(rms * (h->precision == TDP_PRECISION_DOUBLE ? 1e-12 : 1e-6), 1e-300);
        h->max_iter = std::max(cap0, 1000);
        launch_rhs_init<R>(d, amu, st);
        solve_cg<R>(h);
        h->adj_eps = h->epsilon;
        h->adj_iterations = h->iterations;
        h->iterations = it0;
        h->converged = conv0;
        h->status = st0;
        h->epsilon = eps0;
        h->matvecs = mv0;
        h->target_eps = tgt0;
        h->max_iter = cap0;
        TDP_CUDA(cudaMemcpyAsync(lam, d.mu, n3 * 8, cudaMemcpyDeviceToDevice, st));
        TDP_CUDA(cudaMemcpyAsync(d.mu, mu_fwd, n3 * 8, cudaMemcpyDeviceToDevice, st));
        TDP_CUDA(cudaMemcpyAsync(d.E, E_fwd, n3 * 8, cudaMemcpyDeviceToDevice, st));
        launch_adjoint_fixed(d, lam, b5, plist, h->precision, fixed_scratch, st);
        launch_adjoint_matvec_t(d, lam, ct, plist, st);
        launch_set_operand<R>(d, lam, st);
        launch_field<R>(d, 1, st);
        launch_add_field(d, amu, amu_tlam, st);
        if (h->e_shifted) {
            // E_fwd holds E + T mu0: E + T mu = E_fwd + T (mu - mu0) (glab as scratch).
            launch_lincomb(n, 1.0, mu_fwd, -1.0, d.mu0, glab, st);
            launch_set_operand<R>(d, glab, st);
        } else {
            launch_set_operand<R>(d, mu_fwd, st);
        }
        launch_field<R>(d, 1, st);
        launch_add_field(d, E_fwd, e_tmu, st);
    } else if (h->polarization == TDP_EXTRAPOLATED) {
        // The extrapolation recursion backwards (see tdp_adjoint.cu): gbar in
        // amu_tlam, alpha gbar in e_tmu; lambda, dL/dalpha and c_t accumulate.
        const int K = (int)h->extrap.size();
        double* gbar = amu_tlam;
        double* agb = e_tmu;
        TDP_CUDA(cudaMemsetAsync(lam, 0, n3 * 8, st));
        TDP_CUDA(cudaMemsetAsync(galpha, 0, sizeof(double) * n, st));
        TDP_CUDA(cudaMemsetAsync(ct, 0, sizeof(double) * n, st));
        launch_lincomb(n, h->extrap[K - 1], amu, 0.0, nullptr, gbar, st);
        for (int o = K - 1; o >= 0; o--) {
            const double* mu_prev = d.hist + (size_t)(o - 1) * n3;
            launch_alpha_scale(d, gbar, agb, st);
            launch_lincomb(n, 1.0, lam, 1.0, agb, lam, st);
            if (o == 0) {
                launch_dot3_acc(n, gbar, E_fwd, galpha, st);
                break;
            }
            launch_set_operand<R>(d, mu_prev, st);
            launch_field<R>(d, 1, st);
            launch_add_field(d, E_fwd, ext_v, st);
            launch_dot3_acc(n, gbar, ext_v, galpha, st);
            launch_adjoint_matvec_t_mu(d, agb, mu_prev, ct, true, plist, st);
            launch_set_operand<R>(d, agb, st);
            launch_field<R>(d, 1, st);
            launch_lincomb(n, h->extrap[o - 1], amu, 0.0, nullptr, ext_v, st);
            launch_add_field(d, ext_v, gbar, st);
        }
        launch_adjoint_fixed(d, lam, b5, plist, h->precision, fixed_scratch, st);
        h->adj_eps = 0.0;
        h->adj_iterations = 0;
    } else {
        // Direct: mu = alpha E, so lambda = alpha a_mu and dL/dalpha = a_mu . E.
        k_alpha_scale<<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(n, d.alpha, amu, lam);
        launch_adjoint_fixed(d, lam, b5, plist, h->precision, fixed_scratch, st);
        TDP_CUDA(cudaMemsetAsync(ct, 0, sizeof(double) * n, st));
        TDP_CUDA(cudaMemcpyAsync(amu_tlam, amu, n3 * 8, cudaMemcpyDeviceToDevice, st));
        TDP_CUDA(cudaMemcpyAsync(e_tmu, E_fwd, n3 * 8, cudaMemcpyDeviceToDevice, st));
        h->adj_eps = 0.0;
        h->adj_iterations = 0;
    }
    launch_adjoint_split(d, a8, b5, amu, glab, st);
    launch_rotation_vjp(d, glab, gmol, st);
    launch_adjoint_assemble(d, a8, b5, ct, amu_tlam, e_tmu, gmol, out, st,
                            h->polarization == TDP_EXTRAPOLATED ? galpha : nullptr);
    TDP_CUDA(cudaMemcpyAsync(out_dst, out, sizeof(double) * 6 * n,
                             on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
    if (!on_device) TDP_CUDA(cudaStreamSynchronize(st));
    TDP_CUDA(cudaGetLastError());
}

int adjoint_entry(tdp_handle* h, const double* dL_dF, double dL_dE, double* grads, bool on_device) {
    if (!h || !grads) return TDP_ERR_INVALID_ARGUMENT;
    try {
        if (h->n == 0) return TDP_OK;
        if (!h->have_results) throw TdpError{TDP_ERR_INVALID_ARGUMENT, "tdp_adjoint needs a previous tdp_compute"};
        if (h->ew) throw TdpError{TDP_ERR_UNSUPPORTED, "tdp_adjoint does not support the Ewald mode"};
        if (h->precision == TDP_PRECISION_DOUBLE) run_adjoint<double>(h, dL_dF, dL_dE, grads, on_device);
        else run_adjoint<float>(h, dL_dF, dL_dE, grads, on_device);
    } catch (const TdpError& e) {
        return fail(h, e);
    }
    return TDP_OK;
}

}  // namespace

extern "C" {

int tdp_adjoint(tdp_handle* h, const double* dL_dF, double dL_dE, double* grads) {
    return adjoint_entry(h, dL_dF, dL_dE, grads, false);
}

int tdp_adjoint_device(tdp_handle* h, const double* dL_dF, double dL_dE, double* grads) {
    return adjoint_entry(h, dL_dF, dL_dE, grads, true);
}

int tdp_abi_version(void) { return TDP_ABI_VERSION; }

const char* tdp_last_error(const tdp_handle* h) {
    if (h) return h->err.c_str();
    const char* na = noalloc_error_message();
    return na[0] ? na : g_create_error.c_str();
}

int tdp_create(const tdp_system_desc* desc, tdp_handle** out) {
    if (!out) return TDP_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    tdp_handle* h = new tdp_handle();
    try {
        if (!desc) throw TdpError{TDP_ERR_INVALID_ARGUMENT, "desc is NULL"};
        int n = desc->num_particles;
        if (n < 0) throw TdpError{TDP_ERR_INVALID_ARGUMENT, "num_particles < 0"};
        if (n > 0 && (!desc->charges || !desc->molecular_dipoles || !desc->polarizabilities ||
                      !desc->thole_damping || !desc->axis_types || !desc->atom_z || !desc->atom_x || !desc->atom_y))
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, "a per-particle array is NULL"};
        if (desc->nonbonded_method < 0 || desc->nonbonded_method > 1)
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, "TholeDipoleForce: Illegal value for nonbonded method"};
        if (desc->polarization_type < 0 || desc->polarization_type > 2)
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, "Polarization type not recognized."};
        if (desc->precision != TDP_PRECISION_MIXED && desc->precision != TDP_PRECISION_DOUBLE)
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, "unknown precision"};
        if (desc->solver != TDP_SOLVER_CG && desc->solver != TDP_SOLVER_JACOBI)
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, "unknown solver"};
        validate_axes(n, desc->axis_types, desc->atom_z, desc->atom_x, desc->atom_y);

        h->n = n;
        h->method = desc->nonbonded_method;
        h->polarization = desc->polarization_type;
        h->precision = desc->precision;
        h->solver = desc->solver;
        h->flags = desc->flags;
        h->cutoff = desc->cutoff;
        h->ewald_tol = desc->ewald_error_tolerance;
        h->pme_alpha = desc->pme_alpha;
        for (int k = 0; k < 3; k++) h->pme_grid[k] = desc->pme_grid[k];
        h->target_eps = desc->mutual_target_epsilon;
        h->max_iter = std::max(0, desc->mutual_max_iterations);
        if (desc->num_extrapolation_coefficients > 0 && desc->extrapolation_coefficients)
            h->extrap.assign(desc->extrapolation_coefficients,
                             desc->extrapolation_coefficients + desc->num_extrapolation_coefficients);
        else
            h->extrap = {-0.154, 0.017, 0.658, 0.474};  // RTDF.cpp:857-864
        h->charge.assign(desc->charges, desc->charges + n);
        h->dip.assign(desc->molecular_dipoles, desc->molecular_dipoles + 3 * (size_t)n);
        h->alpha.assign(desc->polarizabilities, desc->polarizabilities + n);
        h->thole.assign(desc->thole_damping, desc->thole_damping + n);
        h->axis.resize(4 * (size_t)n);
        for (int i = 0; i < n; i++) {
            h->axis[4 * i] = desc->axis_types[i];
            h->axis[4 * i + 1] = desc->atom_z[i];
            h->axis[4 * i + 2] = desc->atom_x[i];
            h->axis[4 * i + 3] = desc->atom_y[i];
        }

        std::vector<std::vector<std::tuple<int, double, double>>>& exc = h->exc_user;
        exc = covalent_exceptions(n, desc->covalent12_offsets, desc->covalent12_atoms, desc->covalent13_offsets,
                                  desc->covalent13_atoms);
        // Launch geometry of the pair kernels: 32-atom tiles in bands of
        // band_tiles tiles, one CTA per band pair.  Bands are as wide as
        // possible -- 16 tiles (8 in FP64, whose records and sums are twice as
        // large) so that four CTAs' J records and sums fit one SM's shared
        // memory -- while still giving about 16 CTAs per SM.
        Dev& d = h->d;
        const int nt = std::max(1, (n + kTile - 1) / kTile);
        const int widest = h->precision == TDP_PRECISION_DOUBLE ? 8 : 16;
        int band = 1;
        for (int cand : {16, 8, 4, 2}) {
            if (cand > widest) continue;
            long nb = (nt + cand - 1) / cand;
            if (nb * (nb + 1) / 2 >= 16L * 148) {
                band = cand;
                break;
            }
        }
        if (const char* e = getenv("TDP_BAND_TILES")) {
            int v = atoi(e);
            if ((v == 1 || v == 2 || v == 4 || v == 8 || v == 16) && v <= widest) band = v;
        }
        const int pad = kTile * std::max(4, band);
        d.n = n;
        d.n_pad = std::max(pad, ((n + pad - 1) / pad) * pad);
        d.nvb = std::max(1, (n + kVecThreads - 1) / kVecThreads);
        d.pp.band_tiles = band;
        d.pp.n_bands = (nt + band - 1) / band;
        d.nsplit = d.pp.n_bands;
        d.n_eblk = d.pp.n_bands * (d.pp.n_bands + 1) / 2;
        const bool variational = (h->flags & TDP_FLAG_VARIATIONAL) != 0;
        // Both gradient modes rest on an energy functional that is stationary
        // in the induced dipoles: Mutual (mu = alpha (E + T mu)) and Direct
        // (mu = alpha E, the functional without the induced-induced term)
        // have one; the Extrapolated dipoles minimise none.
        if ((h->flags & (TDP_FLAG_VARIATIONAL | TDP_FLAG_EWALD)) && h->polarization == TDP_EXTRAPOLATED)
            throw TdpError{TDP_ERR_UNSUPPORTED,
                           "TDP_FLAG_EWALD and TDP_FLAG_VARIATIONAL need Mutual or Direct polarization (their forces "
                           "are the gradient of an energy that is stationary in the induced dipoles)"};
        if (variational) {
            if (h->method != TDP_NO_CUTOFF)
                throw TdpError{TDP_ERR_INVALID_ARGUMENT,
                               "TDP_FLAG_VARIATIONAL is the NoCutoff mode; PME systems use TDP_FLAG_EWALD"};
            if (h->flags & TDP_FLAG_EWALD)
                throw TdpError{TDP_ERR_INVALID_ARGUMENT, "TDP_FLAG_VARIATIONAL and TDP_FLAG_EWALD exclude each other"};
            // Real space only: one partial slot.
            d.nsplit = 1;
            d.n_eblk = 1;
        }
        const bool ewald = (h->flags & TDP_FLAG_EWALD) != 0;
        if (ewald) {
            if (h->method != TDP_PME)
                throw TdpError{TDP_ERR_INVALID_ARGUMENT, "TDP_FLAG_EWALD needs the PME nonbonded method"};
            if (!(h->cutoff > 0.0)) throw TdpError{TDP_ERR_INVALID_ARGUMENT, "the Ewald mode needs a cutoff > 0"};
            if (!(h->ewald_tol > 0.0 && h->ewald_tol < 0.5) && !(h->pme_alpha > 0.0))
                throw TdpError{TDP_ERR_INVALID_ARGUMENT, "the Ewald error tolerance must lie in (0, 0.5)"};
            // Real space stops at the cutoff, damping corrections included: the
            // least-damped pair at the cutoff (a u^3 = rc^3 / t_max^5) must have
            // exp(-a u^3) <= 1e-12.
            double tmax = 0.0;
            bool bad = false;
            for (double t : h->thole) {
                if (!(t >= 0.0)) bad = true;
                tmax = std::max(tmax, t);
            }
            if (bad || (tmax > 0.0 && h->cutoff * h->cutoff * h->cutoff < 27.631021115928547 * std::pow(tmax, 5.0)))
                throw TdpError{TDP_ERR_INVALID_ARGUMENT,
                               "Ewald mode: the Thole damping at the cutoff exceeds 1e-12 (cutoff too short for the "
                               "largest Thole factor)"};
            // Real space in partial slot 0, reciprocal space + self in slot 1.
            d.nsplit = 2;
            d.n_eblk = 1;
        } else if (h->precision == TDP_PRECISION_MIXED && !variational) {
            // Mixed all-pairs form: the band sums go into the fixed-point
            // accumulator and one flushed slot.  Each atom's word receives at
            // most 2 n_bands adds of magnitude < 2^23, so with 2^bits units
            // per e/nm^2 the sum stays below 2^61.
            d.nsplit = 1;
            int lg = 0;
            while ((1L << lg) < 2L * std::max(1, d.pp.n_bands)) lg++;
            const int bits = std::min(32, 38 - lg);
            d.fix_scale = std::ldexp(1.0, bits);
            d.fix_limit = std::ldexp(1.0, 23);
        }

        std::vector<int> eoff(n + 1, 0), ej;
        std::vector<double> em, es;
        std::vector<int2> etiles(d.n_pad / kTile, make_int2(1 << 30, -1));  // empty range
        for (int i = 0; i < n; i++) {
            for (auto& t : exc[i]) {
                int j = std::get<0>(t);
                ej.push_back(j);
                em.push_back(std::get<1>(t));
                es.push_back(std::get<2>(t));
                int2& r = etiles[i / kTile];
                r.x = std::min(r.x, j / kTile);
                r.y = std::max(r.y, j / kTile);
            }
            eoff[i + 1] = (int)ej.size();
        }

        d.pp.n = n;
        d.pp.n_tiles = (n + kTile - 1) / kTile;
        d.pp.mutual = h->polarization == TDP_MUTUAL ? 1 : 0;
        d.pp.rinv4_power = (h->flags & TDP_FLAG_DD_FORCE_R4) ? 1.0f : 0.0f;
        d.pp.rinv4_fill = 0.0f;
        // The lab-frame energy walk needs rInvVec[4] = 0; TDP_LAB_ENERGY=0
        // keeps every tile pair on the general walk (for comparisons).
        d.pp.lab_energy = (h->flags & TDP_FLAG_DD_FORCE_R4) ? 0 : 1;
        if (const char* e = getenv("TDP_LAB_ENERGY"))
            if (atoi(e) == 0) d.pp.lab_energy = 0;

        size_t rsz = h->precision == TDP_PRECISION_DOUBLE ? sizeof(double4) : sizeof(float4);
        auto& o = h->owned;
        d.pos = dalloc<double>(3 * (size_t)d.n_pad, o);
        d.charge = dalloc<double>(n, o);
        d.dip_mol = dalloc<double>(3 * (size_t)n, o);
        d.alpha = dalloc<double>(n, o);
        d.salpha = dalloc<double>(n, o);
        d.thole = dalloc<double>(n, o);
        d.axis = dalloc<int4>(n, o);
        d.posq = dalloc<char>(rsz * d.n_pad, o);
        d.dipt = dalloc<char>(rsz * d.n_pad, o);
        d.ind = dalloc<char>(rsz * d.n_pad, o);
        d.yz = dalloc<double2>(d.n_pad, o);
        d.tctr = dalloc<double4>(d.n_pad / kTile, o);
        d.text = dalloc<double4>(d.n_pad / kTile, o);
        d.exc_off = dalloc<int>(n + 1, o);
        d.exc_j = dalloc<int>(ej.size(), o);
        d.exc_m = dalloc<double>(em.size(), o);
        d.exc_s = dalloc<double>(es.size(), o);
        d.exc_tiles = dalloc<int2>(etiles.size(), o);
        d.users_off = dalloc<int>(n + 1, o);
        size_t n3 = 3 * (size_t)n;
        d.lab = dalloc<double>(n3, o);
        d.E = dalloc<double>(n3, o);
        d.mu = dalloc<double>(n3, o);
        for (int k = 0; k < kMuHist; k++) d.mu_hist[k] = dalloc<double>(n3, o);
        d.mu0 = dalloc<double>(n3, o);
        d.y = dalloc<double>(n3, o);
        d.r = dalloc<double>(n3, o);
        d.p = dalloc<double>(n3, o);
        d.q = dalloc<double>(n3, o);
        d.hist = dalloc<double>(n3 * h->extrap.size(), o);
        d.partial = dalloc<double>((size_t)d.nsplit * 6 * d.n_pad, o);
        if (d.fix_scale > 0.0) {
            d.fixacc = dalloc<unsigned long long>(6 * (size_t)d.n_pad, o);
            d.fix_err = dalloc<int>(1, o);
        }
        d.energy_partial = dalloc<double>((size_t)d.n_eblk, o);
        d.fpair = dalloc<double>(n3, o);
        d.torque = dalloc<double>(n3, o);
        d.ftotal = dalloc<double>(n3, o);
        d.energy = dalloc<double>(1, o);
        d.rr_part = dalloc<double>(d.nvb, o);
        d.eps_part = dalloc<double>(d.nvb, o);
        d.pq_part = dalloc<double>(d.nvb, o);
        // CG uses one slot per iteration plus one per true-residual check.
        h->nscal = 2 * (size_t)std::max(h->max_iter, 0) + 64;
        size_t nscal = h->nscal;
        d.scal_rr = dalloc<double>(nscal, o);
        d.scal_eps = dalloc<double>(nscal, o);
        d.coef = dalloc<double>(h->extrap.size(), o);
        h->stage_bytes = std::max<size_t>(n3 * sizeof(double), 64 * sizeof(double));
        h->d_stage = dalloc<double>(h->stage_bytes / sizeof(double), o);
        upload(d.exc_off, eoff.data(), sizeof(int) * (n + 1));
        upload(d.exc_j, ej.data(), sizeof(int) * ej.size());
        upload(d.exc_m, em.data(), sizeof(double) * em.size());
        upload(d.exc_s, es.data(), sizeof(double) * es.size());
        upload(d.exc_tiles, etiles.data(), sizeof(int2) * etiles.size());
        h->n_exc = ej.size();
        build_components(h, desc);
        if (const char* e = getenv("TDP_RESORT_INTERVAL")) h->resort_interval = std::max(1, atoi(e));
        if (const char* e = getenv("TDP_FUSED_START"))
            if (atoi(e) == 0) h->fused_start = false;
        if (const char* e = getenv("TDP_PREDICTOR")) h->predictor = std::min(std::max(atoi(e), 1), kMuHist);
        if (const char* e = getenv("TDP_TRUE_RESIDUAL"))
            if (atoi(e) == 1) h->always_true_residual = true;
        d.order = dalloc<int>(d.n_pad, o);
        d.rank = dalloc<int>(n, o);
        d.pos_s = dalloc<double>(3 * (size_t)d.n_pad, o);
        d.posq_s = dalloc<char>(rsz * d.n_pad, o);
        d.dipt_s = dalloc<char>(rsz * d.n_pad, o);
        d.vec_s = dalloc<char>(rsz * d.n_pad, o);
        d.tctr_s = dalloc<double4>(d.n_pad / kTile, o);
        d.text_s = dalloc<double4>(d.n_pad / kTile, o);
        d.exs_off = dalloc<int>(n + 1, o);
        d.exs_j = dalloc<int>(ej.size(), o);
        d.exs_m = dalloc<double>(em.size(), o);
        d.exs_s = dalloc<double>(es.size(), o);
        d.exs_tiles = dalloc<int2>(d.n_pad / kTile, o);
        upload(d.coef, h->extrap.data(), sizeof(double) * h->extrap.size());
        upload_params(h);
        if (ewald || variational)
            h->ew = ewald_create(d, h->precision, variational, h->polarization == TDP_DIRECT);
        // Minimum-image Mutual CG: preconditioned by the Ewald operator of the
        // same box (tdp_precond.cuh).  Its real space stops at 0.6 nm or where
        // the Thole damping of every pair is below 1e-12, whichever is longer;
        // PME tolerance 1e-3; three inner iterations per application.
        // It pays from about 30,000 atoms on (an all-pairs matvec grows as
        // n^2, an application as n; measured on water boxes: 7 % slower at
        // 12,288 atoms, even at 24,000, 1.25-1.5x faster at 41,472), so by
        // default it is used from kPrecondMinAtoms atoms.  TDP_PRECOND=1 at
        // create uses it at any size, TDP_PRECOND=0 never; TDP_PRECOND_INNER
        // sets the inner iterations (1-8).
        constexpr int kPrecondMinAtoms = 32768;
        bool want_pre = h->method == TDP_PME && !ewald && h->polarization == TDP_MUTUAL &&
                        h->solver == TDP_SOLVER_CG && n >= kPrecondMinAtoms;
        if (const char* e = getenv("TDP_PRECOND"))
            want_pre = atoi(e) != 0 && h->method == TDP_PME && !ewald && h->polarization == TDP_MUTUAL &&
                       h->solver == TDP_SOLVER_CG && n > 0;
        if (want_pre) {
            double tmax = 0.0;
            for (double t : h->thole) tmax = std::max(tmax, std::isfinite(t) ? t : 0.0);
            const double rc = std::max(0.6, 1.001 * std::cbrt(27.631021115928547 * std::pow(tmax, 5.0)));
            int inner = 3;
            if (const char* e = getenv("TDP_PRECOND_INNER")) inner = std::min(std::max(atoi(e), 1), 8);
            d.scal_a = dalloc<double>(nscal, o);
            h->pre = precond_create(d, h->precision, rc, 1e-3, inner);
        }
        TDP_CUDA(cudaMallocHost(&h->h_scal, 64 * sizeof(double)));
        TDP_CUDA(cudaMallocHost(&h->h_fixerr, sizeof(int)));
        *h->h_fixerr = 0;
        TDP_CUDA(cudaMallocHost(&h->h_forces, std::max<size_t>(n3, 1) * sizeof(double)));
        for (int k = 0; k < 6; k++) TDP_CUDA(cudaEventCreate(&h->ev[k]));
        refresh_box(h);
        TDP_CUDA(cudaDeviceSynchronize());
    } catch (const TdpError& e) {
        int code = fail(nullptr, e);
        tdp_destroy(h);
        return code;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        noalloc_clear_error();
        tdp_destroy(h);
        return TDP_ERR_INVALID_ARGUMENT;
    }
    *out = h;
    return TDP_OK;
}

void tdp_destroy(tdp_handle* h) {
    if (!h) return;
    if (h->ew) ewald_destroy(h->ew);
    if (h->pre) precond_destroy(h->pre);
    for (void* p : h->owned) cudaFree(p);
    if (h->h_scal) cudaFreeHost(h->h_scal);
    if (h->h_fixerr) cudaFreeHost(h->h_fixerr);
    if (h->h_forces) cudaFreeHost(h->h_forces);
    for (int k = 0; k < 6; k++)
        if (h->ev[k]) cudaEventDestroy(h->ev[k]);
    for (cudaEvent_t e : h->kev) cudaEventDestroy(e);
    delete h;
}

int tdp_set_stream(tdp_handle* h, void* stream) {
    if (!h) return TDP_ERR_INVALID_ARGUMENT;
    h->stream = static_cast<cudaStream_t>(stream);
    return TDP_OK;
}

int tdp_set_box(tdp_handle* h, const double* box9) {
    if (!h || !box9) return TDP_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 9; k++) h->box[k] = box9[k];
    h->have_box = true;
    refresh_box(h);
    return TDP_OK;
}

int tdp_update_params(tdp_handle* h, int32_t num_particles, const double* charges, const double* molecular_dipoles,
                      const double* polarizabilities, const double* thole_damping, const int32_t* axis_types,
                      const int32_t* atom_z, const int32_t* atom_x, const int32_t* atom_y) {
    if (!h) return TDP_ERR_INVALID_ARGUMENT;
    try {
        if (num_particles != h->n)
            throw TdpError{TDP_ERR_SIZE_MISMATCH, "updateParametersInContext: The number of particles has changed"};
        int n = h->n;
        if (n > 0 && (!charges || !molecular_dipoles || !polarizabilities || !thole_damping || !axis_types ||
                      !atom_z || !atom_x || !atom_y))
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, "a per-particle array is NULL"};
        validate_axes(n, axis_types, atom_z, atom_x, atom_y);
        h->charge.assign(charges, charges + n);
        h->dip.assign(molecular_dipoles, molecular_dipoles + 3 * (size_t)n);
        h->alpha.assign(polarizabilities, polarizabilities + n);
        h->thole.assign(thole_damping, thole_damping + n);
        for (int i = 0; i < n; i++) {
            h->axis[4 * i] = axis_types[i];
            h->axis[4 * i + 1] = atom_z[i];
            h->axis[4 * i + 2] = atom_x[i];
            h->axis[4 * i + 3] = atom_y[i];
        }
        TDP_CUDA(cudaStreamSynchronize(h->stream));
        upload_params(h);
        h->n_hist = 0;
        h->have_results = false;
    } catch (const TdpError& e) {
        return fail(h, e);
    }
    return TDP_OK;
}

int tdp_update_particle_params(tdp_handle* h, const double* charges, const double* molecular_dipoles,
                               const double* polarizabilities, const double* thole_damping, int32_t on_device) {
    if (!h) return TDP_ERR_INVALID_ARGUMENT;
    try {
        const int n = h->n;
        if (n == 0) return TDP_OK;
        if (!charges || !molecular_dipoles || !polarizabilities || !thole_damping)
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, "a per-particle array is NULL"};
        if (!on_device) {
            h->charge.assign(charges, charges + n);
            h->dip.assign(molecular_dipoles, molecular_dipoles + 3 * (size_t)n);
            h->alpha.assign(polarizabilities, polarizabilities + n);
            h->thole.assign(thole_damping, thole_damping + n);
            TDP_CUDA(cudaStreamSynchronize(h->stream));
            upload_params(h);
        } else {
            // Device to device, then the derived quantities on the device; only
            // three scalars come back (damping radius, net charge).
            Dev& d = h->d;
            cudaStream_t st = h->stream;
            TDP_CUDA(cudaMemcpyAsync(d.charge, charges, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
            TDP_CUDA(cudaMemcpyAsync(d.dip_mol, molecular_dipoles, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice,
                                     st));
            TDP_CUDA(cudaMemcpyAsync(d.alpha, polarizabilities, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
            TDP_CUDA(cudaMemcpyAsync(d.thole, thole_damping, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
            double* ps = pstat(h);
            k_param_stats<<<1, 1024, 0, st>>>(n, h->precision == TDP_PRECISION_DOUBLE ? 0 : 1, d.alpha, d.thole,
                                              d.charge, d.salpha, ps);
            TDP_CUDA(cudaMemcpyAsync(h->h_scal + 8, ps, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
            TDP_CUDA(cudaStreamSynchronize(st));
            TDP_CUDA(cudaGetLastError());
            const double tmax = h->h_scal[8];
            double r2 = 0.0;
            if (h->h_scal[9] != 0.0) r2 = INFINITY;
            else if (tmax > 0.0) {
                const double r = std::pow(tmax, 5.0 / 3.0) * std::cbrt(50.0) * 1.001;
                r2 = r * r;
            }
            d.pp.damp_r2 = (float)r2;
            h->total_charge = h->h_scal[10];
            // The host copies no longer hold these parameters; a later
            // tdp_update_params replaces them all.
            h->charge.clear();
            h->dip.clear();
            h->alpha.clear();
            h->thole.clear();
        }
        h->n_hist = 0;
        h->have_results = false;
    } catch (const TdpError& e) {
        return fail(h, e);
    }
    return TDP_OK;
}

int tdp_compute(tdp_handle* h, const void* positions, int32_t pos_dtype, int32_t on_device, void* forces_accum,
                int32_t force_dtype, double* energy, uint32_t flags) {
    if (!h) return TDP_ERR_INVALID_ARGUMENT;
    try {
        if (h->n == 0) {
            if (energy) *energy = 0.0;
            h->iterations = 0;
            h->converged = 1;
            return TDP_OK;
        }
        if ((flags & TDP_COMPUTE_FORCES) && !forces_accum)
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, "forces requested but forces_accum is NULL"};
        if ((flags & TDP_COMPUTE_FORCES) && force_dtype != TDP_F64 && force_dtype != TDP_F32)
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, "unknown force dtype"};
        solve_at(h, positions, pos_dtype, on_device);
        if (h->precision == TDP_PRECISION_DOUBLE) run_energy<double>(h);
        else run_energy<float>(h);
        cudaStream_t st = h->stream;
        size_t n3 = 3 * (size_t)h->n;
        if (flags & TDP_COMPUTE_FORCES) {
            if (on_device) {
                launch_add_forces(h->d, forces_accum, force_dtype == TDP_F32, st);
                h->launches++;
            } else {
                TDP_CUDA(cudaMemcpyAsync(h->h_forces, h->d.ftotal, n3 * sizeof(double), cudaMemcpyDeviceToHost, st));
            }
        }
        if (energy) TDP_CUDA(cudaMemcpyAsync(h->h_scal + 1, h->d.energy, sizeof(double), cudaMemcpyDeviceToHost, st));
        enqueue_flags(h);
        TDP_CUDA(cudaStreamSynchronize(st));
        TDP_CUDA(cudaGetLastError());
        if ((flags & TDP_COMPUTE_FORCES) && !on_device) {
            if (force_dtype == TDP_F64) {
                double* acc = static_cast<double*>(forces_accum);
                for (size_t k = 0; k < n3; k++) acc[k] += h->h_forces[k];
            } else {
                float* acc = static_cast<float*>(forces_accum);
                for (size_t k = 0; k < n3; k++) acc[k] += (float)h->h_forces[k];
            }
        }
        check_flags(h);
        if (energy) *energy = h->h_scal[1];
        finish_timing(h);
        if (h->status == TDP_STATUS_NON_FINITE)
            throw TdpError{TDP_ERR_NON_FINITE, "the induced-dipole solve produced a non-finite residual"};
        if ((flags & TDP_COMPUTE_REQUIRE_CONVERGENCE) && !h->converged)
            throw TdpError{TDP_ERR_NOT_CONVERGED, "the induced dipoles did not converge"};
    } catch (const TdpError& e) {
        return fail(h, e);
    }
    return TDP_OK;
}

int tdp_compute_openmm(tdp_handle* h, const void* posq, int32_t posq_is_double, const int32_t* atom_index,
                       int32_t padded_num_atoms, long long* force_fixed, double* energy, uint32_t flags) {
    if (!h) return TDP_ERR_INVALID_ARGUMENT;
    try {
        if (h->n == 0) {
            if (energy) *energy = 0.0;
            h->iterations = 0;
            h->converged = 1;
            return TDP_OK;
        }
        if (!posq || !atom_index) throw TdpError{TDP_ERR_INVALID_ARGUMENT, "posq or atom_index is NULL"};
        if (padded_num_atoms < h->n) throw TdpError{TDP_ERR_INVALID_ARGUMENT, "padded_num_atoms < num_particles"};
        if ((flags & TDP_COMPUTE_FORCES) && !force_fixed)
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, "forces requested but force_fixed is NULL"};
        cudaStream_t st = h->stream;
        check_box(h);
        launch_posq_in(h->d, posq, posq_is_double ? 1 : 0, atom_index, st);
        solve_at(h, &kStaged, TDP_F64, 1);
        if (h->precision == TDP_PRECISION_DOUBLE) run_energy<double>(h);
        else run_energy<float>(h);
        if (flags & TDP_COMPUTE_FORCES) {
            launch_forces_out_fixed(h->d, atom_index, padded_num_atoms, force_fixed, st);
            h->launches++;
        }
        if (energy) TDP_CUDA(cudaMemcpyAsync(h->h_scal + 1, h->d.energy, sizeof(double), cudaMemcpyDeviceToHost, st));
        enqueue_flags(h);
        TDP_CUDA(cudaStreamSynchronize(st));
        TDP_CUDA(cudaGetLastError());
        check_flags(h);
        if (energy) *energy = h->h_scal[1];
        finish_timing(h);
        if (h->status == TDP_STATUS_NON_FINITE)
            throw TdpError{TDP_ERR_NON_FINITE, "the induced-dipole solve produced a non-finite residual"};
        if ((flags & TDP_COMPUTE_REQUIRE_CONVERGENCE) && !h->converged)
            throw TdpError{TDP_ERR_NOT_CONVERGED, "the induced dipoles did not converge"};
    } catch (const TdpError& e) {
        return fail(h, e);
    }
    return TDP_OK;
}

int tdp_get_dipoles(tdp_handle* h, int32_t which, const void* positions, int32_t pos_dtype, int32_t on_device,
                    double* out) {
    if (!h || !out) return TDP_ERR_INVALID_ARGUMENT;
    try {
        if (which < TDP_DIPOLES_INDUCED || which > TDP_DIPOLES_TOTAL)
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, "unknown dipole kind"};
        if (h->n == 0) return TDP_OK;
        solve_at(h, positions, pos_dtype, on_device);
        size_t n3 = 3 * (size_t)h->n;
        cudaStream_t st = h->stream;
        enqueue_flags(h);
        if (which == TDP_DIPOLES_INDUCED) {
            TDP_CUDA(cudaMemcpyAsync(out, h->d.mu, n3 * 8, cudaMemcpyDeviceToHost, st));
            TDP_CUDA(cudaStreamSynchronize(st));
        } else if (which == TDP_DIPOLES_LAB_PERMANENT) {
            TDP_CUDA(cudaMemcpyAsync(out, h->d.lab, n3 * 8, cudaMemcpyDeviceToHost, st));
            TDP_CUDA(cudaStreamSynchronize(st));
        } else {
            TDP_CUDA(cudaMemcpyAsync(out, h->d.lab, n3 * 8, cudaMemcpyDeviceToHost, st));
            TDP_CUDA(cudaMemcpyAsync(h->h_forces, h->d.mu, n3 * 8, cudaMemcpyDeviceToHost, st));
            TDP_CUDA(cudaStreamSynchronize(st));
            for (size_t k = 0; k < n3; k++) out[k] += h->h_forces[k];
        }
        check_flags(h);
    } catch (const TdpError& e) {
        return fail(h, e);
    }
    return TDP_OK;
}

int tdp_get_potential(tdp_handle* h, const void* positions, int32_t pos_dtype, int32_t on_device, const double* grid,
                      int32_t num_points, double* out) {
    if (!h || (num_points > 0 && (!grid || !out)) || num_points < 0) return TDP_ERR_INVALID_ARGUMENT;
    try {
        if (num_points == 0) return TDP_OK;
        if (h->n == 0) {
            for (int g = 0; g < num_points; g++) out[g] = 0.0;
            return TDP_OK;
        }
        solve_at(h, positions, pos_dtype, on_device);
        cudaStream_t st = h->stream;
        double* dgrid = nullptr;
        double* dout = nullptr;
        TDP_CUDA(cudaMallocAsync((void**)&dgrid, sizeof(double) * 3 * num_points, st));
        TDP_CUDA(cudaMallocAsync((void**)&dout, sizeof(double) * num_points, st));
        TDP_CUDA(cudaMemcpyAsync(dgrid, grid, sizeof(double) * 3 * num_points, cudaMemcpyHostToDevice, st));
        launch_potential(h->d, dgrid, num_points, dout, st);
        TDP_CUDA(cudaMemcpyAsync(out, dout, sizeof(double) * num_points, cudaMemcpyDeviceToHost, st));
        TDP_CUDA(cudaFreeAsync(dgrid, st));
        TDP_CUDA(cudaFreeAsync(dout, st));
        TDP_CUDA(cudaStreamSynchronize(st));
    } catch (const TdpError& e) {
        return fail(h, e);
    }
    return TDP_OK;
}

int tdp_get_moments(tdp_handle* h, const void* positions, int32_t pos_dtype, int32_t on_device, const double* masses,
                    double* out13) {
    if (!h || !masses || !out13) return TDP_ERR_INVALID_ARGUMENT;
    try {
        if (h->n == 0) {
            for (int k = 0; k < 13; k++) out13[k] = 0.0;
            return TDP_OK;
        }
        solve_at(h, positions, pos_dtype, on_device);
        cudaStream_t st = h->stream;
        int nb = h->d.nvb;
        double* dmass = nullptr;
        double* scratch = nullptr;
        double* dout = nullptr;
        TDP_CUDA(cudaMallocAsync((void**)&dmass, sizeof(double) * h->n, st));
        TDP_CUDA(cudaMallocAsync((void**)&scratch, sizeof(double) * 14 * nb, st));
        TDP_CUDA(cudaMallocAsync((void**)&dout, sizeof(double) * 13, st));
        TDP_CUDA(cudaMemcpyAsync(dmass, masses, sizeof(double) * h->n, cudaMemcpyHostToDevice, st));
        launch_moments(h->d, dmass, scratch, dout, st);
        TDP_CUDA(cudaMemcpyAsync(out13, dout, sizeof(double) * 13, cudaMemcpyDeviceToHost, st));
        TDP_CUDA(cudaFreeAsync(dmass, st));
        TDP_CUDA(cudaFreeAsync(scratch, st));
        TDP_CUDA(cudaFreeAsync(dout, st));
        TDP_CUDA(cudaStreamSynchronize(st));
    } catch (const TdpError& e) {
        return fail(h, e);
    }
    return TDP_OK;
}

int tdp_get_pme_parameters(const tdp_handle* h, double* alpha, int32_t* nx, int32_t* ny, int32_t* nz) {
    if (!h || !alpha || !nx || !ny || !nz) return TDP_ERR_INVALID_ARGUMENT;
    if (h->method != TDP_PME) {
        const_cast<tdp_handle*>(h)->err = "getPMEParametersInContext: This Context is not using PME";
        return TDP_ERR_NOT_PME;
    }
    if (h->ew) {
        // The Ewald mode reports what it runs with: the alpha and grid planned
        // at its first evaluation (before it, the same rule on the current box).
        double a = 0.0;
        int g[3] = {0, 0, 0};
        ewald_params(h->ew, &a, g);
        if (g[0] == 0) {
            a = h->pme_alpha > 0.0 ? h->pme_alpha : std::sqrt(-std::log(2.0 * h->ewald_tol)) / h->cutoff;
            for (int k = 0; k < 3; k++)
                g[k] = h->pme_grid[0] > 0 ? h->pme_grid[k]
                                          : pme_smooth_size(std::max(6, (int)std::ceil(2.0 * a * h->box[4 * k] /
                                                                                       (3.0 * std::pow(h->ewald_tol, 0.2)))));
        }
        *alpha = a;
        *nx = g[0];
        *ny = g[1];
        *nz = g[2];
        return TDP_OK;
    }
    if (h->pme_alpha != 0.0 && h->pme_grid[0] != 0) {
        *alpha = h->pme_alpha;
        *nx = h->pme_grid[0];
        *ny = h->pme_grid[1];
        *nz = h->pme_grid[2];
        return TDP_OK;
    }
    // OpenMM's documented choice (NonbondedForceImpl::calcPMEParameters, used by
    // ReferenceTholeDipoleKernels.cpp:143-152): alpha = sqrt(-ln(2 tol))/cutoff,
    // n_k = ceil(2 alpha L_k / (3 tol^(1/5))), at least 6.
    double tol = h->ewald_tol;
    double a = std::sqrt(-std::log(2.0 * tol)) / h->cutoff;
    int g[3];
    for (int k = 0; k < 3; k++) {
        g[k] = (int)std::ceil(2.0 * a * h->box[4 * k] / (3.0 * std::pow(tol, 0.2)));
        g[k] = std::max(g[k], 6);
    }
    *alpha = a;
    *nx = g[0];
    *ny = g[1];
    *nz = g[2];
    return TDP_OK;
}

int tdp_solver_stats(const tdp_handle* h, int32_t* iterations, double* epsilon, int32_t* converged, int32_t* status) {
    if (!h) return TDP_ERR_INVALID_ARGUMENT;
    if (iterations) *iterations = h->iterations;
    if (epsilon) *epsilon = h->epsilon;
    if (converged) *converged = h->converged;
    if (status) *status = h->status;
    return TDP_OK;
}

int tdp_solver_history(tdp_handle* h, double* eps_out, int32_t capacity, int32_t* count) {
    if (!h || (capacity > 0 && !eps_out)) return TDP_ERR_INVALID_ARGUMENT;
    try {
        const int m = std::min(std::max(capacity, 0), h->eps_slots);
        if (m > 0) {
            TDP_CUDA(cudaStreamSynchronize(h->stream));
            TDP_CUDA(cudaMemcpy(eps_out, h->d.scal_eps, sizeof(double) * m, cudaMemcpyDeviceToHost));
        }
        if (count) *count = h->eps_slots;
    } catch (const TdpError& e) {
        return fail(h, e);
    }
    return TDP_OK;
}

int tdp_enable_timing(tdp_handle* h, int32_t enable) {
    if (!h) return TDP_ERR_INVALID_ARGUMENT;
    h->timing = enable != 0;
    return TDP_OK;
}

int tdp_stage_times(const tdp_handle* h, double* out) {
    if (!h || !out) return TDP_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < TDP_NUM_STAGE_TIMES; k++) out[k] = h->stage_ms[k];
    return TDP_OK;
}

}  // extern "C"
