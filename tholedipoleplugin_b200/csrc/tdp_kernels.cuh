// tdp_kernels.cuh -- device state and kernel launchers shared by the C ABI
// layer (tdp_capi.cu) and the kernels (tdp_kernels.cu).
#pragma once

#include "tdp_common.cuh"

namespace tdp {

// All device buffers of one system (sizes: n atoms, n_pad = n rounded up to a
// whole number of bands, nsplit partial-sum slots of the pair kernels = one per
// band, n_eblk energy partials = one per band pair, nvb blocks of the O(N)
// kernels).
constexpr int kMuHist = 4;

struct Dev {
    int n = 0, n_pad = 0, nsplit = 1, nvb = 1, n_eblk = 1;
    PairParams pp{};
    // Inputs.
    double* pos = nullptr;       // n_pad*3 (FP64 working copy of the positions)
    double* charge = nullptr;    // n
    double* dip_mol = nullptr;   // n*3 molecular-frame dipoles
    double* alpha = nullptr;     // n
    double* salpha = nullptr;    // n, sqrt(alpha)
    double* thole = nullptr;     // n
    int4* axis = nullptr;        // n: type, Z, X, Y
    // Packed pair-kernel records, Vec4<R> of n_pad entries.
    void* posq = nullptr;        // mixed: (offset from tile centre, q); plain: (x, y, z, q)
    void* dipt = nullptr;        // (lab dipole, thole)
    void* ind = nullptr;         // (induced dipole, 0)
    double2* yz = nullptr;       // n_pad raw (y, z) for the QI frame test
    double4* tctr = nullptr;     // n_pad/32 tile centres
    double4* text = nullptr;     // n_pad/32 tile half-extents
    // Covalent scale exceptions (both directions), CSR over atoms.
    int* exc_off = nullptr;
    int* exc_j = nullptr;
    double* exc_m = nullptr;     // M scale of the pair
    double* exc_s = nullptr;     // I scale of the pair
    int2* exc_tiles = nullptr;   // per 32-atom tile: lowest and highest tile holding a listed partner
    // Spatially sorted copies for the field kernels (permanent field, matvec):
    // slot k holds atom order[k] (-1 for padding), atom i sits in slot rank[i].
    int* order = nullptr;        // n_pad
    int* rank = nullptr;         // n
    double* pos_s = nullptr;     // n_pad*3
    void* posq_s = nullptr;      // Vec4<R>: (offset from tile centre, q)
    void* dipt_s = nullptr;      // Vec4<R>: (lab dipole, thole)
    void* vec_s = nullptr;       // Vec4<R>: (matvec operand, thole)
    double4* tctr_s = nullptr;
    double4* text_s = nullptr;
    int* exs_off = nullptr;      // exceptions by slot, partners as slots
    int* exs_j = nullptr;
    double* exs_m = nullptr;
    double* exs_s = nullptr;
    int2* exs_tiles = nullptr;
    // Torque-mapping users: for atom a, (frame atom, role) entries.
    int* users_off = nullptr;
    int2* users = nullptr;
    // Working vectors (n*3 doubles).
    double* lab = nullptr;
    double* E = nullptr;
    double* mu = nullptr;
    // Converged dipoles of the last kMuHist calls, newest first (warm-start
    // predictor; the handle counts the valid ones).
    double* mu_hist[kMuHist] = {nullptr, nullptr, nullptr, nullptr};
    double* mu0 = nullptr;       // starting dipoles of a fused warm start (E then holds E + T mu0)
    double* y = nullptr;
    double* r = nullptr;
    double* p = nullptr;
    double* q = nullptr;
    double* hist = nullptr;      // extrapolation orders, korder*n*3
    double* partial = nullptr;   // nsplit*6*n_pad pair-kernel partial sums (scratch)
    // Mixed all-pairs form: the field and energy kernels add their per-band
    // sums into one 64-bit fixed-point accumulator (6*n_pad, units of
    // 1/fix_scale; integer addition makes the result independent of the order)
    // that a flush kernel converts into partial slot 0 and clears (nsplit = 1).
    // A sum of magnitude >= fix_limit sets *fix_err instead of wrapping.
    unsigned long long* fixacc = nullptr;
    int* fix_err = nullptr;
    double fix_scale = 0.0, fix_limit = 0.0;
    double* energy_partial = nullptr;
    double* fpair = nullptr;
    double* torque = nullptr;
    double* ftotal = nullptr;
    double* energy = nullptr;    // 1
    double* rr_part = nullptr;   // nvb
    double* eps_part = nullptr;
    double* pq_part = nullptr;
    double* scal_rr = nullptr;   // per-iteration scalars
    double* scal_eps = nullptr;
    double* scal_a = nullptr;    // CG step sizes by slot (preconditioned solves only)
    double* coef = nullptr;      // extrapolation coefficients
};

template <class R> void launch_pack(const Dev& d, cudaStream_t st);
template <class R> void launch_rotate(const Dev& d, cudaStream_t st);
template <class R> void launch_field(const Dev& d, int kind, cudaStream_t st);
template <class R> void launch_energy(const Dev& d, cudaStream_t st);
template <class R> void launch_fixed_done(const Dev& d, cudaStream_t st);
template <class R> void launch_warm_start(const Dev& d, cudaStream_t st);
// mu = sum_k c[k] mu_hist[k] over the first nh history entries.
void launch_predict(const Dev& d, int nh, const double* c, cudaStream_t st);
// use_partial = false: the field term is already in E (the fused start).
template <class R> void launch_cg_residual(const Dev& d, cudaStream_t st, bool use_partial = true);
// The start of a fused warm start: operand records m + mu0 (mu0 in d.mu), and
// afterwards E := E + T mu0 from the walk's partial sums, y = mu0/sqrt(alpha).
template <class R> void launch_pack_total(const Dev& d, cudaStream_t st);
template <class R> void launch_fused_done(const Dev& d, cudaStream_t st);
void launch_cg_q(const Dev& d, cudaStream_t st);
void launch_cg_update(const Dev& d, int slot, cudaStream_t st);
template <class R> void launch_cg_p(const Dev& d, int prev, int slot, cudaStream_t st);
// mu0 != NULL: the packed operand is mu - mu0 (the final check of a fused start).
template <class R> void launch_cg_mu(const Dev& d, cudaStream_t st, const double* mu0 = nullptr);
template <class R> void launch_jacobi(const Dev& d, cudaStream_t st);
template <class R> void launch_extrap_step(const Dev& d, int k, cudaStream_t st);
template <class R> void launch_extrap_combine(const Dev& d, int korder, const double* coef, cudaStream_t st);
void launch_step_eps(const Dev& d, cudaStream_t st);
void launch_eps_scalar(const Dev& d, int slot, cudaStream_t st);
template <class R> void launch_pack_ind(const Dev& d, cudaStream_t st);
void launch_energy_done(const Dev& d, cudaStream_t st);
void launch_torque_gather(const Dev& d, cudaStream_t st);
void launch_add_forces(const Dev& d, void* acc, int is_f32, cudaStream_t st);
void launch_positions_in(const Dev& d, const void* src, int is_f32, cudaStream_t st);
void launch_posq_in(const Dev& d, const void* posq, int is_double, const int* atom_index, cudaStream_t st);
void launch_forces_out_fixed(const Dev& d, const int* atom_index, int padded, long long* acc, cudaStream_t st);
void launch_potential(const Dev& d, const double* grid, int ng, double* out, cudaStream_t st);
void launch_moments(const Dev& d, const double* mass, double* scratch, double* out13, cudaStream_t st);

// Adjoint (tdp_adjoint.cu).
void launch_torque_vjp(const Dev& d, const double* g, double* gt, cudaStream_t st);
// Damped (and degenerate) partners of every atom, listed by the pair VJP per
// (split, atom) in rows of `cap` entries (a count above cap means the row
// overflowed), reused by the fixed-field and matvec Thole VJPs; nsplit = 0:
// no list (those passes scan all pairs).  Valid while the scratch of
// launch_adjoint_pair is untouched.
struct AdjPairList {
    int nsplit = 0, cap = 0;
    const int* slow = nullptr;
    const int* nslow = nullptr;
};
// precision: the arithmetic of the closed-form pairs (FP32 in the mixed form);
// scratch: adjoint_pair_scratch(n) doubles; list (may be NULL) receives the
// damped-partner lists.
size_t adjoint_pair_scratch(int n);
size_t adjoint_fixed_scratch(int n);
void launch_adjoint_pair(const Dev& d, const double* g, const double* gT, double gE, double* a8, int precision,
                         double* scratch, AdjPairList* list, cudaStream_t st);
// scratch: adjoint_fixed_scratch(n) doubles (the split sums of the tiled pass), or NULL.
void launch_adjoint_fixed(const Dev& d, const double* lam, double* b5, const AdjPairList& list, int precision,
                          double* scratch, cudaStream_t st);
void launch_adjoint_matvec_t(const Dev& d, const double* lam, double* ct, const AdjPairList& list, cudaStream_t st);
// ct (+)= d/dt of lam^T T(t) mu for an explicit mu (n*3); accumulate adds to ct.
void launch_adjoint_matvec_t_mu(const Dev& d, const double* lam, const double* mu, double* ct, bool accumulate,
                                const AdjPairList& list, cudaStream_t st);
// out = ca a + cb b (n*3; b may be NULL); acc_i += a_i . b_i (per atom).
void launch_lincomb(int n, double ca, const double* a, double cb, const double* b, double* out, cudaStream_t st);
void launch_dot3_acc(int n, const double* a, const double* b, double* acc, cudaStream_t st);
// out = alpha (.) v (n*3).
void launch_alpha_scale(const Dev& d, const double* v, double* out, cudaStream_t st);
void launch_rotation_vjp(const Dev& d, const double* glab, double* gmol, cudaStream_t st);
void launch_adjoint_split(const Dev& d, const double* a8, const double* b5, double* amu, double* glab,
                          cudaStream_t st);
void launch_add_field(const Dev& d, const double* base, double* out, cudaStream_t st);
template <class R> void launch_rhs_init(const Dev& d, const double* rhs, cudaStream_t st);
template <class R> void launch_set_operand(const Dev& d, const double* x, cudaStream_t st);
// galpha (n, may be NULL) replaces amu_tlam . e_tmu as the polarizability gradient.
void launch_adjoint_assemble(const Dev& d, const double* a8, const double* b5, const double* ct,
                             const double* amu_tlam, const double* e_tmu, const double* gmol, double* out,
                             cudaStream_t st, const double* galpha = nullptr);

}  // namespace tdp
