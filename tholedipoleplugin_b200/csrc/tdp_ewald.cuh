// tdp_ewald.cuh -- the Ewald mode of the box path (TDP_FLAG_EWALD): real space
// over a neighbour list of 32-atom tiles within the cutoff, smooth particle-mesh
// Ewald (order 5, cuFFT) for reciprocal space, self and neutralising-plasma
// terms.  The reference plugin has no Ewald sum (its "PME" is the minimum
// image over all pairs); this mode is the library's own, defined and checked
// against the FP64 restatement in oracle/ewald.py.
#pragma once

#include "tdp_kernels.cuh"

namespace tdp {

struct Ewald;

// State that does not depend on the box (neighbour list, buffers of the
// atom-side kernels); the grid is planned by ewald_prepare.
// vacuum: the variational NoCutoff model (alpha = 0, no cutoff, every tile
// pair in the list, no reciprocal space); direct: Direct polarization (the
// energy pass needs a second set of records).
Ewald* ewald_create(const Dev& d, int precision, bool vacuum = false, bool direct = false);
void ewald_destroy(Ewald* e);

// Chooses alpha and the grid on the first call (alpha_in > 0 and grid_in[0] > 0
// pin them; otherwise alpha = sqrt(-ln(2 tol))/cutoff and n_k = the
// 2,3,5,7-smooth size at or above ceil(2 alpha L_k / (3 tol^(1/5))), at least
// 6) and keeps the grid afterwards, as a context keeps its PME grid; the
// influence function follows every box change.
void ewald_prepare(Ewald* e, const Dev& d, const double box[3], double cutoff, double tol, double alpha_in,
                   const int grid_in[3], cudaStream_t st);
void ewald_params(const Ewald* e, double* alpha, int grid[3]);

// Neighbour list of the sorted tiles within the cutoff (part of
// ewald_fixed_field; alone for a caller that only runs matvecs).
void ewald_build_list(Ewald* e, const Dev& d, cudaStream_t st);
// Permanent field E_M of the sorted records into partial slots 0 (real
// space) and 1 (reciprocal + self); builds the neighbour list first.
// operand (the fused start of a warm-started solve): dipole records
// P = m + mu0 in place of m, giving E_M + T mu0 (covalent partners split
// into their M and I scales).
template <class R> void ewald_fixed_field(Ewald* e, const Dev& d, cudaStream_t st, const void* operand = nullptr);
// Periodic field T v of the operand in vec_s into partial slots 0 and 1.
template <class R> void ewald_matvec(Ewald* e, const Dev& d, cudaStream_t st);
// Energy, forces (fpair) and torques (torque) at the converged dipoles d.mu;
// plasma = -pi Q^2 / (2 V alpha^2) is added to the energy.  direct: the
// Direct-polarization functional (the Mutual one minus the induced dipoles'
// own energy), whose forces are its gradient at mu = alpha E_M.
template <class R> void ewald_energy(Ewald* e, const Dev& d, double total_charge, cudaStream_t st,
                                     bool direct = false);
// Nonzero when the last neighbour-list build overflowed a row (valid after the
// stream has been synchronised).
int ewald_list_overflow(const Ewald* e);
// Kernel launches of the last call of each stage (for the launch count).
int ewald_last_launches(const Ewald* e);
// Smallest size >= n whose prime factors are 2, 3, 5 and 7 only.
int pme_smooth_size(int n);

}  // namespace tdp
