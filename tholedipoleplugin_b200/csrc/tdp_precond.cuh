// tdp_precond.cuh -- Ewald-operator preconditioner of the minimum-image CG
// solve (the default PME mode of the box path).
//
// The reference's "PME" field is the minimum image over all pairs
// (ReferenceTholeDipoleForce.cpp:1414-1423), so every matvec of its Mutual
// solve is an all-pairs walk.  Its operator A = I - S T S (S = diag sqrt(alpha))
// is close to the Ewald operator B of the same box: the near field (every
// Thole-damped pair and its M/I scales) is identical, and the long-range part
// differs only in how the lattice beyond each atom's cube is summed.  The
// largest part of that difference is the uniform-polarisation mode: a
// minimum-image cube around an atom sees the depolarising field -(4 pi / 3V) M
// of its total dipole M, the tin-foil Ewald sum none, so B carries that term.
// Applying B^-1 costs a few real-space walks within a short cutoff plus a
// coarse PME grid, a small fraction of one all-pairs walk (1.2 ms against
// 8.7 ms at 98,304 atoms, mixed form), and cuts the outer iterations there
// from 7 to 2 from a cold start (which also begins at y = M(b), see
// precond_cold_start) and from 5-6 to 2 per warm-started MD step.  Below about
// 30,000 atoms an all-pairs matvec is cheap enough that plain CG is as fast,
// so the C ABI uses it from 32,768 atoms on unless told otherwise.
//
// The preconditioner is z = M(r): `inner` CG iterations on B z = r from z = 0,
// on r scaled to unit RMS (the PME grid of the mixed form is 64-bit fixed
// point, so the operand is kept at the scale of the dipoles whatever the size
// of the residual).  A CG polynomial depends on r, so the outer solve is the
// flexible (Polak-Ribiere) form: beta = z'.(r' - r) / z.r = -a z'.q / z.r.
#pragma once

#include "tdp_kernels.cuh"

namespace tdp {

struct Precond;

// cutoff, tol: real-space cutoff and PME tolerance of B (alpha and the grid
// follow the Ewald mode's rules); inner: B iterations per application.
Precond* precond_create(const Dev& d, int precision, double cutoff, double tol, int inner);
void precond_destroy(Precond* p);
double precond_cutoff(const Precond* p);
// Box (orthorhombic lengths) of this evaluation and the neighbour list of the
// sorted tiles; after launch_pack.
void precond_prepare(Precond* p, const Dev& d, const double box[3], cudaStream_t st);
// One application at outer slot `slot`: z = M(r) from d.r (whose r.r block
// partials are in d.rr_part), then scal_rr[slot] = r.z and
// p = z (first) or z + beta p with the flexible beta from d.q, scal_a[slot-1]
// and scal_rr[slot-1]; packs sqrt(alpha) p as the next matvec operand.
template <class R> void precond_apply(Precond* p, const Dev& d, int slot, bool first, cudaStream_t st);
// Starting point of a cold solve: y = M(b) for b = sqrt(alpha) E (instead of
// y = b), with mu = sqrt(alpha) y packed for the residual's matvec.  Uses d.r
// and d.rr_part as scratch.
template <class R> void precond_cold_start(Precond* p, const Dev& d, cudaStream_t st);
// Kernel launches of the last application (cuFFT's own not counted).
int precond_last_launches(const Precond* p);
// Nonzero when the last neighbour-list build overflowed (after a sync).
int precond_list_overflow(const Precond* p);

}  // namespace tdp
