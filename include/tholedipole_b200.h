/*
 * tholedipole_b200.h -- C ABI of the B200 (sm_100a) TholeDipoleForce kernels.
 *
 * This is the boundary a CUDA-platform kernel of the TholeDipoleForce plugin
 * (aehogan/tholedipoleplugin) binds: every entry point replaces one method of
 * the abstract kernel interface CalcTholeDipoleForceKernel
 * (openmmapi/include/TholeDipoleKernels.h:46-122) or one stage the reference
 * platform runs behind it (platforms/reference/src/ReferenceTholeDipoleKernels.cpp).
 * Plain pointers and sizes only; no C++ or torch types cross it.
 *
 * Conventions
 *  - Every function returns TDP_OK (0) or a negative TDP_ERR_* code; the
 *    message of the last failure on a handle is tdp_last_error(h) (or
 *    tdp_last_error(NULL) for failures before a handle exists).  Nothing
 *    throws across the ABI.
 *  - A handle is single-stream and not thread-safe: the OpenMM caller
 *    (TholeDipoleForceImpl, openmmapi/src/TholeDipoleForceImpl.cpp:110-195)
 *    uses one kernel object from the context's thread.
 *  - Units are the reference's: nm, e, e*nm, nm^3; energies in e^2/nm and
 *    forces in e^2/nm^2 (Coulomb prefactor 1, ReferenceTholeDipoleForce.cpp:20-21).
 *  - Arrays of vectors are AoS, n*3 doubles unless stated otherwise.
 *  - All device work runs on the handle's stream (tdp_set_stream).
 */
#ifndef THOLEDIPOLE_B200_H_
#define THOLEDIPOLE_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TDP_ABI_VERSION 1

/* Status codes. */
#define TDP_OK 0
#define TDP_ERR_INVALID_ARGUMENT (-1)
#define TDP_ERR_CUDA (-2)
#define TDP_ERR_NOT_PME (-3)
#define TDP_ERR_SIZE_MISMATCH (-4)
#define TDP_ERR_BOX_TOO_SMALL (-5)
#define TDP_ERR_NOT_CONVERGED (-6)   /* only returned when TDP_COMPUTE_REQUIRE_CONVERGENCE is set */
#define TDP_ERR_NON_FINITE (-7)
#define TDP_ERR_UNSUPPORTED (-8)

/* Enumerations: same values as TholeDipoleForce (openmmapi/include/TholeDipoleForce.h:58-109). */
#define TDP_NO_CUTOFF 0
#define TDP_PME 1
#define TDP_DIRECT 0
#define TDP_MUTUAL 1
#define TDP_EXTRAPOLATED 2
#define TDP_ZTHENX 0
#define TDP_BISECTOR 1
#define TDP_ZBISECT 2
#define TDP_THREEFOLD 3
#define TDP_ZONLY 4
#define TDP_NO_AXIS_TYPE 5

/* Arithmetic of the pair kernels.
 *  MIXED : FP32 pair arithmetic (positions as FP32 offsets from FP64 tile
 *          centres), FP64 accumulation of every tile's partial sums, FP64 CG
 *          scalars and FP64 recomputation of the true residual.
 *  DOUBLE: FP64 pair arithmetic and accumulation throughout ("plain"). */
#define TDP_PRECISION_MIXED 0
#define TDP_PRECISION_DOUBLE 1

/* Mutual-polarization solver.  Both stop on the reference's criterion: the
 * RMS change a Jacobi step would make, sqrt(sum|alpha(E+T mu)-mu|^2 / N)
 * (ReferenceTholeDipoleForce.cpp:838-846), below the target epsilon.
 *  CG    : conjugate gradients on the symmetric (alpha^-1 - T) system
 *          (Jacobi-preconditioned), converging to the same fixed point.  In
 *          the minimum-image PME mode (not TDP_FLAG_EWALD) each residual is
 *          also preconditioned by three CG iterations on the Ewald operator
 *          of the same box (real space within max(0.6 nm, the 1e-12 damping
 *          range), PME tolerance 1e-3, plus the minimum-image cube's uniform
 *          depolarising field -4 pi M / 3V), with flexible directions, from
 *          32,768 atoms on (below that plain CG is as fast); a cold solve
 *          starts from the preconditioned right-hand side.  A box edge below
 *          twice that cutoff runs unpreconditioned.  At create, TDP_PRECOND=1
 *          uses the preconditioner at any size, TDP_PRECOND=0 never, and
 *          TDP_PRECOND_INNER sets the inner iterations (1-8).
 *  JACOBI: the reference's own fixed-point iteration, step for step. */
#define TDP_SOLVER_CG 0
#define TDP_SOLVER_JACOBI 1

/* Flags of tdp_system_desc.flags. */
/* The reference reads rInvVec[4] past the end of a 4-element vector in every
 * dipole-dipole force coefficient (ReferenceTholeDipoleForce.cpp:196 vs
 * :264,277,323,333).  By default the kernels use 0.0 for that word -- the
 * value a fresh process of the compiled reference reads, which makes results
 * reproducible against it.  With this flag they use 1/r^4 instead. */
#define TDP_FLAG_DD_FORCE_R4 (1u << 0)
/* Start the Mutual CG solve from the previous calls' induced dipoles (the
 * reference restarts from mu0 = alpha*E every call): the polynomial through
 * the last converged solutions (up to three by default, TDP_PREDICTOR = 1..4
 * at create), evaluated one call ahead.  With CG the first walk then gives the
 * permanent field and the starting matvec together (TDP_FUSED_START=0 at create
 * keeps them apart).  The converged result is the same fixed point to the
 * solver tolerance; only the iteration count changes. */
#define TDP_FLAG_WARM_START (1u << 1)
/* Ewald mode (with TDP_PME only).  The reference has no Ewald sum: its "PME"
 * is the minimum image over all pairs (ReferenceTholeDipoleForce.cpp:1414-1423)
 * and alpha/grid are only reported (ReferenceTholeDipoleKernels.cpp:143-152).
 * With this flag the handle runs a true Ewald sum instead: real space within
 * the cutoff over a neighbour list of 32-atom tiles, smooth particle-mesh Ewald
 * of order 5 (the TholeDipoleForce default, TholeDipoleForce.cpp:43) on the
 * grid tdp_get_pme_parameters reports, and the self and neutralising-plasma
 * terms.  The fields and induced dipoles are the periodic versions of the
 * reference's (same Thole damping, M and I scales); the energy is the
 * variational one, U_perm - 1/2 mu.E_M, and the forces are its exact negative
 * gradient (Mutual and Direct polarization, whose energies are stationary in
 * the induced dipoles -- Direct's functional drops the induced-induced term;
 * Extrapolated gives TDP_ERR_UNSUPPORTED; frames whose torque map is the
 * gradient of their rotation, i.e. not ZOnly).
 * Orthorhombic boxes only; real space, damping corrections
 * included, stops at the cutoff, where exp(-a u^3) of every pair must be
 * <= 1e-12 (cutoff^3 >= 27.63 t_max^5); tdp_adjoint is unsupported.
 * alpha = pme_alpha and the grid = pme_grid when both are set, otherwise
 * alpha = sqrt(-ln(2 tol))/cutoff and
 * n_k = the smallest 2,3,5,7-smooth size >= ceil(2 alpha L_k / (3 tol^(1/5)))
 * (at least 6), fixed at the first evaluation. */
#define TDP_FLAG_EWALD (1u << 2)
/* Variational mode of a NoCutoff system (TDP_NO_CUTOFF only; PME systems use
 * TDP_FLAG_EWALD).  Fields and induced dipoles are exactly the reference's;
 * the energy is the variational one, U_perm - 1/2 mu.E_M, summed over all pairs
 * with bare kernels, and the forces are its exact negative gradient (the
 * reference's own forces follow its quasi-internal-frame convention and are
 * not the gradient of its energy, ReferenceTholeDipoleForce.cpp:129-366).  Runs
 * on the Ewald mode's real-space kernels with alpha = 0, no cutoff and no
 * reciprocal space; the same limits as TDP_FLAG_EWALD (Mutual or Direct
 * polarization, no ZOnly frames, no tdp_adjoint). */
#define TDP_FLAG_VARIATIONAL (1u << 3)

/* Flags of tdp_compute. */
#define TDP_COMPUTE_FORCES (1u << 0)
#define TDP_COMPUTE_ENERGY (1u << 1)
#define TDP_COMPUTE_REQUIRE_CONVERGENCE (1u << 2)

/* Element types of position / force buffers. */
#define TDP_F64 0
#define TDP_F32 1

/* Which dipoles tdp_get_dipoles returns (TholeDipoleKernels.h:91-105). */
#define TDP_DIPOLES_INDUCED 0
#define TDP_DIPOLES_LAB_PERMANENT 1
#define TDP_DIPOLES_TOTAL 2

/* Solver status (tdp_solver_stats). */
#define TDP_STATUS_CONVERGED 0
#define TDP_STATUS_MAX_ITERATIONS 1
#define TDP_STATUS_NON_FINITE 2

typedef struct tdp_handle tdp_handle;

/* Everything ReferenceCalcTholeDipoleForceKernel::initialize copies out of a
 * TholeDipoleForce (ReferenceTholeDipoleKernels.cpp:83-158). */
typedef struct tdp_system_desc {
    int32_t num_particles;
    const double* charges;              /* n */
    const double* molecular_dipoles;    /* n*3, local frame */
    const double* polarizabilities;     /* n */
    const double* thole_damping;        /* n */
    const int32_t* axis_types;          /* n */
    const int32_t* atom_z;              /* n, -1 for none */
    const int32_t* atom_x;              /* n */
    const int32_t* atom_y;              /* n */
    /* Covalent12 (M scale) and Covalent13 (I scale) lists as CSR; offsets have
     * n+1 entries.  NULL offsets mean empty lists. */
    const int32_t* covalent12_offsets;
    const int32_t* covalent12_atoms;
    const int32_t* covalent13_offsets;
    const int32_t* covalent13_atoms;
    int32_t nonbonded_method;           /* TDP_NO_CUTOFF / TDP_PME */
    int32_t polarization_type;          /* TDP_DIRECT / TDP_MUTUAL / TDP_EXTRAPOLATED */
    double cutoff;                      /* nm (PME: box must be >= 2*cutoff) */
    double ewald_error_tolerance;
    double pme_alpha;                   /* 0 -> chosen from the tolerance */
    int32_t pme_grid[3];
    double mutual_target_epsilon;
    int32_t mutual_max_iterations;
    int32_t num_extrapolation_coefficients;
    const double* extrapolation_coefficients;
    int32_t precision;                  /* TDP_PRECISION_* */
    int32_t solver;                     /* TDP_SOLVER_* */
    uint32_t flags;                     /* TDP_FLAG_* */
} tdp_system_desc;

/* ABI version of the loaded library. */
int tdp_abi_version(void);

/* Message of the last failure on h (NULL h: the last failure of a create). */
const char* tdp_last_error(const tdp_handle* h);

/* CalcTholeDipoleForceKernel::initialize (TholeDipoleKernels.h:59); validation
 * as TholeDipoleForceImpl::initialize (openmmapi/src/TholeDipoleForceImpl.cpp:52-108).
 * Uploads parameters, builds the exclusion/scale tables and device buffers. */
int tdp_create(const tdp_system_desc* desc, tdp_handle** out);
void tdp_destroy(tdp_handle* h);

/* CUDA stream (a cudaStream_t) for all later work; NULL = legacy default stream. */
int tdp_set_stream(tdp_handle* h, void* stream);

/* Periodic box, 9 doubles (three box vectors, row-major).  Only the diagonal
 * enters the minimum image (ReferenceTholeDipoleForce.cpp:1414-1423).  PME
 * requires every diagonal entry >= 1.999999*cutoff
 * (ReferenceTholeDipoleKernels.cpp:168-172), checked at compute time. */
int tdp_set_box(tdp_handle* h, const double* box9);

/* CalcTholeDipoleForceKernel::copyParametersToContext (TholeDipoleKernels.h:75,
 * ReferenceTholeDipoleKernels.cpp:317-339): per-particle parameters and axis
 * atoms only; num_particles must not change (TDP_ERR_SIZE_MISMATCH). */
int tdp_update_params(tdp_handle* h, int32_t num_particles, const double* charges,
                      const double* molecular_dipoles, const double* polarizabilities,
                      const double* thole_damping, const int32_t* axis_types, const int32_t* atom_z,
                      const int32_t* atom_x, const int32_t* atom_y);

/* The per-particle half of copyParametersToContext (same reference lines as
 * tdp_update_params): charges (n), molecular_dipoles (n*3),
 * polarizabilities (n), thole_damping (n), on the device if on_device else on
 * the host; axis frames and covalent maps stay.  With device arrays the
 * parameters never pass through the host (the damping radius and net charge
 * are reduced on the device); this is the forward of the Python layer's
 * torch.autograd.Function on CUDA tensors. */
int tdp_update_particle_params(tdp_handle* h, const double* charges, const double* molecular_dipoles,
                               const double* polarizabilities, const double* thole_damping, int32_t on_device);

/* CalcTholeDipoleForceKernel::execute (TholeDipoleKernels.h:68,
 * ReferenceTholeDipoleKernels.cpp:201-215).  positions: n*3 of pos_dtype, on
 * the device if on_device else on the host.  With TDP_COMPUTE_FORCES the
 * forces are ADDED to forces_accum (n*3 of force_dtype, same residency as the
 * positions); energy (host double) may be NULL. */
int tdp_compute(tdp_handle* h, const void* positions, int32_t pos_dtype, int32_t on_device,
                void* forces_accum, int32_t force_dtype, double* energy, uint32_t flags);

/* execute on the OpenMM CUDA platform's own buffers (what a CUDA-platform
 * kernel gets from its CudaContext, as CudaTholeDipoleKernelFactory.cpp:68-73
 * hands it contexts[0]): posq holds x, y, z, q per slot as float4 (single and
 * mixed precision) or double4 (posq_is_double, double precision) in the
 * context's current atom order, slot k holding atom atom_index[k]; the forces
 * are ADDED to the 64-bit fixed-point accumulator force_fixed (2^32 units per
 * force unit, component c of slot k at k + c * padded_num_atoms, truncated
 * toward zero) -- the layout the platform sums all forces in.  All pointers
 * are device memory; the energy (host double, may be NULL) is returned as in
 * tdp_compute.  The positions are taken as given: molecules must be whole, as
 * the platform keeps them. */
int tdp_compute_openmm(tdp_handle* h, const void* posq, int32_t posq_is_double, const int32_t* atom_index,
                       int32_t padded_num_atoms, long long* force_fixed, double* energy, uint32_t flags);

/* getInducedDipoles / getLabFramePermanentDipoles / getTotalDipoles
 * (TholeDipoleKernels.h:91-105) at the given positions (NULL: the positions
 * of the last tdp_compute).  out: n*3 host doubles. */
int tdp_get_dipoles(tdp_handle* h, int32_t which, const void* positions, int32_t pos_dtype,
                    int32_t on_device, double* out);

/* getElectrostaticPotential (TholeDipoleKernels.h:113,
 * ReferenceTholeDipoleForce.cpp:1315-1372): bare 1/r and 1/r^3 sums of the
 * charges, lab-frame and induced dipoles at num_points host grid points. */
int tdp_get_potential(tdp_handle* h, const void* positions, int32_t pos_dtype, int32_t on_device,
                      const double* grid, int32_t num_points, double* out);

/* Electrostatic potential at grid points that allocates no device memory.
 * No counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc -- a host program whose pool allocator owns all device memory,
 * or a loop that must not hit the implicit device synchronisation of
 * cudaMalloc/cudaFree.  Same sums as tdp_get_potential (bare 1/r and 1/r^3
 * of the charges and the total dipoles, minimum image when periodic != 0 with
 * the box diagonal box3, a host array), but every input and output is a
 * device pointer the caller owns: positions and total_dipoles (n*3),
 * charges (n), grid (num_points*3), out (num_points), and no handle is needed.
 * Its scratch (per-atom-chunk partial sums) is one file-scope device array of
 * TDP_NOALLOC_SCRATCH_DOUBLES doubles (8 MiB) that every GPU loading this
 * library keeps until exit; num_points above that count is rejected with
 * TDP_ERR_INVALID_ARGUMENT.  The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress) with that device current, so make it
 * before any stream capture; the address is kept for the life of the process,
 * so do not call this on a device after a cudaDeviceReset of it.  The call
 * clears any pending non-sticky CUDA error on entry, so that it reports only
 * its own launch failures.  All calls share the array and leave their
 * partial sums in it (every slot a call reads, it first writes, so nothing
 * needs clearing); calls that overlap on the GPU race on it.  Errors:
 * tdp_last_error(NULL). */
#define TDP_NOALLOC_SCRATCH_DOUBLES (1 << 20)
int tdp_potential_noalloc(int32_t num_particles, const double* positions, const double* charges,
                          const double* total_dipoles, int32_t num_points, const double* grid, int32_t periodic,
                          const double* box3, double* out, void* stream);

/* getSystemMultipoleMoments (TholeDipoleKernels.h:121,
 * ReferenceTholeDipoleForce.cpp:1225-1313): 13 values (charge, dipole in
 * Debye, traceless quadrupole), masses: n host doubles. */
int tdp_get_moments(tdp_handle* h, const void* positions, int32_t pos_dtype, int32_t on_device,
                    const double* masses, double* out13);

/* getPMEParameters (TholeDipoleKernels.h:84, ReferenceTholeDipoleKernels.cpp:341-348):
 * TDP_ERR_NOT_PME unless the method is PME. */
int tdp_get_pme_parameters(const tdp_handle* h, double* alpha, int32_t* nx, int32_t* ny, int32_t* nz);

/* Solver report of the last solve (ReferenceTholeDipoleForce.h:136-150:
 * getMutualInducedDipoleIterations / Epsilon / Converged) plus a status. */
int tdp_solver_stats(const tdp_handle* h, int32_t* iterations, double* epsilon, int32_t* converged,
                     int32_t* status);

/* The stopping quantity of every step of the last Mutual CG or Jacobi solve
 * (the RMS change a Jacobi step would make, as tdp_solver_stats reports the
 * final one), oldest first: the start, then one per iteration and one per
 * true-residual check.  After tdp_adjoint it is the adjoint solve's.  Copies min(capacity, *count) values into eps_out
 * (host doubles); *count receives the number available (0 after Direct or
 * Extrapolated polarization).  No reference counterpart: a convergence
 * monitor of this library's solvers. */
int tdp_solver_history(tdp_handle* h, double* eps_out, int32_t capacity, int32_t* count);

/* Reverse mode of the last tdp_compute (its positions and parameters):
 * gradients of  L = dL_dE * E + sum_i dL_dF_i . F_i  (F the total force,
 * torque mapping included) with respect to every particle's charge,
 * polarizability, Thole factor and molecular-frame dipole.  dL_dF: n*3 host
 * doubles (NULL = zero); grads: n*6 host doubles, per particle
 * (dq, dalpha, dthole, dmu_mol_x, dmu_mol_y, dmu_mol_z).  Mutual polarization
 * costs one adjoint solve of the same symmetric (alpha^-1 - T) system; pair
 * damping terms are recomputed, not stored.  The plugin has no counterpart:
 * this is the backward of the torch.autograd.Function in the Python layer.
 * Every polarization type; Extrapolated runs its perturbation recursion
 * (ReferenceTholeDipoleForce.cpp:853-909) backwards instead of a solve.
 * TDP_ERR_UNSUPPORTED in the Ewald and variational modes. */
int tdp_adjoint(tdp_handle* h, const double* dL_dF, double dL_dE, double* grads);

/* tdp_adjoint with dL_dF (n*3, NULL = zero) and grads (n*6) in device memory;
 * nothing is synchronised with the host beyond the adjoint solve's scalars. */
int tdp_adjoint_device(tdp_handle* h, const double* dL_dF, double dL_dE, double* grads);

/* Device timing of the last tdp_compute (CUDA events on the handle's stream),
 * recorded only after tdp_enable_timing(h, 1).  out[TDP_NUM_STAGE_TIMES]:
 * [0] pack+rotation ms, [1] permanent field ms, [2] induced-dipole solve ms,
 * [3] energy/force stage ms, [4] torque mapping ms, [5] total ms,
 * [6] mutual-field matvec launches, [7] summed matvec kernel ms,
 * [8] energy/force kernel ms, [9] kernel launches of the call,
 * [10] fused-start walks (0 or 1: a warm-started solve's single walk giving
 * the permanent field plus the starting matvec), [11] their kernel ms.  The
 * fused walk is counted in neither [6] nor [7].  [12] preconditioner
 * applications of the minimum-image CG (each a few matvecs of the Ewald
 * operator of the same box), [13] their ms (counted in neither [6] nor [7]). */
#define TDP_NUM_STAGE_TIMES 14
int tdp_enable_timing(tdp_handle* h, int32_t enable);
int tdp_stage_times(const tdp_handle* h, double* out);

/* ---------------------------------------------------------------------------
 * Cluster batches.  No reference counterpart: the reference evaluates one
 * System per context (ReferenceCalcTholeDipoleForceKernel::execute,
 * platforms/reference/src/ReferenceTholeDipoleKernels.cpp); a batch evaluates
 * many independent NoCutoff systems -- the clusters -- in one persistent
 * launch, each with exactly the per-system semantics of tdp_compute.
 *
 * desc describes all clusters' particles concatenated; cluster c owns the
 * particles [cluster_offsets[c], cluster_offsets[c+1]) and every axis atom and
 * covalent partner of a particle must lie in its cluster.  Indices in desc are
 * global.  Requirements: nonbonded_method TDP_NO_CUTOFF, solver TDP_SOLVER_CG;
 * precision as for tdp_create.  The largest cluster must fit one CTA's shared
 * memory (about 300 bytes per particle in the mixed form); otherwise
 * TDP_ERR_UNSUPPORTED.  Errors: tdp_batch_last_error(b), or (NULL) for create.
 * ------------------------------------------------------------------------- */
typedef struct tdp_batch tdp_batch;

int tdp_batch_create(const tdp_system_desc* desc, int32_t num_clusters, const int32_t* cluster_offsets,
                     tdp_batch** out);
void tdp_batch_destroy(tdp_batch* b);
const char* tdp_batch_last_error(const tdp_batch* b);
int tdp_batch_set_stream(tdp_batch* b, void* stream);

/* One evaluation of every cluster: positions (n*3 doubles) in; forces (n*3,
 * WRITTEN, torque mapping included) and per-cluster energies (num_clusters)
 * out, either may be NULL.  on_device: all three pointers are device memory
 * (no host synchronisation beyond the timing event) rather than host memory.
 * The first call picks the tile shape (CTA size, lanes per particle) by timing
 * every candidate on this batch, then captures the launch in a CUDA graph that
 * every call replays. */
int tdp_batch_compute(tdp_batch* b, const double* positions, int32_t on_device, double* forces, double* energies);

/* Induced dipoles of the last compute, n*3 host doubles. */
int tdp_batch_get_induced_dipoles(tdp_batch* b, double* out);

/* New per-particle parameters for every cluster (copyParametersToContext of
 * each cluster at once, ReferenceTholeDipoleKernels.cpp:317-339): charges (n),
 * molecular_dipoles (n*3), polarizabilities (n), thole_damping (n), on the
 * device if on_device else on the host.  Axis frames and covalent maps stay.
 * A change of the largest Thole factor moves the damping radius and
 * re-captures the launch graph. */
int tdp_batch_update_params(tdp_batch* b, const double* charges, const double* molecular_dipoles,
                            const double* polarizabilities, const double* thole_damping, int32_t on_device);

/* Reverse mode of the last tdp_batch_compute, every cluster in one persistent
 * launch: per cluster c, the gradients of
 *   L_c = dL_dE[c] * E_c + sum over its particles of dL_dF_i . F_i
 * with respect to every particle's charge, polarizability, Thole factor and
 * molecular-frame dipole -- tdp_adjoint (the backward of the Python
 * layer's torch.autograd.Function) for all clusters at once, one adjoint solve
 * of each cluster's (alpha^-1 - T) system for Mutual polarization.  dL_dF: n*3
 * (NULL = zero), dL_dE: num_clusters (NULL = zero), grads: n*6 per particle
 * (dq, dalpha, dthole, dmu_mol_x, dmu_mol_y, dmu_mol_z); all three on the
 * device if on_device else on the host.  No reference counterpart.  Direct and
 * Mutual polarization (TDP_ERR_UNSUPPORTED for Extrapolated). */
int tdp_batch_adjoint(tdp_batch* b, const double* dL_dF, const double* dL_dE, int32_t on_device, double* grads);

/* Per-cluster adjoint CG iterations and final residual of the last
 * tdp_batch_adjoint (Mutual; 0 otherwise); either may be NULL. */
int tdp_batch_adjoint_stats(tdp_batch* b, int32_t* iterations, double* epsilons);

/* Per-cluster solver report of the last compute: CG iterations (Extrapolated:
 * the order) and the final RMS dipole change; either may be NULL. */
int tdp_batch_solver_stats(tdp_batch* b, int32_t* iterations, double* epsilons);

/* Tile shape chosen by the autotuner (0s before the first compute) and the
 * device time of the last launch in ms. */
int tdp_batch_tile(const tdp_batch* b, int32_t* threads, int32_t* lanes, int32_t* ctas, double* last_ms);

/* The autotuner's candidates and their measured ms per launch (-1: not
 * timed); fills up to capacity entries, returns the number of candidates. */
int tdp_batch_tile_candidates(const tdp_batch* b, int32_t capacity, int32_t* threads, int32_t* lanes, double* ms);

#ifdef __cplusplus
}
#endif
#endif
