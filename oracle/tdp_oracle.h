/*
 * tdp_oracle.h -- CPU restatement (FP64, plain C) of the reference plugin's
 * TholeDipoleForce physics, used ONLY as test infrastructure: the parity
 * tests, the smoke check and the CPU-baseline leg of bench.py call it as the
 * checker.  Nothing in the shipped library links or calls it.
 *
 * Every function follows one routine of the reference, cited by file:line in
 * aehogan/tholedipoleplugin:
 *   platforms/reference/src/ReferenceTholeDipoleForce.cpp   (physics, "RTDF.cpp")
 *   platforms/reference/src/ReferenceTholeDipoleKernels.cpp (kernel wrapper)
 *
 * Parity pin: tests/test_oracle_pin.py compares this restatement against the
 * reference's own ReferenceTholeDipoleForce.cpp compiled by oracle/Makefile
 * into oracle/_ref/ (see oracle/ref_driver.cpp), and the committed golden
 * fixtures under tests/golden/ were produced by that compiled reference.
 */
#ifndef TDP_ORACLE_H_
#define TDP_ORACLE_H_

#ifdef __cplusplus
extern "C" {
#endif

/* Enumerations match openmmapi/include/TholeDipoleForce.h:58-109. */
enum { TDPO_NOCUTOFF = 0, TDPO_PME = 1 };
enum { TDPO_DIRECT = 0, TDPO_MUTUAL = 1, TDPO_EXTRAPOLATED = 2 };
enum { TDPO_ZTHENX = 0, TDPO_BISECTOR = 1, TDPO_ZBISECT = 2, TDPO_THREEFOLD = 3,
       TDPO_ZONLY = 4, TDPO_NOAXISTYPE = 5 };

/* How the pair routine's fifth inverse-power slot is filled.  The reference
 * sizes rInvVec to 4 entries (RTDF.cpp:196) but reads rInvVec[4] in every
 * dipole-dipole force coefficient (RTDF.cpp:264,277,323,333): an
 * out-of-bounds heap read.  TDPO_RINV4_FILL uses the constant rinv4_value
 * for that word (0.0 is what a fresh process of the compiled reference
 * reads); TDPO_RINV4_POWER uses 1/r^4, the value the code evidently intends. */
enum { TDPO_RINV4_FILL = 0, TDPO_RINV4_POWER = 1 };

typedef struct tdpo_system {
    int n;
    const double* pos;       /* n*3, nm */
    const double* charge;    /* n, e */
    const double* dipole;    /* n*3, molecular-frame permanent dipole, e*nm */
    const double* polarity;  /* n, nm^3 */
    const double* thole;     /* n */
    const int* axis;         /* n*4: axisType, atomZ, atomX, atomY */
    const int* cov12_off;    /* n+1 CSR offsets of the Covalent12 lists (M scale) */
    const int* cov12;
    const int* cov13_off;    /* n+1 CSR offsets of the Covalent13 lists (I scale) */
    const int* cov13;
    int method;              /* TDPO_NOCUTOFF or TDPO_PME (orthorhombic minimum image) */
    double box[3];           /* box diagonal (PME only) */
    int polarization;        /* TDPO_DIRECT / TDPO_MUTUAL / TDPO_EXTRAPOLATED */
    double target_eps;       /* Mutual: RMS dipole-change target */
    int max_iter;            /* Mutual: iteration cap */
    int n_extrap;            /* Extrapolated: coefficient count (0 -> OPT4 defaults) */
    const double* extrap;
    int rinv4_mode;          /* TDPO_RINV4_FILL or TDPO_RINV4_POWER */
    double rinv4_value;      /* constant for TDPO_RINV4_FILL */
} tdpo_system;

typedef struct tdpo_stats {
    int iterations;
    double epsilon;
    int converged;
} tdpo_stats;

/* All functions return 0 on success, nonzero on invalid input. */
int tdpo_validate(const tdpo_system* s);
int tdpo_lab_dipoles(const tdpo_system* s, double* lab);
int tdpo_fixed_field(const tdpo_system* s, const double* lab, double* field);
int tdpo_induced_field(const tdpo_system* s, const double* mu, double* field);
int tdpo_induced_dipoles(const tdpo_system* s, const double* lab, double* fixed_field,
                         double* mu, tdpo_stats* stats);
int tdpo_electrostatic(const tdpo_system* s, const double* lab, const double* mu,
                       double* energy, double* forces, double* torques);
int tdpo_map_torque(const tdpo_system* s, const double* torques, double* forces);
int tdpo_compute(const tdpo_system* s, double* energy, double* forces, double* mu,
                 double* lab, tdpo_stats* stats);
int tdpo_potential(const tdpo_system* s, const double* grid, int ngrid, double* out);
int tdpo_moments(const tdpo_system* s, const double* masses, double* out13);

#ifdef __cplusplus
}
#endif
#endif
