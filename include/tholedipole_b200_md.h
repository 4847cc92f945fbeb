/*
 * tholedipole_b200_md.h -- device-resident rigid-water velocity-Verlet step
 * used to time TholeDipoleForce inside molecular dynamics.  The plugin has no
 * counterpart (integration and constraints belong to OpenMM's integrators);
 * these entry points stand in for a VerletIntegrator with rigid water so that
 * an MD step can run without leaving the GPU.
 *
 * Each molecule is three consecutive atoms (O, H1, H2) held rigid by three
 * distance constraints (O-H1, O-H2, H1-H2), solved per molecule with bounded
 * SHAKE/RATTLE iterations.  All arrays are device pointers of n*3 doubles
 * (n = 3 * num_waters); masses in g/mol, forces in energy/nm with the force's
 * energy unit taken as kJ/mol, dt in ps.
 */
#ifndef THOLEDIPOLE_B200_MD_H_
#define THOLEDIPOLE_B200_MD_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* v += dt/2 * F/m; x += dt*v; then SHAKE x (and the matching velocity
 * correction) back onto the constraints, using the constraint directions of
 * the positions before the drift.  Returns 0 or a negative TDP_ERR_* code. */
int tdp_md_kick_drift(int32_t num_waters, double d_oh, double d_hh, double m_o, double m_h, double dt,
                      double* positions, double* velocities, const double* forces, void* stream);

/* v += dt/2 * F/m; then RATTLE the velocities onto the constraint manifold
 * (zero relative velocity along each constrained bond). */
int tdp_md_kick(int32_t num_waters, double d_oh, double d_hh, double m_o, double m_h, double dt,
                const double* positions, double* velocities, const double* forces, void* stream);

/* Project velocities onto the constraints (RATTLE only, no kick). */
int tdp_md_constrain_velocities(int32_t num_waters, double d_oh, double d_hh, double m_o, double m_h,
                                const double* positions, double* velocities, void* stream);

/* The same two half steps on HOST arrays (positions, velocities, forces of
 * n*3 doubles in host memory), for an integrator loop that hands host
 * positions to tdp_compute each step.  Runs on host threads (up to 16, each
 * over its own range of waters); no CUDA call.  forces may be NULL in
 * tdp_md_host_kick (RATTLE only). */
int tdp_md_host_kick_drift(int32_t num_waters, double d_oh, double d_hh, double m_o, double m_h, double dt,
                           double* positions, double* velocities, const double* forces);
int tdp_md_host_kick(int32_t num_waters, double d_oh, double d_hh, double m_o, double m_h, double dt,
                     const double* positions, double* velocities, const double* forces);

/* Kinetic energy sum(m v^2)/2 into *out (device double), for the temperature. */
int tdp_md_kinetic_energy(int32_t num_waters, double m_o, double m_h, const double* velocities, double* out,
                          void* stream);

#ifdef __cplusplus
}
#endif
#endif
