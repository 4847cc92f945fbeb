// tdp_pairs.cuh -- per-pair arithmetic of the TholeDipoleForce hot path, in
// the reference's semantics (aehogan/tholedipoleplugin,
// platforms/reference/src/ReferenceTholeDipoleForce.cpp, "RTDF.cpp").  R is
// float (mixed form) or double (plain form).  Every function works on the
// displacement d = p_j - p_i already minimum-imaged; a masked pair (self or
// padding) arrives with r2 = +inf, which makes rinv = 0 and every term zero.
#pragma once

#include "tdp_common.cuh"

namespace tdp {

// Thole damping of 1/r^3 and 3/r^5 as getAndScaleInverseRs (RTDF.cpp:646-676).
// Pairs with r2 >= damp_r2 have a*u^3 >= 50 and are left undamped there too.
template <class R>
__device__ __forceinline__ void damp_field(R r2, R rinv, R ti, R tj, R damp_r2, R& rr3, R& rr5) {
    if (r2 < damp_r2) {
        R dmp = ti * tj;
        if (dmp != R(0)) {
            R pgamma = ti < tj ? ti : tj;
            R r = r2 * rinv;
            R ratio = sizeof(R) == 4 ? (R)__fdividef((float)r, (float)dmp) : r / dmp;
            ratio = ratio * ratio * ratio;
            R damp = -pgamma * ratio;
            if (damp > R(-50)) {
                R e = exp_r(damp);
                rr3 *= R(1) - e;
                rr5 *= R(1) - (R(1) - damp) * e;
            }
        }
    }
}

// One term of the mutual field (T mu)_i, calculateInducedDipolePairIxn with
// rr3 -> -rr3 (RTDF.cpp:766-818), I scale applied by the caller.
template <class R, bool DAMP = true>
__device__ __forceinline__ void pair_matvec(R dx, R dy, R dz, R r2, R vx, R vy, R vz, R ti, R tj, R damp_r2,
                                            R& fx, R& fy, R& fz) {
    R rinv = rsqrt_r(r2);
    R rinv2 = rinv * rinv;
    R rr3 = rinv * rinv2;
    R rr5 = R(3) * rr3 * rinv2;
    if (DAMP) damp_field(r2, rinv, ti, tj, damp_r2, rr3, rr5);
    R dd = rr5 * (vx * dx + vy * dy + vz * dz);
    fx += dd * dx - rr3 * vx;
    fy += dd * dy - rr3 * vy;
    fz += dd * dz - rr3 * vz;
}

// One term of the permanent field at i from the charge and lab-frame dipole of
// j, calculateFixedDipoleFieldPairIxn (RTDF.cpp:678-713), M scale applied by
// the caller:  E_i -= d (rr3 q_j - rr5 mu_j.d) + mu_j rr3.
template <class R, bool DAMP = true>
__device__ __forceinline__ void pair_fixed(R dx, R dy, R dz, R r2, R qj, R mx, R my, R mz, R ti, R tj, R damp_r2,
                                           R& fx, R& fy, R& fz) {
    R rinv = rsqrt_r(r2);
    R rinv2 = rinv * rinv;
    R rr3 = rinv * rinv2;
    R rr5 = R(3) * rr3 * rinv2;
    if (DAMP) damp_field(r2, rinv, ti, tj, damp_r2, rr3, rr5);
    R f = rr3 * qj - rr5 * (mx * dx + my * dy + mz * dz);
    fx -= dx * f + mx * rr3;
    fy -= dy * f + my * rr3;
    fz -= dz * f + mz * rr3;
}

// Inputs of one particle to the pair energy routine.
template <class R>
struct EAtom {
    R q, mx, my, mz;   // charge, lab-frame permanent dipole
    R ux, uy, uz;      // induced dipole
    R t;               // Thole factor
};

// calculateElectrostaticPairIxn (RTDF.cpp:129-366) with formQIRotationMatrix
// (:573-607), in its canonical orientation I = lower index, K = higher index,
// d = p_K - p_I.  The QI frame has rows [X, Y, Z] with Z along d, and the
// multipole algebra below treats component 0 as the bond axis and back-rotates
// with the permuted matrix of :150-159, exactly as the reference does.
// SIDES = 1 adds the force and torque on I (and the pair energy) to f/t;
// SIDES = 2 adds the force and torque on K to f/t; SIDES = 3 adds I's to f/t,
// K's to g/u and the pair energy.  Linear in (mScale, iScale).
template <class R, int SIDES>
__device__ __forceinline__ void pair_energy_sides(R dx, R dy, R dz, R r2, bool yz_differ, const EAtom<R>& I,
                                                  const EAtom<R>& K, R mS, R iS, R damp_r2, R rv4_power,
                                                  R rv4_fill, bool mutual, R& fx, R& fy, R& fz, R& tx, R& ty, R& tz,
                                                  R& gx, R& gy, R& gz, R& ux, R& uy, R& uz, R& en) {
    R rinv = rsqrt_r(r2);
    // QI frame.
    R zx = dx * rinv, zy = dy * rinv, zz = dz * rinv;
    R xx = zx, xy = zy, xz = zz;
    if (yz_differ) xx += R(1);
    else xy += R(1);
    R dt = zx * xx + zy * xy + zz * xz;
    xx -= zx * dt;
    xy -= zy * dt;
    xz -= zz * dt;
    R xn2 = xx * xx + xy * xy + xz * xz;
    if (xn2 > R(0)) {
        R s = rsqrt_r(xn2);
        xx *= s;
        xy *= s;
        xz *= s;
    }
    R yx = zy * xz - zz * xy, yy = zz * xx - zx * xz, yz = zx * xy - zy * xx;

    R uI0 = xx * I.ux + xy * I.uy + xz * I.uz;
    R uI1 = yx * I.ux + yy * I.uy + yz * I.uz;
    R uI2 = zx * I.ux + zy * I.uy + zz * I.uz;
    R uJ0 = xx * K.ux + xy * K.uy + xz * K.uz;
    R uJ1 = yx * K.ux + yy * K.uy + yz * K.uz;
    R uJ2 = zx * K.ux + zy * K.uy + zz * K.uz;
    R QI0 = I.q, QJ0 = K.q;
    R QI1 = xx * I.mx + xy * I.my + xz * I.mz;
    R QI2 = yx * I.mx + yy * I.my + yz * I.mz;
    R QI3 = zx * I.mx + zy * I.my + zz * I.mz;
    R QJ1 = xx * K.mx + xy * K.my + xz * K.mz;
    R QJ2 = yx * K.mx + yy * K.my + yz * K.mz;
    R QJ3 = zx * K.mx + zy * K.my + zz * K.mz;

    R rv1 = rinv;
    R rv2 = rv1 * rinv;
    R rv3 = rv2 * rinv;
    // rInvVec[4]: read past the end of the reference's 4-element vector.
    R rv4 = rv4_power * (rv3 * rinv) + rv4_fill;

    // Thole factors; beyond damp_r2 every factor is exactly 1 in the reference too.
    R tc = R(1), td0 = R(1), td1 = R(1), dtc = R(1), dtd0 = R(1), dtd1 = R(1);
    if (r2 < damp_r2) {
        R dmp = I.t * K.t;
        if (fabs(dmp) > R(1.0e-5)) {
            R a = I.t < K.t ? I.t : K.t;
            R r = r2 * rinv;
            R u = sizeof(R) == 4 ? (R)__fdividef((float)r, (float)dmp) : r / dmp;
            R au3 = a * u * u * u;
            R e = exp_r(-au3);
            tc = R(1) - e;
            td0 = R(1) - e * (R(1) + R(1.5) * au3);
            td1 = R(1) - e;
            dtc = R(1) - e * (R(1) + R(1.5) * au3);
            dtd0 = R(1) - e * (R(1) + au3 + R(1.5) * au3 * au3);
            dtd1 = R(1) - e * (R(1) + au3);
        }
    }

    R Vij0, Vij1, Vij2, Vij3, Vji0, Vji1, Vji2, Vji3;
    R VijR0, VijR1, VijR2, VijR3, VjiR0, VjiR1, VjiR2, VjiR3;
    R Vijd0, Vijd1, Vijd2, Vjid0, Vjid1, Vjid2;

    R eP = rv1 * mS;
    R dP = R(-0.5) * mS * rv2;
    Vij0 = eP * QJ0;
    Vji0 = eP * QI0;
    VijR0 = dP * QJ0;
    VjiR0 = dP * QI0;

    eP = rv2 * mS;
    R eU = rv2 * iS * tc;
    dP = -rv3 * mS;
    R dU = R(-2) * rv3 * iS * dtc;
    Vij0 += -(eP * QJ1 + eU * uJ0);
    Vji1 = -(eP * QI0);
    VijR0 += -(dP * QJ1 + dU * uJ0);
    VjiR1 = -(dP * QI0);
    Vjid0 = -(eU * QI0);
    Vij1 = eP * QJ0;
    Vji0 += eP * QI1 + eU * uI0;
    VijR1 = dP * QJ0;
    VjiR0 += dP * QI1 + dU * uI0;
    Vijd0 = eU * QJ0;

    eP = R(-2) * rv3 * mS;
    eU = R(-2) * rv3 * iS * td0;
    dP = R(3) * rv4 * mS;
    dU = R(6) * rv4 * iS * dtd0;
    Vij1 += eP * QJ1 + eU * uJ0;
    Vji1 += eP * QI1 + eU * uI0;
    VijR1 += dP * QJ1 + dU * uJ0;
    VjiR1 += dP * QI1 + dU * uI0;
    Vijd0 += eU * QJ1;
    Vjid0 += eU * QI1;

    eP = rv3 * mS;
    eU = rv3 * iS * td1;
    dP = R(-1.5) * rv4 * mS;
    dU = R(-3) * rv4 * iS * dtd1;
    Vij2 = eP * QJ2 + eU * uJ1;
    Vji2 = eP * QI2 + eU * uI1;
    VijR2 = dP * QJ2 + dU * uJ1;
    VjiR2 = dP * QI2 + dU * uI1;
    Vijd1 = eU * QJ2;
    Vjid1 = eU * QI2;
    Vij3 = eP * QJ3 + eU * uJ2;
    Vji3 = eP * QI3 + eU * uI2;
    VijR3 = dP * QJ3 + dU * uJ2;
    VjiR3 = dP * QI3 + dU * uI2;
    Vijd2 = eU * QJ3;
    Vjid2 = eU * QI3;

    R fIZ = QI0 * VijR0 + QI1 * VijR1 + QI2 * VijR2 + QI3 * VijR3;
    R fJZ = QJ0 * VjiR0 + QJ1 * VjiR1 + QJ2 * VjiR2 + QJ3 * VjiR3;
    R EIX = QI3 * Vij1 - QI1 * Vij3;
    R EIY = QI1 * Vij2 - QI2 * Vij1;
    R EJX = QJ3 * Vji1 - QJ1 * Vji3;
    R EJY = QJ1 * Vji2 - QJ2 * Vji1;
    R iEIX = uI2 * Vijd0 - uI0 * Vijd2;
    R iEJX = uJ2 * Vjid0 - uJ0 * Vjid2;
    R iEIY = uI0 * Vijd1 - uI1 * Vijd0;
    R iEJY = uJ0 * Vjid1 - uJ1 * Vjid0;
    if (mutual) {
        R eC = R(-4) * rv3 * iS * td0;
        R dC = R(6) * rv4 * iS * dtd0;
        iEIX += eC * uI2 * uJ0;
        iEJX += eC * uJ2 * uI0;
        iEIY -= eC * uI1 * uJ0;
        iEJY -= eC * uJ1 * uI0;
        fIZ += dC * uI0 * uJ0;
        fJZ += dC * uJ0 * uI0;
        eC = R(2) * rv3 * iS * td1;
        dC = R(-3) * rv4 * iS * dtd1;
        iEIX -= eC * uI0 * uJ2;
        iEJX -= eC * uJ0 * uI2;
        iEIY += eC * uI0 * uJ1;
        iEJY += eC * uJ0 * uI1;
        fIZ += dC * (uI1 * uJ1 + uI2 * uJ2);
        fJZ += dC * (uJ1 * uI1 + uJ2 * uI2);
    }
    R qf0 = rinv * (EIY + EJY + iEIY + iEJY);
    R qf1 = -rinv * (EIX + EJX + iEIX + iEJX);
    R qf2 = -(fJZ + fIZ);
    // Back rotation with the reference's permuted matrix: rows (Y.y, Z.y, X.y),
    // (Y.z, Z.z, X.z), (Y.x, Z.x, X.x).
    R fvx = yy * qf0 + zy * qf1 + xy * qf2;
    R fvy = yz * qf0 + zz * qf1 + xz * qf2;
    R fvz = yx * qf0 + zx * qf1 + xx * qf2;
    if (SIDES & 1) {
        R EIZ = QI2 * Vij3 - QI3 * Vij2;
        R q0 = -EIX, q1 = -EIY, q2 = -EIZ;
        tx += yy * q0 + zy * q1 + xy * q2;
        ty += yz * q0 + zz * q1 + xz * q2;
        tz += yx * q0 + zx * q1 + xx * q2;
        fx -= fvx;
        fy -= fvy;
        fz -= fvz;
        R e = R(0.5) * (QI0 * Vij0 + QJ0 * Vji0);
        e += R(0.5) * (QI1 * Vij1 + QJ1 * Vji1);
        e += R(0.5) * (QI2 * Vij2 + QJ2 * Vji2);
        e += R(0.5) * (QI3 * Vij3 + QJ3 * Vji3);
        en += e;
    }
    if (SIDES & 2) {
        R EJZ = QJ2 * Vji3 - QJ3 * Vji2;
        R q0 = -EJX, q1 = -EJY, q2 = -EJZ;
        R& ox = SIDES == 3 ? ux : tx;
        R& oy = SIDES == 3 ? uy : ty;
        R& oz = SIDES == 3 ? uz : tz;
        R& px = SIDES == 3 ? gx : fx;
        R& py = SIDES == 3 ? gy : fy;
        R& pz = SIDES == 3 ? gz : fz;
        ox += yy * q0 + zy * q1 + xy * q2;
        oy += yz * q0 + zz * q1 + xz * q2;
        oz += yx * q0 + zx * q1 + xx * q2;
        px += fvx;
        py += fvy;
        pz += fvz;
    }
}

// pair_energy_sides<R, 3> for a pair that Thole damping does not reach (all
// six damping factors 1), with unit scales and rInvVec[4] = 0, computed in the
// lab frame.  With those factors the reference's QI-frame algebra
// (RTDF.cpp:212-340) reduces to expressions in the frame's X row alone, the
// axis its multipole algebra treats as the bond axis.  With P = m + u and
// W = m + 2u (W = m unless Mutual), and _0 the component along X:
//   E    = q_i q_j / r + (q_j (P_i0 + m_i0) - q_i (P_j0 + m_j0)) / (2 r^2)
//          + (m_i.P_j + m_j.P_i - 3 (m_i0 P_j0 + m_j0 P_i0)) / (2 r^3)
//   V_ij = (q_j/r^2 - 3 P_j0/r^3) X + P_j/r^3,  V_ji = (-q_i/r^2 - 3 P_i0/r^3) X + P_i/r^3
//   Vd_ij, Vd_ji: the same with W in place of P
//   S    = m_i x V_ij + m_j x V_ji + u_i x Vd_ij + u_j x Vd_ji
//   f    = (S x X) / r + (q_i q_j / r^2 - 2 (q_i P_j0 - q_j P_i0) / r^3) X
//   F_I -= perm(f), F_K += perm(f), tau_I = -perm(m_i x V_ij), tau_K = -perm(m_j x V_ji),
// perm(v) = (v_y, v_z, v_x) being the permuted back rotation of :150-159.  X is
// the frame test's (:580-593): (x^ - Z_x Z)/|.| = (d_y^2 + d_z^2, -d_x d_y,
// -d_x d_z) / (r sqrt(d_y^2 + d_z^2)) when the y or z coordinates differ,
// the Gram-Schmidt form otherwise.  kap = 1 (Mutual) or -1: W = P + kap u.
// VSUM: (tx, ty, tz) and (ux, uy, uz) receive V_ij and V_ji in place of the
// torques, and en only the charge terms.  The torque of an atom is linear in
// V with its own dipole fixed, tau_I = -perm(m_i x sum_j V_ij), and the
// dipole terms of the energy are 0.5 (m_i.V_ij + m_j.V_ji) (expand m.V with
// the expressions above: E = q_i q_j / r + (q_j P_i0 - q_i P_j0) / (2 r^2)
// + (m_i.V_ij + m_j.V_ji) / 2), so a walk can sum V over its partners and
// take one cross product and one dot product per atom at the end.
template <class R, bool VSUM = false>
__device__ __forceinline__ void pair_energy_lab(R dx, R dy, R dz, R r2, bool yz_differ, const EAtom<R>& I,
                                                const EAtom<R>& K, R kap, R& fx, R& fy, R& fz, R& tx, R& ty, R& tz,
                                                R& gx, R& gy, R& gz, R& ux, R& uy, R& uz, R& en) {
    const R rinv = rsqrt_r(r2);
    const R rho2 = dy * dy + dz * dz;
    R xx, xy, xz;
    if (yz_differ && rho2 > R(0)) {
        const R s = rinv * rsqrt_r(rho2);
        xx = rho2 * s;
        xy = -dx * dy * s;
        xz = -dx * dz * s;
    } else {
        const R zx = dx * rinv, zy = dy * rinv, zz = dz * rinv;
        xx = zx + (yz_differ ? R(1) : R(0));
        xy = zy + (yz_differ ? R(0) : R(1));
        xz = zz;
        const R dt = zx * xx + zy * xy + zz * xz;
        xx -= zx * dt;
        xy -= zy * dt;
        xz -= zz * dt;
        const R n2 = xx * xx + xy * xy + xz * xz;
        const R s = n2 > R(0) ? rsqrt_r(n2) : R(1);
        xx *= s;
        xy *= s;
        xz *= s;
    }
    const R pix = I.mx + I.ux, piy = I.my + I.uy, piz = I.mz + I.uz;
    const R pjx = K.mx + K.ux, pjy = K.my + K.uy, pjz = K.mz + K.uz;
    const R qi1 = xx * I.mx + xy * I.my + xz * I.mz, ui0 = xx * I.ux + xy * I.uy + xz * I.uz;
    const R qj1 = xx * K.mx + xy * K.my + xz * K.mz, uj0 = xx * K.ux + xy * K.uy + xz * K.uz;
    const R pi0 = qi1 + ui0, pj0 = qj1 + uj0;
    const R rv2 = rinv * rinv, rv3 = rv2 * rinv;
    const R qq = I.q * K.q;
    if (VSUM) {
        en += rinv * qq + R(0.5) * rv2 * (K.q * pi0 - I.q * pj0);
    } else {
        const R t1 = K.q * (pi0 + qi1) - I.q * (pj0 + qj1);
        const R t2 = I.mx * pjx + I.my * pjy + I.mz * pjz + K.mx * pix + K.my * piy + K.mz * piz -
                     R(3) * (qi1 * pj0 + qj1 * pi0);
        en += rinv * qq + R(0.5) * (rv2 * t1 + rv3 * t2);
    }
    // V_ij = a X + rv3 P_j, V_ji = b X + rv3 P_i, Vd_ij = c X + rv3 W_j,
    // Vd_ji = d X + rv3 W_i.  In S = m_i x V_ij + m_j x V_ji + u_i x Vd_ij +
    // u_j x Vd_ji the rv3 terms cancel pairwise (m_i x P_j + m_j x P_i +
    // u_i x W_j + u_j x W_i = 0 for P = m + u, W = m + (1 + kap) u), so
    // S = K x X with K = a m_i + b m_j + c u_i + d u_j, and for the unit X
    // S x X = (K.X) X - K.
    const R a = rv2 * K.q - R(3) * rv3 * pj0;
    const R b = -rv2 * I.q - R(3) * rv3 * pi0;
    {
        const R vx = a * xx + rv3 * pjx, vy = a * xy + rv3 * pjy, vz = a * xz + rv3 * pjz;
        if (VSUM) {
            tx += vx;
            ty += vy;
            tz += vz;
        } else {
            tx -= I.mz * vx - I.mx * vz;
            ty -= I.mx * vy - I.my * vx;
            tz -= I.my * vz - I.mz * vy;
        }
    }
    {
        const R vx = b * xx + rv3 * pix, vy = b * xy + rv3 * piy, vz = b * xz + rv3 * piz;
        if (VSUM) {
            ux += vx;
            uy += vy;
            uz += vz;
        } else {
            ux -= K.mz * vx - K.mx * vz;
            uy -= K.mx * vy - K.my * vx;
            uz -= K.my * vz - K.mz * vy;
        }
    }
    const R c = rv2 * K.q - R(3) * rv3 * (pj0 + kap * uj0);
    const R d = -rv2 * I.q - R(3) * rv3 * (pi0 + kap * ui0);
    const R kx = a * I.mx + b * K.mx + c * I.ux + d * K.ux;
    const R ky = a * I.my + b * K.my + c * I.uy + d * K.uy;
    const R kz = a * I.mz + b * K.mz + c * I.uz + d * K.uz;
    const R qf2 = rv2 * qq - R(2) * rv3 * (I.q * pj0 - K.q * pi0);
    const R cf = rinv * (kx * xx + ky * xy + kz * xz) + qf2;
    const R fvx = cf * xx - rinv * kx;
    const R fvy = cf * xy - rinv * ky;
    const R fvz = cf * xz - rinv * kz;
    fx -= fvy;
    fy -= fvz;
    fz -= fvx;
    gx += fvy;
    gy += fvz;
    gz += fvx;
}

// One side of the pair: SIDE_I adds the force and torque on I and the pair
// energy; otherwise the force and torque on K.
template <class R, bool SIDE_I>
__device__ __forceinline__ void pair_energy(R dx, R dy, R dz, R r2, bool yz_differ, const EAtom<R>& I,
                                            const EAtom<R>& K, R mS, R iS, R damp_r2, R rv4_power, R rv4_fill,
                                            bool mutual, R& fx, R& fy, R& fz, R& tx, R& ty, R& tz, R& en) {
    R d0 = 0, d1 = 0, d2 = 0, d3 = 0, d4 = 0, d5 = 0;
    pair_energy_sides<R, SIDE_I ? 1 : 2>(dx, dy, dz, r2, yz_differ, I, K, mS, iS, damp_r2, rv4_power, rv4_fill,
                                         mutual, fx, fy, fz, tx, ty, tz, d0, d1, d2, d3, d4, d5, en);
}

// Both sides of the mutual-field pair: the field at i from v_j and the field
// at j from v_i (the dipole-field tensor is even in d), I scale applied by the
// caller.
template <class R, bool DAMP = true>
__device__ __forceinline__ void pair_matvec2(R dx, R dy, R dz, R r2, R vix, R viy, R viz, R vjx, R vjy, R vjz, R ti,
                                             R tj, R damp_r2, R& fix, R& fiy, R& fiz, R& fjx, R& fjy, R& fjz) {
    R rinv = rsqrt_r(r2);
    R rinv2 = rinv * rinv;
    R rr3 = rinv * rinv2;
    R rr5 = R(3) * rr3 * rinv2;
    if (DAMP) damp_field(r2, rinv, ti, tj, damp_r2, rr3, rr5);
    R ddj = rr5 * (vjx * dx + vjy * dy + vjz * dz);
    R ddi = rr5 * (vix * dx + viy * dy + viz * dz);
    fix += ddj * dx - rr3 * vjx;
    fiy += ddj * dy - rr3 * vjy;
    fiz += ddj * dz - rr3 * vjz;
    fjx += ddi * dx - rr3 * vix;
    fjy += ddi * dy - rr3 * viy;
    fjz += ddi * dz - rr3 * viz;
}

// Both sides of the permanent-field pair (calculateFixedDipoleFieldPairIxn,
// RTDF.cpp:678-713), M scale applied by the caller:
//   E_i -= d (rr3 q_j - rr5 mu_j.d) + mu_j rr3,  E_j += d (rr3 q_i + rr5 mu_i.d) - mu_i rr3.
template <class R, bool DAMP = true>
__device__ __forceinline__ void pair_fixed2(R dx, R dy, R dz, R r2, R qi, R mix, R miy, R miz, R qj, R mjx, R mjy,
                                            R mjz, R ti, R tj, R damp_r2, R& fix, R& fiy, R& fiz, R& fjx, R& fjy,
                                            R& fjz) {
    R rinv = rsqrt_r(r2);
    R rinv2 = rinv * rinv;
    R rr3 = rinv * rinv2;
    R rr5 = R(3) * rr3 * rinv2;
    if (DAMP) damp_field(r2, rinv, ti, tj, damp_r2, rr3, rr5);
    R a = rr3 * qj - rr5 * (mjx * dx + mjy * dy + mjz * dz);
    R b = rr3 * qi + rr5 * (mix * dx + miy * dy + miz * dz);
    fix -= dx * a + mjx * rr3;
    fiy -= dy * a + mjy * rr3;
    fiz -= dz * a + mjz * rr3;
    fjx += dx * b - mix * rr3;
    fjy += dy * b - miy * rr3;
    fjz += dz * b - miz * rr3;
}

}  // namespace tdp
