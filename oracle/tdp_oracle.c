/*
 * tdp_oracle.c -- FP64 CPU restatement of the reference TholeDipoleForce
 * physics.  TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check and
 * the CPU-baseline leg of bench.py use it as the checker; the shipped library
 * never links or calls it.
 *
 * Each routine restates one routine of the reference (aehogan/
 * tholedipoleplugin, platforms/reference/src/ReferenceTholeDipoleForce.cpp,
 * cited as RTDF.cpp:line) in the same floating-point operation order, so that
 * the compiled reference (oracle/_ref, built by oracle/Makefile) and this file
 * agree to rounding level.  Where the reference has undefined behaviour the
 * restatement makes a documented choice (see the comment at each site).
 */
#include "tdp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double v[3]; } v3;

static inline v3 mk(double x, double y, double z) { v3 r; r.v[0] = x; r.v[1] = y; r.v[2] = z; return r; }
static inline v3 ld(const double* p) { return mk(p[0], p[1], p[2]); }
static inline v3 add(v3 a, v3 b) { return mk(a.v[0] + b.v[0], a.v[1] + b.v[1], a.v[2] + b.v[2]); }
static inline v3 sub(v3 a, v3 b) { return mk(a.v[0] - b.v[0], a.v[1] - b.v[1], a.v[2] - b.v[2]); }
static inline v3 scl(v3 a, double s) { return mk(a.v[0] * s, a.v[1] * s, a.v[2] * s); }
static inline double dot(v3 a, v3 b) { return a.v[0] * b.v[0] + a.v[1] * b.v[1] + a.v[2] * b.v[2]; }
static inline v3 cross(v3 a, v3 b) {
    return mk(a.v[1] * b.v[2] - a.v[2] * b.v[1], a.v[2] * b.v[0] - a.v[0] * b.v[2],
              a.v[0] * b.v[1] - a.v[1] * b.v[0]);
}
/* RTDF.cpp:469-475 (normalizeVec3): scale by 1/norm when norm > 0. */
static inline double normalize(v3* a) {
    double norm = sqrt(dot(*a, *a));
    if (norm > 0.0) *a = scl(*a, 1.0 / norm);
    return norm;
}

/* ReferencePmeTholeDipoleForce::getPeriodicDelta, RTDF.cpp:1414-1423:
 * orthorhombic minimum image from the box diagonal only. */
static inline v3 periodic(const tdpo_system* s, v3 d) {
    if (s->method == TDPO_PME) {
        for (int k = 0; k < 3; k++) {
            double b = s->box[k];
            if (b > 0) d.v[k] -= b * floor(d.v[k] / b + 0.5);
        }
    }
    return d;
}

/* Scale lookup, RTDF.cpp:609-644 with the guard at :382-385 / :806-808.  The
 * scale of pair (i<j) comes from atom i's maps only: the M scale is
 * _mScale[pos] for j at list position pos of Covalent12(i), the I scale
 * _iScale[pos] for Covalent13(i); a later duplicate overwrites an earlier one
 * (std::map assignment).  Lists longer than 5 read past _mScale/_iScale in the
 * reference (undefined); tdpo_validate rejects them. */
static const double kMScale[5] = {0.0, 0.0, 0.0, 0.5, 1.0};
static const double kIScale[5] = {0.0, 1.0, 1.0, 1.0, 1.0};

static double scale_lookup(const int* off, const int* atoms, const double* table, int i, int j) {
    double s = 1.0;
    if (!off) return s;
    for (int p = off[i]; p < off[i + 1]; p++)
        if (atoms[p] == j) s = table[p - off[i]];
    return s;
}
static inline double mscale(const tdpo_system* s, int i, int j) { return scale_lookup(s->cov12_off, s->cov12, kMScale, i, j); }
static inline double iscale(const tdpo_system* s, int i, int j) { return scale_lookup(s->cov13_off, s->cov13, kIScale, i, j); }

int tdpo_validate(const tdpo_system* s) {
    if (s->n < 0) return 1;
    for (int i = 0; i < s->n; i++) {
        int t = s->axis[4 * i], z = s->axis[4 * i + 1], x = s->axis[4 * i + 2], y = s->axis[4 * i + 3];
        /* TholeDipoleForceImpl.cpp:63-107 */
        if (t < TDPO_ZTHENX || t > TDPO_NOAXISTYPE) return 2;
        if (t != TDPO_NOAXISTYPE && (z < 0 || z >= s->n)) return 3;
        if (t != TDPO_NOAXISTYPE && t != TDPO_ZONLY && (x < 0 || x >= s->n)) return 4;
        if ((t == TDPO_ZBISECT || t == TDPO_THREEFOLD) && (y < 0 || y >= s->n)) return 5;
        /* RTDF.cpp:556-568: any atom with 0 <= Z != i is rotated, and every
         * axis type but ZOnly dereferences the X atom; X < 0 there is a null
         * dereference in the reference.  Out-of-range Z/X/Y likewise. */
        if (z >= s->n || x >= s->n || y >= s->n) return 6;
        if (z >= 0 && z != i && t != TDPO_ZONLY && x < 0) return 7;
        if (s->cov12_off && s->cov12_off[i + 1] - s->cov12_off[i] > 5) return 8;
        if (s->cov13_off && s->cov13_off[i + 1] - s->cov13_off[i] > 5) return 8;
    }
    return 0;
}

/* checkChiralCenterAtParticle / checkChiral (RTDF.cpp:432-467) followed by
 * applyRotationMatrixToParticle / applyRotationMatrix (RTDF.cpp:477-571). */
int tdpo_lab_dipoles(const tdpo_system* s, double* lab) {
    int err = tdpo_validate(s);
    if (err) return err;
    for (int i = 0; i < s->n; i++) {
        v3 d = ld(s->dipole + 3 * i);
        int t = s->axis[4 * i], z = s->axis[4 * i + 1], x = s->axis[4 * i + 2], y = s->axis[4 * i + 3];
        v3 pi = ld(s->pos + 3 * i);
        if (y > -1 && t == TDPO_ZTHENX) {
            v3 py = ld(s->pos + 3 * y);
            v3 ad = sub(pi, py), bd = sub(ld(s->pos + 3 * z), py), cd = sub(ld(s->pos + 3 * x), py);
            double volume = dot(cross(bd, cd), ad);
            if (volume < 0.0) d.v[1] *= -1.0;
        }
        if (z >= 0 && z != i) {
            v3 vz = sub(ld(s->pos + 3 * z), pi);
            normalize(&vz);
            v3 vx, vy;
            if (t == TDPO_ZONLY) {
                vx = fabs(vz.v[0]) < 0.866 ? mk(1.0, 0.0, 0.0) : mk(0.0, 1.0, 0.0);
            } else {
                vx = sub(ld(s->pos + 3 * x), pi);
                if (t == TDPO_BISECTOR) {
                    normalize(&vx);
                    vz = add(vz, vx);
                    normalize(&vz);
                } else if (t == TDPO_ZBISECT) {
                    normalize(&vx);
                    vy = sub(ld(s->pos + 3 * y), pi);
                    normalize(&vy);
                    vx = add(vx, vy);
                    normalize(&vx);
                } else if (t == TDPO_THREEFOLD) {
                    normalize(&vx);
                    vy = sub(ld(s->pos + 3 * y), pi);
                    normalize(&vy);
                    vz = add(vz, add(vx, vy));
                    normalize(&vz);
                }
            }
            double dt = dot(vz, vx);
            vx = sub(vx, scl(vz, dt));
            normalize(&vx);
            vy = cross(vz, vx);
            v3 rows[3] = {vx, vy, vz};
            v3 o;
            for (int c = 0; c < 3; c++) {
                o.v[c] = 0.0;
                for (int r = 0; r < 3; r++) o.v[c] += d.v[r] * rows[r].v[c];
            }
            d = o;
        }
        lab[3 * i] = d.v[0];
        lab[3 * i + 1] = d.v[1];
        lab[3 * i + 2] = d.v[2];
    }
    return 0;
}

/* getAndScaleInverseRs with rrI.size()==2, RTDF.cpp:646-676. */
static inline void inverse_rs(double ti, double tj, double r, double* rr3, double* rr5) {
    double rI = 1.0 / r;
    double r2I = rI * rI;
    double a3 = rI * r2I;
    double a5 = 3.0 * a3 * r2I;
    double damp = ti * tj;
    if (damp != 0.0) {
        double pgamma = ti < tj ? ti : tj;
        double ratio = r / damp;
        ratio = ratio * ratio * ratio;
        damp = -pgamma * ratio;
        if (damp > -50.0) {
            double e = exp(damp);
            a3 *= 1.0 - e;
            a5 *= 1.0 - (1.0 - damp) * e;
        }
    }
    *rr3 = a3;
    *rr5 = a5;
}

/* calculateFixedDipoleField / ...PairIxn, RTDF.cpp:678-733. */
int tdpo_fixed_field(const tdpo_system* s, const double* lab, double* field) {
    memset(field, 0, sizeof(double) * 3 * (size_t)s->n);
    for (int i = 0; i < s->n; i++) {
        v3 pi = ld(s->pos + 3 * i), mi = ld(lab + 3 * i);
        double qi = s->charge[i], ti = s->thole[i];
        for (int j = i + 1; j < s->n; j++) {
            double m = mscale(s, i, j);
            v3 dr = periodic(s, sub(ld(s->pos + 3 * j), pi));
            double r = sqrt(dot(dr, dr));
            double rr3, rr5;
            inverse_rs(ti, s->thole[j], r, &rr3, &rr5);
            v3 mj = ld(lab + 3 * j);
            double fj = rr3 * s->charge[j] - rr5 * dot(mj, dr);
            v3 fieldJ = add(scl(dr, fj), scl(mj, rr3));
            v3 fi3 = sub(ld(field + 3 * i), scl(fieldJ, m));
            double fi = rr3 * qi + rr5 * dot(mi, dr);
            v3 fieldI = sub(scl(dr, fi), scl(mi, rr3));
            v3 fj3 = add(ld(field + 3 * j), scl(fieldI, m));
            for (int c = 0; c < 3; c++) { field[3 * i + c] = fi3.v[c]; field[3 * j + c] = fj3.v[c]; }
        }
    }
    return 0;
}

/* calculateInducedDipoleFields / calculateInducedDipolePairIxn,
 * RTDF.cpp:766-818: field = T mu. */
int tdpo_induced_field(const tdpo_system* s, const double* mu, double* field) {
    memset(field, 0, sizeof(double) * 3 * (size_t)s->n);
    for (int i = 0; i < s->n; i++) {
        v3 pi = ld(s->pos + 3 * i);
        for (int j = i + 1; j < s->n; j++) {
            v3 dr = periodic(s, sub(ld(s->pos + 3 * j), pi));
            double r = sqrt(dot(dr, dr));
            double a3, a5;
            inverse_rs(s->thole[i], s->thole[j], r, &a3, &a5);
            double rr3 = -a3, rr5 = a5;
            double sc = iscale(s, i, j);
            if (sc != 0.0) {
                rr3 *= sc;
                rr5 *= sc;
                v3 mj = ld(mu + 3 * j), mi = ld(mu + 3 * i);
                double dd = rr5 * dot(mj, dr);
                v3 a = add(ld(field + 3 * i), add(scl(mj, rr3), scl(dr, dd)));
                dd = rr5 * dot(mi, dr);
                v3 b = add(ld(field + 3 * j), add(scl(mi, rr3), scl(dr, dd)));
                for (int c = 0; c < 3; c++) { field[3 * i + c] = a.v[c]; field[3 * j + c] = b.v[c]; }
            }
        }
    }
    return 0;
}

/* calculateInducedDipoles (RTDF.cpp:735-764) with the Jacobi loop of
 * convergeInducedDipolesByDIIS (:820-851) and the perturbation-theory
 * extrapolation of convergeInducedDipolesByExtrapolation (:853-909). */
int tdpo_induced_dipoles(const tdpo_system* s, const double* lab, double* fixed_field,
                         double* mu, tdpo_stats* st) {
    int n = s->n;
    tdpo_fixed_field(s, lab, fixed_field);
    for (int i = 0; i < 3 * n; i++) mu[i] = fixed_field[i] * s->polarity[i / 3];
    st->iterations = 0;
    st->epsilon = 1.0e+50;
    st->converged = 0;
    if (s->polarization == TDPO_DIRECT) {
        st->converged = 1;
        return 0;
    }
    double* f = (double*)malloc(sizeof(double) * 3 * (size_t)(n > 0 ? n : 1));
    if (s->polarization == TDPO_MUTUAL) {
        double eps = 1.0;
        int it;
        for (it = 0; it < s->max_iter && eps > s->target_eps; it++) {
            tdpo_induced_field(s, mu, f);
            eps = 0.0;
            for (int i = 0; i < n; i++) {
                v3 nw = scl(add(ld(fixed_field + 3 * i), ld(f + 3 * i)), s->polarity[i]);
                v3 dl = sub(nw, ld(mu + 3 * i));
                eps += dot(dl, dl);
                for (int c = 0; c < 3; c++) mu[3 * i + c] = nw.v[c];
            }
            eps = sqrt(eps / (double)(unsigned)n);
        }
        st->iterations = it;
        st->epsilon = eps;
        st->converged = eps < s->target_eps ? 1 : 0;
    } else if (s->polarization == TDPO_EXTRAPOLATED) {
        static const double opt4[4] = {-0.154, 0.017, 0.658, 0.474};
        int k = s->n_extrap > 0 ? s->n_extrap : 4;
        const double* c = s->n_extrap > 0 ? s->extrap : opt4;
        double* hist = (double*)malloc(sizeof(double) * 3 * (size_t)n * (size_t)k + 8);
        memcpy(hist, mu, sizeof(double) * 3 * (size_t)n);
        for (int o = 1; o < k; o++) {
            tdpo_induced_field(s, mu, f);
            for (int i = 0; i < 3 * n; i++) {
                mu[i] = (fixed_field[i] + f[i]) * s->polarity[i / 3];
                hist[(size_t)o * 3 * n + i] = mu[i];
            }
        }
        for (int i = 0; i < 3 * n; i++) {
            double acc = 0.0;
            for (int o = 0; o < k; o++) acc += hist[(size_t)o * 3 * n + i] * c[o];
            mu[i] = acc;
        }
        tdpo_induced_field(s, mu, f);
        double eps = 0.0;
        for (int i = 0; i < n; i++) {
            v3 nw = scl(add(ld(fixed_field + 3 * i), ld(f + 3 * i)), s->polarity[i]);
            v3 dl = sub(nw, ld(mu + 3 * i));
            eps += dot(dl, dl);
        }
        st->epsilon = sqrt(eps / (double)(unsigned)n);
        st->converged = 1;
        st->iterations = k;
        free(hist);
    }
    free(f);
    return 0;
}

/* calculateElectrostaticPairIxn, RTDF.cpp:129-366, including
 * formQIRotationMatrix (:573-607).  Adds into forces/torques, returns the pair
 * energy.  The frame convention is reproduced as written: rows are [X, Y, Z]
 * with Z along the bond, and the multipole algebra treats row 0 as the bond
 * axis (see :237-292), with the axis-permuting back rotation of :150-159. */
static double pair_electrostatic(const tdpo_system* s, int I, int K, const double* lab,
                                 const double* ind, double mScale, double iScale,
                                 double* forces, double* torques) {
    v3 pI = ld(s->pos + 3 * I), pK = ld(s->pos + 3 * K);
    v3 dr = periodic(s, sub(pK, pI));
    double r2 = dot(dr, dr);
    double r = sqrt(r2);

    v3 vz = scl(dr, 1.0 / r);
    v3 vx = vz;
    if (pI.v[1] != pK.v[1] || pI.v[2] != pK.v[2]) vx.v[0] += 1.0;
    else vx.v[1] += 1.0;
    double dt = dot(vz, vx);
    vx = sub(vx, scl(vz, dt));
    normalize(&vx);
    v3 vy = cross(vz, vx);
    double R[3][3] = {{vx.v[0], vx.v[1], vx.v[2]}, {vy.v[0], vy.v[1], vy.v[2]}, {vz.v[0], vz.v[1], vz.v[2]}};
    double FR[3][3] = {{R[1][1], R[2][1], R[0][1]}, {R[1][2], R[2][2], R[0][2]}, {R[1][0], R[2][0], R[0][0]}};

    double uI[3], uJ[3], QI[4], QJ[4];
    for (int a = 0; a < 3; a++) {
        uI[a] = 0.0; uJ[a] = 0.0;
        for (int b = 0; b < 3; b++) {
            uI[a] += R[a][b] * ind[3 * I + b];
            uJ[a] += R[a][b] * ind[3 * K + b];
        }
    }
    QI[0] = s->charge[I];
    QJ[0] = s->charge[K];
    for (int a = 0; a < 3; a++) {
        QI[a + 1] = 0.0; QJ[a + 1] = 0.0;
        for (int b = 0; b < 3; b++) {
            QI[a + 1] += R[a][b] * lab[3 * I + b];
            QJ[a + 1] += R[a][b] * lab[3 * K + b];
        }
    }
    double QIX[4] = {0.0, QI[3], 0.0, -QI[1]}, QIY[4] = {0.0, -QI[2], QI[1], 0.0}, QIZ[4] = {0.0, 0.0, -QI[3], QI[2]};
    double QJX[4] = {0.0, QJ[3], 0.0, -QJ[1]}, QJY[4] = {0.0, -QJ[2], QJ[1], 0.0}, QJZ[4] = {0.0, 0.0, -QJ[3], QJ[2]};

    double rInv = 1.0 / r;
    double rv[5];
    rv[0] = 0.0;
    rv[1] = 1.0 * rInv; /* prefac = _electric/_dielectric = 1 (RTDF.cpp:20-21) */
    rv[2] = rv[1] * rInv;
    rv[3] = rv[2] * rInv;
    /* rInvVec[4]: out-of-bounds read in the reference (see tdp_oracle.h). */
    rv[4] = s->rinv4_mode == TDPO_RINV4_POWER ? rv[3] * rInv : s->rinv4_value;

    double tI = s->thole[I], tK = s->thole[K];
    double dmp = tI * tK;
    double a = tI < tK ? tI : tK;
    double u = r / dmp;
    double au3 = fabs(dmp) > 1.0e-5 ? a * u * u * u : 0.0;
    double expau3 = fabs(dmp) > 1.0e-5 ? exp(-au3) : 0.0;
    double thole_c = 1.0 - expau3;
    double thole_d0 = 1.0 - expau3 * (1.0 + 1.5 * au3);
    double thole_d1 = 1.0 - expau3;
    double dthole_c = 1.0 - expau3 * (1.0 + 1.5 * au3);
    double dthole_d0 = 1.0 - expau3 * (1.0 + au3 + 1.5 * au3 * au3);
    double dthole_d1 = 1.0 - expau3 * (1.0 + au3);

    double Vij[4], Vji[4], VijR[4], VjiR[4], Vijd[3], Vjid[3];
    double ePermCoef = rv[1] * mScale;
    double dPermCoef = -0.5 * mScale * rv[2];
    Vij[0] = ePermCoef * QJ[0];
    Vji[0] = ePermCoef * QI[0];
    VijR[0] = dPermCoef * QJ[0];
    VjiR[0] = dPermCoef * QI[0];

    ePermCoef = rv[2] * mScale;
    double eUIndCoef = rv[2] * iScale * thole_c;
    dPermCoef = -rv[3] * mScale;
    double dUIndCoef = -2.0 * rv[3] * iScale * dthole_c;
    Vij[0] += -(ePermCoef * QJ[1] + eUIndCoef * uJ[0]);
    Vji[1] = -(ePermCoef * QI[0]);
    VijR[0] += -(dPermCoef * QJ[1] + dUIndCoef * uJ[0]);
    VjiR[1] = -(dPermCoef * QI[0]);
    Vjid[0] = -(eUIndCoef * QI[0]);

    Vij[1] = ePermCoef * QJ[0];
    Vji[0] += ePermCoef * QI[1] + eUIndCoef * uI[0];
    VijR[1] = dPermCoef * QJ[0];
    VjiR[0] += dPermCoef * QI[1] + dUIndCoef * uI[0];
    Vijd[0] = eUIndCoef * QJ[0];

    ePermCoef = -2.0 * rv[3] * mScale;
    eUIndCoef = -2.0 * rv[3] * iScale * thole_d0;
    dPermCoef = 3.0 * rv[4] * mScale;
    dUIndCoef = 6.0 * rv[4] * iScale * dthole_d0;
    Vij[1] += ePermCoef * QJ[1] + eUIndCoef * uJ[0];
    Vji[1] += ePermCoef * QI[1] + eUIndCoef * uI[0];
    VijR[1] += dPermCoef * QJ[1] + dUIndCoef * uJ[0];
    VjiR[1] += dPermCoef * QI[1] + dUIndCoef * uI[0];
    Vijd[0] += eUIndCoef * QJ[1];
    Vjid[0] += eUIndCoef * QI[1];

    ePermCoef = rv[3] * mScale;
    eUIndCoef = rv[3] * iScale * thole_d1;
    dPermCoef = -1.5 * rv[4] * mScale;
    dUIndCoef = -3.0 * rv[4] * iScale * dthole_d1;
    Vij[2] = ePermCoef * QJ[2] + eUIndCoef * uJ[1];
    Vji[2] = ePermCoef * QI[2] + eUIndCoef * uI[1];
    VijR[2] = dPermCoef * QJ[2] + dUIndCoef * uJ[1];
    VjiR[2] = dPermCoef * QI[2] + dUIndCoef * uI[1];
    Vijd[1] = eUIndCoef * QJ[2];
    Vjid[1] = eUIndCoef * QI[2];
    Vij[3] = ePermCoef * QJ[3] + eUIndCoef * uJ[2];
    Vji[3] = ePermCoef * QI[3] + eUIndCoef * uI[2];
    VijR[3] = dPermCoef * QJ[3] + dUIndCoef * uJ[2];
    VjiR[3] = dPermCoef * QI[3] + dUIndCoef * uI[2];
    Vijd[2] = eUIndCoef * QJ[3];
    Vjid[2] = eUIndCoef * QI[3];

    double energy = 0.5 * (QI[0] * Vij[0] + QJ[0] * Vji[0]);
    double fIZ = QI[0] * VijR[0];
    double fJZ = QJ[0] * VjiR[0];
    double EIX = 0.0, EIY = 0.0, EIZ = 0.0, EJX = 0.0, EJY = 0.0, EJZ = 0.0;
    for (int k = 1; k < 4; k++) {
        energy += 0.5 * (QI[k] * Vij[k] + QJ[k] * Vji[k]);
        fIZ += QI[k] * VijR[k];
        fJZ += QJ[k] * VjiR[k];
        EIX += QIX[k] * Vij[k];
        EIY += QIY[k] * Vij[k];
        EIZ += QIZ[k] * Vij[k];
        EJX += QJX[k] * Vji[k];
        EJY += QJY[k] * Vji[k];
        EJZ += QJZ[k] * Vji[k];
    }
    double iEIX = uI[2] * Vijd[0] - uI[0] * Vijd[2];
    double iEJX = uJ[2] * Vjid[0] - uJ[0] * Vjid[2];
    double iEIY = uI[0] * Vijd[1] - uI[1] * Vijd[0];
    double iEJY = uJ[0] * Vjid[1] - uJ[1] * Vjid[0];
    if (s->polarization == TDPO_MUTUAL) {
        double eCoef = -4.0 * rv[3] * iScale * thole_d0;
        double dCoef = 6.0 * rv[4] * iScale * dthole_d0;
        iEIX += eCoef * uI[2] * uJ[0];
        iEJX += eCoef * uJ[2] * uI[0];
        iEIY -= eCoef * uI[1] * uJ[0];
        iEJY -= eCoef * uJ[1] * uI[0];
        fIZ += dCoef * uI[0] * uJ[0];
        fJZ += dCoef * uJ[0] * uI[0];
        eCoef = 2.0 * rv[3] * iScale * thole_d1;
        dCoef = -3.0 * rv[4] * iScale * dthole_d1;
        iEIX -= eCoef * uI[0] * uJ[2];
        iEJX -= eCoef * uJ[0] * uI[2];
        iEIY += eCoef * uI[0] * uJ[1];
        iEJY += eCoef * uJ[0] * uI[1];
        fIZ += dCoef * (uI[1] * uJ[1] + uI[2] * uJ[2]);
        fJZ += dCoef * (uJ[1] * uI[1] + uJ[2] * uI[2]);
    }
    double qf[3] = {rInv * (EIY + EJY + iEIY + iEJY), -rInv * (EIX + EJX + iEIX + iEJX), -(fJZ + fIZ)};
    double qtI[3] = {-EIX, -EIY, -EIZ};
    double qtJ[3] = {-EJX, -EJY, -EJZ};
    for (int c = 0; c < 3; c++) {
        double fv = 0.0, tiv = 0.0, tjv = 0.0;
        for (int b = 0; b < 3; b++) {
            fv += FR[c][b] * qf[b];
            tiv += FR[c][b] * qtI[b];
            tjv += FR[c][b] * qtJ[b];
        }
        torques[3 * I + c] += tiv;
        torques[3 * K + c] += tjv;
        forces[3 * I + c] -= fv;
        forces[3 * K + c] += fv;
    }
    return energy;
}

/* calculateElectrostatic, RTDF.cpp:368-393. */
int tdpo_electrostatic(const tdpo_system* s, const double* lab, const double* mu,
                       double* energy, double* forces, double* torques) {
    double e = 0.0;
    for (int i = 0; i < s->n; i++)
        for (int j = i + 1; j < s->n; j++)
            e += pair_electrostatic(s, i, j, lab, mu, mscale(s, i, j), iscale(s, i, j), forces, torques);
    *energy = e;
    return 0;
}

/* mapTorqueToForceForParticle / mapTorqueToForce, RTDF.cpp:915-1115.
 * ZOnly with X < 0: the reference indexes particleData[-1] (:1107, undefined);
 * here the second vector is the unit axis the rotation picks for ZOnly
 * (x-hat unless |u_x| >= 0.866, then y-hat; :491-497) with norm 1. */
static void map_torque_particle(const tdpo_system* s, int i, const double* torque, double* forces) {
    int t = s->axis[4 * i], iz = s->axis[4 * i + 1], ix = s->axis[4 * i + 2], iy = s->axis[4 * i + 3];
    if (t == TDPO_NOAXISTYPE) return;
    v3 pi = ld(s->pos + 3 * i);
    v3 U = sub(ld(s->pos + 3 * iz), pi);
    double normU = normalize(&U);
    v3 V;
    double normV;
    if (ix >= 0) {
        V = sub(ld(s->pos + 3 * ix), pi);
        normV = normalize(&V);
    } else {
        V = fabs(U.v[0]) < 0.866 ? mk(1.0, 0.0, 0.0) : mk(0.0, 1.0, 0.0);
        normV = 1.0;
    }
    v3 W;
    if (iy > -1 && (t == TDPO_ZBISECT || t == TDPO_THREEFOLD)) W = sub(ld(s->pos + 3 * iy), pi);
    else W = cross(U, V);
    double normW = normalize(&W);
    v3 UV = cross(V, U), UW = cross(W, U), VW = cross(W, V);
    normalize(&UV);
    normalize(&UW);
    normalize(&VW);
    double cosUV = dot(U, V), sinUV = sqrt(1.0 - cosUV * cosUV);
    double cosUW = dot(U, W), sinUW = sqrt(1.0 - cosUW * cosUW);
    double cosVW = dot(V, W), sinVW = sqrt(1.0 - cosVW * cosVW);
    v3 T = ld(torque);
    double dphi[3] = {dot(U, T), dot(V, T), dot(W, T)};
    for (int c = 0; c < 3; c++) dphi[c] *= -1.0;
    double* fU = forces + 3 * iz;
    double* fI = forces + 3 * i;
    if (t == TDPO_ZTHENX || t == TDPO_BISECTOR) {
        double* fV = forces + 3 * ix;
        double f1 = dphi[1] / (normU * sinUV);
        double f2 = dphi[2] / normU;
        double f3 = -dphi[0] / (normV * sinUV);
        double f4;
        if (t == TDPO_BISECTOR) {
            f2 *= 0.5;
            f4 = 0.5 * dphi[2] / normV;
        } else {
            f4 = 0.0;
        }
        for (int c = 0; c < 3; c++) {
            double forceU = UV.v[c] * f1 + f2 * UW.v[c];
            fU[c] -= forceU;
            double forceV = UV.v[c] * f3 + f4 * VW.v[c];
            fV[c] -= forceV;
            fI[c] += (forceU + forceV);
        }
    } else if (t == TDPO_ZBISECT) {
        v3 Rv = add(V, W);
        v3 S = cross(U, Rv);
        double normR = normalize(&Rv);
        double normS = normalize(&S);
        (void)normR; (void)normS;
        v3 UR = cross(Rv, U), US = cross(S, U), VS = cross(S, V), WS = cross(S, W);
        normalize(&UR);
        normalize(&US);
        normalize(&VS);
        normalize(&WS);
        double cosUR = dot(U, Rv), sinUR = sqrt(1.0 - cosUR * cosUR);
        double cosUS = dot(U, S), sinUS = sqrt(1.0 - cosUS * cosUS);
        double cosVS = dot(V, S), sinVS = sqrt(1.0 - cosVS * cosVS);
        double cosWS = dot(W, S), sinWS = sqrt(1.0 - cosWS * cosWS);
        (void)sinUS;
        v3 t1 = sub(V, scl(S, cosVS)), t2 = sub(W, scl(S, cosWS));
        normalize(&t1);
        normalize(&t2);
        double ut1cos = dot(U, t1), ut1sin = sqrt(1.0 - ut1cos * ut1cos);
        double ut2cos = dot(U, t2), ut2sin = sqrt(1.0 - ut2cos * ut2cos);
        double dphiR = dot(Rv, T) * (-1.0);
        double dphiS = dot(S, T) * (-1.0);
        double f1 = dphiR / (normU * sinUR);
        double f2 = dphiS / normU;
        double f3 = dphi[0] / (normV * (ut1sin + ut2sin));
        double f4 = dphi[0] / (normW * (ut1sin + ut2sin));
        v3 forceU = add(scl(UR, f1), scl(US, f2));
        v3 forceV = scl(sub(scl(S, sinVS), scl(t1, cosVS)), f3);
        v3 forceW = scl(sub(scl(S, sinWS), scl(t2, cosWS)), f4);
        double* fV = forces + 3 * ix;
        double* fW = forces + 3 * iy;
        for (int c = 0; c < 3; c++) fU[c] -= forceU.v[c];
        for (int c = 0; c < 3; c++) fV[c] -= forceV.v[c];
        for (int c = 0; c < 3; c++) fW[c] -= forceW.v[c];
        v3 tot = add(add(forceU, forceV), forceW);
        for (int c = 0; c < 3; c++) fI[c] += tot.v[c];
    } else if (t == TDPO_THREEFOLD) {
        double* fV = forces + 3 * ix;
        for (int c = 0; c < 3; c++) {
            double du = UW.v[c] * dphi[2] / (normU * sinUW) + UV.v[c] * dphi[1] / (normU * sinUV) -
                        UW.v[c] * dphi[0] / (normU * sinUW) - UV.v[c] * dphi[0] / (normU * sinUV);
            double dv = VW.v[c] * dphi[2] / (normV * sinVW) - UV.v[c] * dphi[0] / (normV * sinUV) -
                        VW.v[c] * dphi[1] / (normV * sinVW) + UV.v[c] * dphi[1] / (normV * sinUV);
            double dw = -UW.v[c] * dphi[0] / (normW * sinUW) - VW.v[c] * dphi[1] / (normW * sinVW) +
                        UW.v[c] * dphi[2] / (normW * sinUW) + VW.v[c] * dphi[2] / (normW * sinVW);
            du /= 3.0;
            dv /= 3.0;
            dw /= 3.0;
            fU[c] -= du;
            fV[c] -= dv;
            if (iy > -1) forces[3 * iy + c] -= dw;
            fI[c] += (du + dv + dw);
        }
    } else if (t == TDPO_ZONLY) {
        for (int c = 0; c < 3; c++) {
            double du = UV.v[c] * dphi[1] / (normU * sinUV) + UW.v[c] * dphi[2] / normU;
            fU[c] -= du;
            fI[c] += du;
        }
    }
}

int tdpo_map_torque(const tdpo_system* s, const double* torques, double* forces) {
    for (int i = 0; i < s->n; i++) map_torque_particle(s, i, torques + 3 * i, forces);
    return 0;
}

/* calculateForceAndEnergy (RTDF.cpp:100-127) via setup (:1117-1155).
 * forces are ADDED to (the kernel wrapper passes the context's force array,
 * ReferenceTholeDipoleKernels.cpp:201-215). */
int tdpo_compute(const tdpo_system* s, double* energy, double* forces, double* mu, double* lab,
                 tdpo_stats* st) {
    int n = s->n;
    int err = tdpo_validate(s);
    if (err) return err;
    size_t bytes = sizeof(double) * 3 * (size_t)(n > 0 ? n : 1);
    double* fixed = (double*)malloc(bytes);
    double* torques = (double*)calloc(3 * (size_t)(n > 0 ? n : 1), sizeof(double));
    tdpo_lab_dipoles(s, lab);
    tdpo_induced_dipoles(s, lab, fixed, mu, st);
    tdpo_electrostatic(s, lab, mu, energy, forces, torques);
    tdpo_map_torque(s, torques, forces);
    free(fixed);
    free(torques);
    return 0;
}

/* calculateElectrostaticPotential / ...ForParticleGridPoint, RTDF.cpp:1315-1372.
 * Bare 1/r and 1/r^3: no damping and no scaling. */
int tdpo_potential(const tdpo_system* s, const double* grid, int ngrid, double* out) {
    int n = s->n;
    size_t bytes = sizeof(double) * 3 * (size_t)(n > 0 ? n : 1);
    double* lab = (double*)malloc(bytes);
    double* mu = (double*)malloc(bytes);
    double* fixed = (double*)malloc(bytes);
    tdpo_stats st;
    int err = tdpo_lab_dipoles(s, lab);
    if (!err) tdpo_induced_dipoles(s, lab, fixed, mu, &st);
    for (int g = 0; !err && g < ngrid; g++) {
        double pot = 0.0;
        v3 gp = ld(grid + 3 * g);
        for (int i = 0; i < n; i++) {
            v3 dr = periodic(s, sub(ld(s->pos + 3 * i), gp));
            double r2 = dot(dr, dr);
            double r = sqrt(r2);
            double rr1 = 1.0 / r, rr2 = rr1 * rr1, rr3 = rr1 * rr2;
            double p = s->charge[i] * rr1;
            double scd = dot(ld(lab + 3 * i), dr);
            double scu = dot(ld(mu + 3 * i), dr);
            p -= (scd + scu) * rr3;
            pot += p;
        }
        out[g] = pot;
    }
    free(lab);
    free(mu);
    free(fixed);
    return err;
}

/* calculateTholeDipoleSystemMultipoleMoments, RTDF.cpp:1225-1313. */
int tdpo_moments(const tdpo_system* s, const double* masses, double* out) {
    int n = s->n;
    size_t bytes = sizeof(double) * 3 * (size_t)(n > 0 ? n : 1);
    double* lab = (double*)malloc(bytes);
    double* mu = (double*)malloc(bytes);
    double* fixed = (double*)malloc(bytes);
    tdpo_stats st;
    int err = tdpo_lab_dipoles(s, lab);
    if (err) { free(lab); free(mu); free(fixed); return err; }
    tdpo_induced_dipoles(s, lab, fixed, mu, &st);
    double totalMass = 0.0;
    v3 com = mk(0, 0, 0);
    for (int i = 0; i < n; i++) {
        totalMass += masses[i];
        com = add(com, scl(ld(s->pos + 3 * i), masses[i]));
    }
    if (totalMass > 0.0) com = scl(com, 1.0 / totalMass);
    double netchg = 0.0;
    v3 dpl = mk(0, 0, 0);
    double xx = 0, xy = 0, xz = 0, yy = 0, yz = 0, zz = 0;
    for (int i = 0; i < n; i++) {
        double q = s->charge[i];
        v3 p = sub(ld(s->pos + 3 * i), com);
        netchg += q;
        v3 nd = add(ld(lab + 3 * i), ld(mu + 3 * i));
        dpl = add(dpl, add(scl(p, q), nd));
        xx += p.v[0] * p.v[0] * q + 2.0 * p.v[0] * nd.v[0];
        xy += p.v[0] * p.v[1] * q + p.v[0] * nd.v[1] + p.v[1] * nd.v[0];
        xz += p.v[0] * p.v[2] * q + p.v[0] * nd.v[2] + p.v[2] * nd.v[0];
        yy += p.v[1] * p.v[1] * q + 2.0 * p.v[1] * nd.v[1];
        yz += p.v[1] * p.v[2] * q + p.v[1] * nd.v[2] + p.v[2] * nd.v[1];
        zz += p.v[2] * p.v[2] * q + 2.0 * p.v[2] * nd.v[2];
    }
    double qave = (xx + yy + zz) / 3.0;
    out[4] = 0.5 * (xx - qave);
    out[5] = 0.5 * xy;
    out[6] = 0.5 * xz;
    out[8] = 0.5 * (yy - qave);
    out[9] = 0.5 * yz;
    out[12] = 0.5 * (zz - qave);
    out[7] = out[5];
    out[10] = out[6];
    out[11] = out[9];
    double debye = 4.80321;
    out[0] = netchg;
    dpl = scl(dpl, 10.0 * debye);
    out[1] = dpl.v[0];
    out[2] = dpl.v[1];
    out[3] = dpl.v[2];
    debye *= 3.0;
    for (int k = 4; k < 13; k++) out[k] *= 100.0 * debye;
    free(lab);
    free(mu);
    free(fixed);
    return 0;
}
