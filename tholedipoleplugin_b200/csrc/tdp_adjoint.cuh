// tdp_adjoint.cuh -- per-pair reverse-mode building blocks of the
// TholeDipoleForce evaluation (reference semantics, FP64), shared by the box
// adjoint (tdp_adjoint.cu) and the batched-cluster adjoint (tdp_batch.cu).
// See tdp_adjoint.cu for the chain they differentiate.
#pragma once

#include "tdp_frames.cuh"
#include "tdp_kernels.cuh"

#include <math.h>

namespace tdp {
namespace adj {

struct Dual {
    double v, d;
};
__device__ __forceinline__ Dual mk(double v, double d = 0.0) { return {v, d}; }
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.v * b.d + a.d * b.v}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
    double iv = 1.0 / b.v;
    return {a.v * iv, (a.d - a.v * iv * b.d) * iv};
}
__device__ __forceinline__ Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
__device__ __forceinline__ Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
__device__ __forceinline__ Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
__device__ __forceinline__ Dual& operator+=(Dual& a, Dual b) { return a = a + b; }
__device__ __forceinline__ Dual& operator-=(Dual& a, Dual b) { return a = a - b; }
__device__ __forceinline__ Dual dexp(Dual a) {
    double e = exp(a.v);
    return {e, e * a.d};
}
__device__ __forceinline__ double dexp(double a) { return exp(a); }
__device__ __forceinline__ double val(double a) { return a; }
__device__ __forceinline__ double val(Dual a) { return a.v; }
__device__ __forceinline__ double der(double) { return 0.0; }
__device__ __forceinline__ double der(Dual a) { return a.d; }
// min(t_i, t_j) of the damping (RTDF.cpp:206, :662).  It has a kink where the
// factors are equal; there the symmetric subgradient is used (each side gets
// half), which is what a central difference sees and which sums to the exact
// derivative when both factors move together.
__device__ __forceinline__ double tmin(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ Dual tmin(Dual a, Dual b) {
    if (a.v < b.v) return a;
    if (b.v < a.v) return b;
    return {a.v, 0.5 * (a.d + b.d)};
}
template <class T> __device__ __forceinline__ T cst(double v);
template <> __device__ __forceinline__ double cst<double>(double v) { return v; }
template <> __device__ __forceinline__ Dual cst<Dual>(double v) { return mk(v); }

template <class T>
struct V3T {
    T x, y, z;
};
typedef V3T<double> V3;
__device__ __forceinline__ V3 ld(const double* p) { return {p[0], p[1], p[2]}; }

// Thole factors of the pair energy routine (RTDF.cpp:204-220).
template <class T>
__device__ __forceinline__ void energy_damping(double r, double r2, double damp_r2, T tI, T tK, T& tc, T& td0, T& td1,
                                               T& dtc, T& dtd0, T& dtd1) {
    tc = td0 = td1 = dtc = dtd0 = dtd1 = cst<T>(1.0);
    if (r2 < damp_r2) {
        T dmp = tI * tK;
        if (fabs(val(dmp)) > 1.0e-5) {
            T a = tmin(tI, tK);
            T u = cst<T>(r) / dmp;
            T au3 = a * u * u * u;
            T e = dexp(-au3);
            tc = 1.0 - e;
            td0 = 1.0 - e * (1.0 + 1.5 * au3);
            td1 = 1.0 - e;
            dtc = 1.0 - e * (1.0 + 1.5 * au3);
            dtd0 = 1.0 - e * (1.0 + au3 + 1.5 * au3 * au3);
            dtd1 = 1.0 - e * (1.0 + au3);
        }
    }
}

// Damped 1/r^3 and 3/r^5 of getAndScaleInverseRs (RTDF.cpp:646-676).
template <class T>
__device__ __forceinline__ void field_damping(double r, double r2, double damp_r2, T ti, T tj, T& rr3, T& rr5) {
    double rI = 1.0 / r, r2I = rI * rI;
    rr3 = cst<T>(rI * r2I);
    rr5 = cst<T>(3.0 * rI * r2I * r2I);
    if (r2 < damp_r2) {
        T dmp = ti * tj;
        if (val(dmp) != 0.0) {
            T pg = tmin(ti, tj);
            T ratio = cst<T>(r) / dmp;
            ratio = ratio * ratio * ratio;
            T damp = -pg * ratio;
            if (val(damp) > -50.0) {
                T e = dexp(damp);
                rr3 = rr3 * (1.0 - e);
                rr5 = rr5 * (1.0 - (1.0 - damp) * e);
            }
        }
    }
}

// One pair of calculateElectrostaticPairIxn in its canonical orientation
// (I lower index, d = p_K - p_I), contracted with the cotangents:
//   l = gE*energy + cf.qf + ctI.qtI + ctK.qtJ
// where cf = FR^T (gF_K - gF_I), ctI = FR^T gT_I, ctK = FR^T gT_K are the
// force/torque cotangents brought into the QI frame.  Same operations and
// frame convention as pair_energy (tdp_pairs.cuh).
template <class T>
__device__ T pair_loss(double dx, double dy, double dz, bool yzd, T qI, const T* mI, const T* uIl, T tI, T qK,
                       const T* mK, const T* uKl, T tK, double mS, double iS, double damp_r2, double rv4p,
                       double rv4f, bool mutual, double gE, V3 gFI, V3 gFK, V3 gTI, V3 gTK) {
    double r2 = dx * dx + dy * dy + dz * dz;
    double r = sqrt(r2);
    double rinv = 1.0 / r;
    double zx = dx * rinv, zy = dy * rinv, zz = dz * rinv;
    double xx = zx, xy = zy, xz = zz;
    if (yzd) xx += 1.0;
    else xy += 1.0;
    double dt = zx * xx + zy * xy + zz * xz;
    xx -= zx * dt;
    xy -= zy * dt;
    xz -= zz * dt;
    double xn = sqrt(xx * xx + xy * xy + xz * xz);
    if (xn > 0.0) {
        xx /= xn;
        xy /= xn;
        xz /= xn;
    }
    double yx = zy * xz - zz * xy, yy = zz * xx - zx * xz, yz = zx * xy - zy * xx;
    // Force rotation rows (Y.y, Z.y, X.y), (Y.z, Z.z, X.z), (Y.x, Z.x, X.x).
    double FR[3][3] = {{yy, zy, xy}, {yz, zz, xz}, {yx, zx, xx}};
    double gd[3] = {gFK.x - gFI.x, gFK.y - gFI.y, gFK.z - gFI.z};
    double gti[3] = {gTI.x, gTI.y, gTI.z}, gtk[3] = {gTK.x, gTK.y, gTK.z};
    double cf[3], cti[3], ctk[3];
    for (int b = 0; b < 3; b++) {
        cf[b] = FR[0][b] * gd[0] + FR[1][b] * gd[1] + FR[2][b] * gd[2];
        cti[b] = FR[0][b] * gti[0] + FR[1][b] * gti[1] + FR[2][b] * gti[2];
        ctk[b] = FR[0][b] * gtk[0] + FR[1][b] * gtk[1] + FR[2][b] * gtk[2];
    }
    T uI0 = xx * uIl[0] + xy * uIl[1] + xz * uIl[2];
    T uI1 = yx * uIl[0] + yy * uIl[1] + yz * uIl[2];
    T uI2 = zx * uIl[0] + zy * uIl[1] + zz * uIl[2];
    T uJ0 = xx * uKl[0] + xy * uKl[1] + xz * uKl[2];
    T uJ1 = yx * uKl[0] + yy * uKl[1] + yz * uKl[2];
    T uJ2 = zx * uKl[0] + zy * uKl[1] + zz * uKl[2];
    T QI0 = qI, QJ0 = qK;
    T QI1 = xx * mI[0] + xy * mI[1] + xz * mI[2];
    T QI2 = yx * mI[0] + yy * mI[1] + yz * mI[2];
    T QI3 = zx * mI[0] + zy * mI[1] + zz * mI[2];
    T QJ1 = xx * mK[0] + xy * mK[1] + xz * mK[2];
    T QJ2 = yx * mK[0] + yy * mK[1] + yz * mK[2];
    T QJ3 = zx * mK[0] + zy * mK[1] + zz * mK[2];
    double rv1 = rinv, rv2 = rv1 * rinv, rv3 = rv2 * rinv;
    double rv4 = rv4p * (rv3 * rinv) + rv4f;
    T tc, td0, td1, dtc, dtd0, dtd1;
    energy_damping<T>(r, r2, damp_r2, tI, tK, tc, td0, td1, dtc, dtd0, dtd1);

    double eP = rv1 * mS, dP = -0.5 * mS * rv2;
    T Vij0 = eP * QJ0, Vji0 = eP * QI0, VijR0 = dP * QJ0, VjiR0 = dP * QI0;
    eP = rv2 * mS;
    T eU = (rv2 * iS) * tc;
    dP = -rv3 * mS;
    T dU = (-2.0 * rv3 * iS) * dtc;
    Vij0 = Vij0 - (eP * QJ1 + eU * uJ0);
    T Vji1 = -(eP * QI0);
    VijR0 = VijR0 - (dP * QJ1 + dU * uJ0);
    T VjiR1 = -(dP * QI0);
    T Vjid0 = -(eU * QI0);
    T Vij1 = eP * QJ0;
    Vji0 = Vji0 + eP * QI1 + eU * uI0;
    T VijR1 = dP * QJ0;
    VjiR0 = VjiR0 + dP * QI1 + dU * uI0;
    T Vijd0 = eU * QJ0;
    eP = -2.0 * rv3 * mS;
    eU = (-2.0 * rv3 * iS) * td0;
    dP = 3.0 * rv4 * mS;
    dU = (6.0 * rv4 * iS) * dtd0;
    Vij1 = Vij1 + eP * QJ1 + eU * uJ0;
    Vji1 = Vji1 + eP * QI1 + eU * uI0;
    VijR1 = VijR1 + dP * QJ1 + dU * uJ0;
    VjiR1 = VjiR1 + dP * QI1 + dU * uI0;
    Vijd0 = Vijd0 + eU * QJ1;
    Vjid0 = Vjid0 + eU * QI1;
    eP = rv3 * mS;
    eU = (rv3 * iS) * td1;
    dP = -1.5 * rv4 * mS;
    dU = (-3.0 * rv4 * iS) * dtd1;
    T Vij2 = eP * QJ2 + eU * uJ1, Vji2 = eP * QI2 + eU * uI1;
    T VijR2 = dP * QJ2 + dU * uJ1, VjiR2 = dP * QI2 + dU * uI1;
    T Vijd1 = eU * QJ2, Vjid1 = eU * QI2;
    T Vij3 = eP * QJ3 + eU * uJ2, Vji3 = eP * QI3 + eU * uI2;
    T VijR3 = dP * QJ3 + dU * uJ2, VjiR3 = dP * QI3 + dU * uI2;
    T Vijd2 = eU * QJ3, Vjid2 = eU * QI3;

    T energy = 0.5 * (QI0 * Vij0 + QJ0 * Vji0) + 0.5 * (QI1 * Vij1 + QJ1 * Vji1) + 0.5 * (QI2 * Vij2 + QJ2 * Vji2) +
               0.5 * (QI3 * Vij3 + QJ3 * Vji3);
    T fIZ = QI0 * VijR0 + QI1 * VijR1 + QI2 * VijR2 + QI3 * VijR3;
    T fJZ = QJ0 * VjiR0 + QJ1 * VjiR1 + QJ2 * VjiR2 + QJ3 * VjiR3;
    T EIX = QI3 * Vij1 - QI1 * Vij3, EIY = QI1 * Vij2 - QI2 * Vij1, EIZ = QI2 * Vij3 - QI3 * Vij2;
    T EJX = QJ3 * Vji1 - QJ1 * Vji3, EJY = QJ1 * Vji2 - QJ2 * Vji1, EJZ = QJ2 * Vji3 - QJ3 * Vji2;
    T iEIX = uI2 * Vijd0 - uI0 * Vijd2, iEJX = uJ2 * Vjid0 - uJ0 * Vjid2;
    T iEIY = uI0 * Vijd1 - uI1 * Vijd0, iEJY = uJ0 * Vjid1 - uJ1 * Vjid0;
    if (mutual) {
        T eC = (-4.0 * rv3 * iS) * td0;
        T dC = (6.0 * rv4 * iS) * dtd0;
        iEIX += eC * uI2 * uJ0;
        iEJX += eC * uJ2 * uI0;
        iEIY -= eC * uI1 * uJ0;
        iEJY -= eC * uJ1 * uI0;
        fIZ += dC * uI0 * uJ0;
        fJZ += dC * uJ0 * uI0;
        eC = (2.0 * rv3 * iS) * td1;
        dC = (-3.0 * rv4 * iS) * dtd1;
        iEIX -= eC * uI0 * uJ2;
        iEJX -= eC * uJ0 * uI2;
        iEIY += eC * uI0 * uJ1;
        iEJY += eC * uJ0 * uI1;
        fIZ += dC * (uI1 * uJ1 + uI2 * uJ2);
        fJZ += dC * (uJ1 * uI1 + uJ2 * uI2);
    }
    T qf0 = rinv * (EIY + EJY + iEIY + iEJY);
    T qf1 = -rinv * (EIX + EJX + iEIX + iEJX);
    T qf2 = -(fJZ + fIZ);
    T l = gE * energy + cf[0] * qf0 + cf[1] * qf1 + cf[2] * qf2;
    l = l - (cti[0] * EIX + cti[1] * EIY + cti[2] * EIZ) - (ctk[0] * EJX + ctk[1] * EJY + ctk[2] * EJZ);
    return l;
}

__device__ __forceinline__ V3 min_image(const PairParams& P, V3 d) {
    if (P.periodic) {
        d.x = fold_d(d.x, P.box[0], P.inv_box[0]);
        d.y = fold_d(d.y, P.box[1], P.inv_box[1]);
        d.z = fold_d(d.z, P.box[2], P.inv_box[2]);
    }
    return d;
}

struct AtomData {
    const double* pos;     // n*3
    const double* q;       // n
    const double* lab;     // n*3
    const double* mu;      // n*3
    const double* thole;   // n
    const double2* yz;     // raw (y, z) for the QI frame test (NULL: taken from pos)
};

template <class T>
__device__ __forceinline__ V3T<T> cross3(V3T<T> a, V3T<T> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T>
__device__ __forceinline__ T dot3(V3T<T> a, V3T<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T>
__device__ __forceinline__ V3T<T> axpy(T a, V3T<T> x, V3T<T> y) { return {a * x.x + y.x, a * x.y + y.y, a * x.z + y.z}; }
template <class T>
__device__ __forceinline__ V3T<T> scl(T a, V3T<T> x) { return {a * x.x, a * x.y, a * x.z}; }
template <class T>
__device__ __forceinline__ V3T<T> add3(V3T<T> a, V3T<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T>
__device__ __forceinline__ V3T<T> sub3v(V3T<T> a, V3T<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
// Transpose of the permuted back rotation: a . perm(v) = permT(a) . v with
// perm(v) = (v_y, v_z, v_x).
template <class T>
__device__ __forceinline__ V3T<T> permT(V3T<T> a) { return {a.z, a.x, a.y}; }
// a / sqrt(x): exact division in FP64, the reciprocal square root in FP32.
__device__ __forceinline__ double div_sqrt(double a, double x) { return a / sqrt(x); }
__device__ __forceinline__ float div_sqrt(float a, float x) { return a * rsqrtf(x); }

// Closed-form VJP of the pair routine for a pair that Thole damping does not
// reach, with unit scales and rInvVec[4] = 0: the derivatives of
//   l = gE e + gF_I . F_I + gF_K . F_K + gT_I . tau_I + gT_K . tau_K
// with respect to one side's (q, m_lab, mu_ind), from the lab-frame form of
// the routine (pair_energy_lab in tdp_pairs.cuh).  With c = permT(gF_K - gF_I),
// D = (X x c)/r, G_side = D - permT(gT_side), tau_s = G_s x m_s,
// sigma_s = D x u_s, kap = 1 (Mutual) or -1, the loss is bilinear in the two
// sides' multipoles and its gradient is written out term by term below.  The
// Thole factors do not enter (their derivative is 0 here).  out[0..6]: dq,
// dm_lab[3], du[3] of side I (side_I) or side K.
template <class T>
__device__ __forceinline__ void pair_vjp_lab(V3T<T> d, T qI, V3T<T> mI, V3T<T> uI, T qK, V3T<T> mK, V3T<T> uK, T kap,
                                             T gE, V3T<T> gFI, V3T<T> gFK, V3T<T> gTI, V3T<T> gTK, bool side_I,
                                             T* out) {
    typedef V3T<T> W;
    const T r2 = dot3(d, d), rinv = div_sqrt(T(1), r2), rv2 = rinv * rinv, rv3 = rv2 * rinv;
    const T rho2 = d.y * d.y + d.z * d.z;
    const T xs = div_sqrt(rinv, rho2);
    const W X = {rho2 * xs, -d.x * d.y * xs, -d.x * d.z * xs};
    const W PI = add3(mI, uI), PK = add3(mK, uK);
    const T QI1 = dot3(X, mI), UI0 = dot3(X, uI), QK1 = dot3(X, mK), UK0 = dot3(X, uK);
    const T PI0 = QI1 + UI0, PK0 = QK1 + UK0;
    const W cf = permT(sub3v(gFK, gFI));
    const W D = scl(rinv, cross3(X, cf));
    const T cX = dot3(cf, X);
    const T w = T(1) + kap;   // dW/du
    if (side_I) {
        const W GI = sub3v(D, permT(gTI)), GK = sub3v(D, permT(gTK));
        const W tauK = cross3(GK, mK), sigK = cross3(D, uK);
        const W WK = axpy(kap, uK, PK);
        const T WK0 = PK0 + kap * UK0;
        const W Vij = axpy(rv2 * qK - T(3) * rv3 * PK0, X, scl(rv3, PK));
        const W Vdij = axpy(rv2 * qK - T(3) * rv3 * WK0, X, scl(rv3, WK));
        const W t2 = axpy(-T(3) * rv3 * dot3(X, tauK), X, scl(rv3, tauK));
        const W t4 = axpy(-T(3) * rv3 * dot3(X, sigK), X, scl(rv3, sigK));
        const T c5 = T(2) * rv3 * cX * qK;
        // Energy partials.
        const T de_q = rinv * qK - T(0.5) * rv2 * (PK0 + QK1);
        const W de_m = axpy(rv2 * qK - T(1.5) * rv3 * (PK0 + QK1), X, scl(T(0.5) * rv3, add3(PK, mK)));
        const W de_u = axpy(T(0.5) * rv2 * qK - T(1.5) * rv3 * QK1, X, scl(T(0.5) * rv3, mK));
        out[0] = gE * de_q - rv2 * (dot3(X, tauK) + dot3(X, sigK)) + cX * (rv2 * qK - T(2) * rv3 * PK0);
        const W gm = add3(add3(scl(gE, de_m), cross3(Vij, GI)), axpy(c5, X, add3(t2, t4)));
        const W gu = add3(add3(scl(gE, de_u), cross3(Vdij, D)), axpy(c5, X, axpy(w, t4, t2)));
        out[1] = gm.x;
        out[2] = gm.y;
        out[3] = gm.z;
        out[4] = gu.x;
        out[5] = gu.y;
        out[6] = gu.z;
    } else {
        const W GI = sub3v(D, permT(gTI)), GK = sub3v(D, permT(gTK));
        const W tauI = cross3(GI, mI), sigI = cross3(D, uI);
        const W WI = axpy(kap, uI, PI);
        const T WI0 = PI0 + kap * UI0;
        const W Vji = axpy(-rv2 * qI - T(3) * rv3 * PI0, X, scl(rv3, PI));
        const W Vdji = axpy(-rv2 * qI - T(3) * rv3 * WI0, X, scl(rv3, WI));
        const W t1 = axpy(-T(3) * rv3 * dot3(X, tauI), X, scl(rv3, tauI));
        const W t3 = axpy(-T(3) * rv3 * dot3(X, sigI), X, scl(rv3, sigI));
        const T c5 = -T(2) * rv3 * cX * qI;
        const T de_q = rinv * qI + T(0.5) * rv2 * (PI0 + QI1);
        const W de_m = axpy(-rv2 * qI - T(1.5) * rv3 * (PI0 + QI1), X, scl(T(0.5) * rv3, add3(PI, mI)));
        const W de_u = axpy(-T(0.5) * rv2 * qI - T(1.5) * rv3 * QI1, X, scl(T(0.5) * rv3, mI));
        out[0] = gE * de_q + rv2 * (dot3(X, tauI) + dot3(X, sigI)) + cX * (rv2 * qI + T(2) * rv3 * PI0);
        const W gm = add3(add3(scl(gE, de_m), cross3(Vji, GK)), axpy(c5, X, add3(t1, t3)));
        const W gu = add3(add3(scl(gE, de_u), cross3(Vdji, D)), axpy(c5, X, axpy(w, t3, t1)));
        out[1] = gm.x;
        out[2] = gm.y;
        out[3] = gm.z;
        out[4] = gu.x;
        out[5] = gu.y;
        out[6] = gu.z;
    }
}

__device__ inline void visit_pair(const PairParams& P, const AtomData& A, const double* g, const double* gT, double gE,
                           int me, int j, double mS, double iS, double* acc) {
    const bool meI = me < j;
    const int I = meI ? me : j, K = meI ? j : me;
    V3 d = min_image(P, {A.pos[3 * K] - A.pos[3 * I], A.pos[3 * K + 1] - A.pos[3 * I + 1],
                         A.pos[3 * K + 2] - A.pos[3 * I + 2]});
    bool yzd;
    if (A.yz) {
        const double2 yzI = A.yz[I], yzK = A.yz[K];
        yzd = (yzI.x != yzK.x) || (yzI.y != yzK.y);
    } else {
        yzd = (A.pos[3 * I + 1] != A.pos[3 * K + 1]) || (A.pos[3 * I + 2] != A.pos[3 * K + 2]);
    }
    V3 gFI = ld(g + 3 * I), gFK = ld(g + 3 * K), gTI = ld(gT + 3 * I), gTK = ld(gT + 3 * K);
    const double rv4p = P.rinv4_power, rv4f = P.rinv4_fill;
    const double damp_r2 = P.damp_r2 == 0.0f ? 0.0 : (double)P.damp_r2;
    const double r2 = d.x * d.x + d.y * d.y + d.z * d.z;
    if (mS == 1.0 && iS == 1.0 && rv4p == 0.0 && rv4f == 0.0 && !(r2 < damp_r2) && yzd &&
        d.y * d.y + d.z * d.z > 0.0) {
        // Beyond the damping range: the closed-form lab-frame VJP (Thole derivative 0).
        double o[7];
        pair_vjp_lab(d, A.q[I], ld(A.lab + 3 * I), ld(A.mu + 3 * I), A.q[K], ld(A.lab + 3 * K), ld(A.mu + 3 * K),
                     P.mutual ? 1.0 : -1.0, gE, gFI, gFK, gTI, gTK, meI, o);
        for (int a = 0; a < 7; a++) acc[a] += o[a];
        return;
    }
    // Multipole derivatives: the pair function with my multipoles set to unit vectors.
    double oq = A.q[meI ? K : I];
    double om[3] = {A.lab[3 * (meI ? K : I)], A.lab[3 * (meI ? K : I) + 1], A.lab[3 * (meI ? K : I) + 2]};
    double ou[3] = {A.mu[3 * (meI ? K : I)], A.mu[3 * (meI ? K : I) + 1], A.mu[3 * (meI ? K : I) + 2]};
    double tI = A.thole[I], tK = A.thole[K];
    for (int a = 0; a < 7; a++) {
        double bq = a == 0 ? 1.0 : 0.0;
        double bm[3] = {a == 1 ? 1.0 : 0.0, a == 2 ? 1.0 : 0.0, a == 3 ? 1.0 : 0.0};
        double bu[3] = {a == 4 ? 1.0 : 0.0, a == 5 ? 1.0 : 0.0, a == 6 ? 1.0 : 0.0};
        double l = meI ? pair_loss<double>(d.x, d.y, d.z, yzd, bq, bm, bu, tI, oq, om, ou, tK, mS, iS, damp_r2, rv4p,
                                           rv4f, P.mutual, gE, gFI, gFK, gTI, gTK)
                       : pair_loss<double>(d.x, d.y, d.z, yzd, oq, om, ou, tI, bq, bm, bu, tK, mS, iS, damp_r2, rv4p,
                                           rv4f, P.mutual, gE, gFI, gFK, gTI, gTK);
        acc[a] += l;
    }
    // Thole-factor derivative: dual number seeded on my t.
    Dual dq[2], dm[2][3], du[2][3];
    for (int s = 0; s < 2; s++) {
        int at = s == 0 ? I : K;
        dq[s] = mk(A.q[at]);
        for (int c = 0; c < 3; c++) {
            dm[s][c] = mk(A.lab[3 * at + c]);
            du[s][c] = mk(A.mu[3 * at + c]);
        }
    }
    Dual dtI = mk(tI, meI ? 1.0 : 0.0), dtK = mk(tK, meI ? 0.0 : 1.0);
    Dual l = pair_loss<Dual>(d.x, d.y, d.z, yzd, dq[0], dm[0], du[0], dtI, dq[1], dm[1], du[1], dtK, mS, iS, damp_r2,
                             rv4p, rv4f, P.mutual, gE, gFI, gFK, gTI, gTK);
    acc[7] += l.d;
}

template <class T>
__device__ __forceinline__ T lam_dot_field(V3 d, double r, double r2, double damp_r2, T ti, T tk, double qk,
                                           const double* labk, V3 lam_i, double m) {
    T rr3, rr5;
    field_damping<T>(r, r2, damp_r2, ti, tk, rr3, rr5);
    double ld = lam_i.x * d.x + lam_i.y * d.y + lam_i.z * d.z;
    double md = labk[0] * d.x + labk[1] * d.y + labk[2] * d.z;
    double lm = lam_i.x * labk[0] + lam_i.y * labk[1] + lam_i.z * labk[2];
    return -m * (ld * (rr3 * qk - rr5 * md) + rr3 * lm);
}

// Contribution of the pair (i, k) with M scale m to atom k's
// d/d(q_k, lab_k, t_k) of lambda . Efix (k_fixed_vjp), added to acc[5].
// dual = false leaves out the Thole-factor term (acc[4]); fixed_vjp_dual adds
// it alone.
__device__ __forceinline__ void fixed_vjp_visit(const PairParams& P, const AtomData& A, const double* lam, int k,
                                                int i, double m, double* acc, bool dual = true) {
    const double damp_r2 = (double)P.damp_r2;
    const double* labk = A.lab + 3 * k;
    const V3 lk = ld(lam + 3 * k);
    V3 d = min_image(P, {A.pos[3 * k] - A.pos[3 * i], A.pos[3 * k + 1] - A.pos[3 * i + 1],
                         A.pos[3 * k + 2] - A.pos[3 * i + 2]});  // p_k - p_i
    double r2 = d.x * d.x + d.y * d.y + d.z * d.z, r = sqrt(r2);
    V3 li = ld(lam + 3 * i);
    double rr3, rr5;
    field_damping<double>(r, r2, damp_r2, A.thole[i], A.thole[k], rr3, rr5);
    double ldd = li.x * d.x + li.y * d.y + li.z * d.z;
    acc[0] += -m * rr3 * ldd;  // d(lambda_i . f_ik)/dq_k
    acc[1] += m * (rr5 * ldd * d.x - rr3 * li.x);
    acc[2] += m * (rr5 * ldd * d.y - rr3 * li.y);
    acc[3] += m * (rr5 * ldd * d.z - rr3 * li.z);
    // t_k enters f_ik and f_ki (only within the damping range): dual number on t_k.
    if (!dual || !(r2 < damp_r2)) return;
    V3 dn = {-d.x, -d.y, -d.z};
    Dual tk = mk(A.thole[k], 1.0), ti = mk(A.thole[i]);
    Dual s1 = lam_dot_field<Dual>(d, r, r2, damp_r2, ti, tk, A.q[k], labk, li, m);
    Dual s2 = lam_dot_field<Dual>(dn, r, r2, damp_r2, tk, ti, A.q[i], A.lab + 3 * i, lk, m);
    acc[4] += s1.d + s2.d;
}

// The Thole-factor term of fixed_vjp_visit alone (zero beyond the damping range).
__device__ __forceinline__ double fixed_vjp_dual(const PairParams& P, const AtomData& A, const double* lam, int k,
                                                 int i, double m) {
    const double damp_r2 = (double)P.damp_r2;
    V3 d = min_image(P, {A.pos[3 * k] - A.pos[3 * i], A.pos[3 * k + 1] - A.pos[3 * i + 1],
                         A.pos[3 * k + 2] - A.pos[3 * i + 2]});  // p_k - p_i
    const double r2 = d.x * d.x + d.y * d.y + d.z * d.z;
    if (!(r2 < damp_r2)) return 0.0;
    const double r = sqrt(r2);
    const V3 li = ld(lam + 3 * i), lk = ld(lam + 3 * k);
    const V3 dn = {-d.x, -d.y, -d.z};
    Dual tk = mk(A.thole[k], 1.0), ti = mk(A.thole[i]);
    Dual s1 = lam_dot_field<Dual>(d, r, r2, damp_r2, ti, tk, A.q[k], A.lab + 3 * k, li, m);
    Dual s2 = lam_dot_field<Dual>(dn, r, r2, damp_r2, tk, ti, A.q[i], A.lab + 3 * i, lk, m);
    return s1.d + s2.d;
}

// d/dt_k of the pair (k, j) terms of lambda^T T(t) mu with I scale s
// (k_matvec_t_vjp).  Undamped pairs do not depend on t.
__device__ __forceinline__ double matvec_t_visit(const PairParams& P, const AtomData& A, const double* lam, int k,
                                                 int j, double s) {
    const double damp_r2 = (double)P.damp_r2;
    V3 d = min_image(P, {A.pos[3 * j] - A.pos[3 * k], A.pos[3 * j + 1] - A.pos[3 * k + 1],
                         A.pos[3 * j + 2] - A.pos[3 * k + 2]});
    double r2 = d.x * d.x + d.y * d.y + d.z * d.z, r = sqrt(r2);
    if (!(r2 < damp_r2)) return 0.0;
    Dual rr3, rr5;
    field_damping<Dual>(r, r2, damp_r2, mk(A.thole[k], 1.0), mk(A.thole[j]), rr3, rr5);
    V3 lk = ld(lam + 3 * k), uk = ld(A.mu + 3 * k);
    V3 lj = ld(lam + 3 * j), uj = ld(A.mu + 3 * j);
    // lambda_k.(T_kj mu_j) + lambda_j.(T_jk mu_k); T_kj v = -rr3 v + rr5 (v.d) d.
    double a1 = (lk.x * d.x + lk.y * d.y + lk.z * d.z) * (uj.x * d.x + uj.y * d.y + uj.z * d.z);
    double b1 = lk.x * uj.x + lk.y * uj.y + lk.z * uj.z;
    double a2 = (lj.x * d.x + lj.y * d.y + lj.z * d.z) * (uk.x * d.x + uk.y * d.y + uk.z * d.z);
    double b2 = lj.x * uk.x + lj.y * uk.y + lj.z * uk.z;
    Dual v = s * (rr5 * (a1 + a2) - rr3 * (b1 + b2));
    return v.d;
}

}  // namespace adj
}  // namespace tdp
