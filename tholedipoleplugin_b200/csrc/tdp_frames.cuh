// tdp_frames.cuh -- FP64 device helpers for the local frames of the
// reference's axis types (aehogan/tholedipoleplugin
// platforms/reference/src/ReferenceTholeDipoleForce.cpp, "RTDF.cpp"): the
// lab-frame rotation rows with the chirality sign, and the torque-to-force
// mapping of one frame role.  Shared by the forward kernels and the adjoint.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace tdp {

struct d3 {
    double x, y, z;
};
__device__ __forceinline__ d3 ld3(const double* p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ d3 operator+(d3 a, d3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ d3 operator-(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ d3 operator*(d3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ d3 cross(d3 a, d3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double normalize(d3& a) {
    double nrm = sqrt(dot(a, a));
    if (nrm > 0.0) a = a * (1.0 / nrm);
    return nrm;
}

// Rows [X, Y, Z] of the local frame of atom i, checkChiral
// (RTDF.cpp:432-467) then applyRotationMatrixToParticle (:477-546): the lab
// dipole is sum_j (S d)_j R[j], with sy = -1 where the chirality check flips
// the y component.  Atoms without a Z atom (or Z == i) get the identity.
__device__ __forceinline__ void frame_rows(const double* __restrict__ pos, int4 ax, int i, double R[3][3],
                                           double& sy) {
    d3 pi = ld3(pos + 3 * i);
    sy = 1.0;
    if (ax.w > -1 && ax.x == 0 /* ZThenX */) {
        d3 py = ld3(pos + 3 * ax.w);
        d3 ad = pi - py, bd = ld3(pos + 3 * ax.y) - py, cd = ld3(pos + 3 * ax.z) - py;
        if (dot(cross(bd, cd), ad) < 0.0) sy = -1.0;
    }
    R[0][0] = 1.0; R[0][1] = 0.0; R[0][2] = 0.0;
    R[1][0] = 0.0; R[1][1] = 1.0; R[1][2] = 0.0;
    R[2][0] = 0.0; R[2][1] = 0.0; R[2][2] = 1.0;
    if (!(ax.y >= 0 && ax.y != i)) return;
    d3 vz = ld3(pos + 3 * ax.y) - pi;
    normalize(vz);
    d3 vx, vy;
    if (ax.x == 4 /* ZOnly */) {
        vx = fabs(vz.x) < 0.866 ? d3{1.0, 0.0, 0.0} : d3{0.0, 1.0, 0.0};
    } else {
        vx = ld3(pos + 3 * ax.z) - pi;
        if (ax.x == 1) {  // Bisector
            normalize(vx);
            vz = vz + vx;
            normalize(vz);
        } else if (ax.x == 2) {  // ZBisect
            normalize(vx);
            vy = ld3(pos + 3 * ax.w) - pi;
            normalize(vy);
            vx = vx + vy;
            normalize(vx);
        } else if (ax.x == 3) {  // ThreeFold
            normalize(vx);
            vy = ld3(pos + 3 * ax.w) - pi;
            normalize(vy);
            vz = vz + (vx + vy);
            normalize(vz);
        }
    }
    double dt = dot(vz, vx);
    vx = vx - vz * dt;
    normalize(vx);
    vy = cross(vz, vx);
    R[0][0] = vx.x; R[0][1] = vx.y; R[0][2] = vx.z;
    R[1][0] = vy.x; R[1][1] = vy.y; R[1][2] = vy.z;
    R[2][0] = vz.x; R[2][1] = vz.y; R[2][2] = vz.z;
}

// ---------------------------------------------------------------------------
// Torque -> force, gather form of mapTorqueToForceForParticle
// (RTDF.cpp:915-1090): atom a sums, over every frame it belongs to, the force
// its role (I, U=Z, V=X, W=Y) receives.  role: 0 I, 1 U, 2 V, 3 W.
// ---------------------------------------------------------------------------
__device__ __forceinline__ d3 torque_role_force(const double* __restrict__ pos, int4 ax, int i, int role, d3 T) {
    const int t = ax.x, iz = ax.y, ix = ax.z, iy = ax.w;
    d3 zero = {0.0, 0.0, 0.0};
    if (t == 5) return zero;
    d3 pi = ld3(pos + 3 * i);
    d3 U = ld3(pos + 3 * iz) - pi;
    double normU = normalize(U);
    d3 V;
    double normV;
    if (ix >= 0) {
        V = ld3(pos + 3 * ix) - pi;
        normV = normalize(V);
    } else {  // ZOnly without an X atom (undefined in the reference): the rotation's fixed axis
        V = fabs(U.x) < 0.866 ? d3{1.0, 0.0, 0.0} : d3{0.0, 1.0, 0.0};
        normV = 1.0;
    }
    d3 W;
    if (iy > -1 && (t == 2 || t == 3)) W = ld3(pos + 3 * iy) - pi;
    else W = cross(U, V);
    double normW = normalize(W);
    d3 UV = cross(V, U), UW = cross(W, U), VW = cross(W, V);
    normalize(UV);
    normalize(UW);
    normalize(VW);
    double cosUV = dot(U, V), sinUV = sqrt(1.0 - cosUV * cosUV);
    double cosUW = dot(U, W), sinUW = sqrt(1.0 - cosUW * cosUW);
    double cosVW = dot(V, W), sinVW = sqrt(1.0 - cosVW * cosVW);
    double dphi0 = dot(U, T) * -1.0, dphi1 = dot(V, T) * -1.0, dphi2 = dot(W, T) * -1.0;
    if (t == 0 || t == 1) {
        double f1 = dphi1 / (normU * sinUV);
        double f2 = dphi2 / normU;
        double f3 = -dphi0 / (normV * sinUV);
        double f4 = 0.0;
        if (t == 1) {
            f2 *= 0.5;
            f4 = 0.5 * dphi2 / normV;
        }
        d3 fU = {UV.x * f1 + f2 * UW.x, UV.y * f1 + f2 * UW.y, UV.z * f1 + f2 * UW.z};
        d3 fV = {UV.x * f3 + f4 * VW.x, UV.y * f3 + f4 * VW.y, UV.z * f3 + f4 * VW.z};
        if (role == 0) return fU + fV;
        if (role == 1) return fU * -1.0;
        if (role == 2) return fV * -1.0;
        return zero;
    }
    if (t == 2) {
        d3 Rv = V + W;
        d3 S = cross(U, Rv);
        normalize(Rv);
        normalize(S);
        d3 UR = cross(Rv, U), US = cross(S, U);
        normalize(UR);
        normalize(US);
        double cosUR = dot(U, Rv), sinUR = sqrt(1.0 - cosUR * cosUR);
        double cosVS = dot(V, S), sinVS = sqrt(1.0 - cosVS * cosVS);
        double cosWS = dot(W, S), sinWS = sqrt(1.0 - cosWS * cosWS);
        d3 t1 = V - S * cosVS, t2 = W - S * cosWS;
        normalize(t1);
        normalize(t2);
        double ut1cos = dot(U, t1), ut1sin = sqrt(1.0 - ut1cos * ut1cos);
        double ut2cos = dot(U, t2), ut2sin = sqrt(1.0 - ut2cos * ut2cos);
        double dphiR = dot(Rv, T) * (-1.0);
        double dphiS = dot(S, T) * (-1.0);
        double f1 = dphiR / (normU * sinUR);
        double f2 = dphiS / normU;
        double f3 = dphi0 / (normV * (ut1sin + ut2sin));
        double f4 = dphi0 / (normW * (ut1sin + ut2sin));
        d3 fU = UR * f1 + US * f2;
        d3 fV = (S * sinVS - t1 * cosVS) * f3;
        d3 fW = (S * sinWS - t2 * cosWS) * f4;
        if (role == 0) return (fU + fV) + fW;
        if (role == 1) return fU * -1.0;
        if (role == 2) return fV * -1.0;
        return fW * -1.0;
    }
    if (t == 3) {
        double du[3], dv[3], dw[3];
        double uwc[3] = {UW.x, UW.y, UW.z}, uvc[3] = {UV.x, UV.y, UV.z}, vwc[3] = {VW.x, VW.y, VW.z};
        for (int c = 0; c < 3; c++) {
            du[c] = uwc[c] * dphi2 / (normU * sinUW) + uvc[c] * dphi1 / (normU * sinUV) -
                    uwc[c] * dphi0 / (normU * sinUW) - uvc[c] * dphi0 / (normU * sinUV);
            dv[c] = vwc[c] * dphi2 / (normV * sinVW) - uvc[c] * dphi0 / (normV * sinUV) -
                    vwc[c] * dphi1 / (normV * sinVW) + uvc[c] * dphi1 / (normV * sinUV);
            dw[c] = -uwc[c] * dphi0 / (normW * sinUW) - vwc[c] * dphi1 / (normW * sinVW) +
                    uwc[c] * dphi2 / (normW * sinUW) + vwc[c] * dphi2 / (normW * sinVW);
            du[c] /= 3.0;
            dv[c] /= 3.0;
            dw[c] /= 3.0;
        }
        if (role == 0) return {du[0] + dv[0] + dw[0], du[1] + dv[1] + dw[1], du[2] + dv[2] + dw[2]};
        if (role == 1) return {-du[0], -du[1], -du[2]};
        if (role == 2) return {-dv[0], -dv[1], -dv[2]};
        if (iy > -1) return {-dw[0], -dw[1], -dw[2]};
        return zero;
    }
    if (t == 4) {
        d3 du = {UV.x * dphi1 / (normU * sinUV) + UW.x * dphi2 / normU,
                 UV.y * dphi1 / (normU * sinUV) + UW.y * dphi2 / normU,
                 UV.z * dphi1 / (normU * sinUV) + UW.z * dphi2 / normU};
        if (role == 0) return du;
        if (role == 1) return du * -1.0;
        return zero;
    }
    return zero;
}

}  // namespace tdp
