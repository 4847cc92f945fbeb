// tdp_f32x2.cuh -- packed FP32 arithmetic of sm_100 (f32x2): two FP32 lanes in
// one 64-bit register, so every add/mul/fma instruction serves two pairs.  The
// mixed form's pair walks use it; subnormals are flushed (.ftz), as the scalar
// walks are compiled.
#pragma once

namespace tdp {

typedef unsigned long long f2;
__device__ __forceinline__ f2 pk2(float lo, float hi) {
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ f2 bc2(float v) { return pk2(v, v); }
__device__ __forceinline__ void un2(f2 v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2 add2(f2 a, f2 b) {
    f2 d;
    asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b) {
    f2 d;
    asm("sub.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b) {
    f2 d;
    asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
    f2 d;
    asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ f2 neg2(f2 a) { return mul2(a, bc2(-1.0f)); }
__device__ __forceinline__ f2 dot2(f2 ax, f2 ay, f2 az, f2 bx, f2 by, f2 bz) {
    return fma2(ax, bx, fma2(ay, by, mul2(az, bz)));
}
// Minimum image on both halves: t = rn(d/L) via the 1.5*2^23 constant, d - t L
// (nL = -L).
__device__ __forceinline__ f2 fold2(f2 d, f2 nL, f2 invL) {
    const f2 magic = bc2(12582912.0f), nmagic = bc2(-12582912.0f);
    f2 t = add2(fma2(d, invL, magic), nmagic);
    return fma2(t, nL, d);
}

}  // namespace tdp
