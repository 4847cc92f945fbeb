// tdp_sym.cu -- the all-pairs kernels of the box path (permanent field,
// mutual-field matvec, energy/force/torque), each unordered pair evaluated
// once with both of its sides.
//
// Work decomposition.  Atoms form 32-atom tiles and tiles form bands of
// band_tiles tiles.  One CTA (4 warps) owns a band pair (p, q), p <= q, and
// evaluates every tile pair (I in band p, J in band q, I <= J).  A warp holds
// the atoms of its I tile(s) in registers (lane = atom) and walks the atoms of
// J along the diagonals of the tile pair, the J-side sums travelling with them
// from lane to lane by shuffles, so that at the end each lane holds the
// J-side sums of "its" J atom.  The scalar walks (FP64 form, and SLOW tile
// pairs) pair lane l with J atom (l + s) mod 32 at step s.  The mixed form's
// packed walks (f32x2, tdp_f32x2.cuh) pair lane l with J atoms m and m + 16,
// m = (l + s) mod 16, in the two halves of each register; lanes l and l ^ 16
// then hold two copies of the same J sums, added by one xor-16 exchange.
//
// J-side sums of band q.  Field kernels: each warp sums into its own area of
// shared memory, the four areas are added in warp order at the end.  Energy
// kernel: one FP64 area; the warps visit disjoint J tiles within each window
// of band_tiles / 4 steps and a barrier separates the windows, so the order
// of the additions is fixed.
//
// Output.  Plain form: partial sums go to slot s of a [n_bands][components]
// [n_pad] FP64 buffer -- CTA (p, q) writes the I-side sums of band p into
// slot q and the J-side sums of band q into slot p -- and the consumers sum an
// atom's slots in slot order.  Mixed form: every CTA adds its band sums into
// one 64-bit fixed-point accumulator (integer addition, independent of the
// order).  Either way results are bitwise deterministic.
//
// Tile pairs are classified as in the reference's arithmetic requires: FOLD
// where the tiles' extents reach half a box (per-pair minimum image with an
// FP64 fallback near the half-box boundary), DAMP where some pair may lie
// within the Thole damping range, SLOW on the diagonal tile, the ragged last
// tile and tiles holding covalent partners.  In SLOW tile pairs, self and
// padding pairs and the partners are masked out of the diagonal walk; each
// partner pair is then evaluated once per side with its M/I scales.
#include "tdp_frames.cuh"
#include "tdp_f32x2.cuh"
#include "tdp_kernels.cuh"
#include "tdp_pairs.cuh"

#include <math.h>

namespace tdp {

namespace {

constexpr int kSymWarps = 4;
constexpr int kSymThreads = 32 * kSymWarps;
constexpr unsigned kFull = 0xffffffffu;

// Band pair of CTA k, enumerated q = 0, 1, ... and p = 0..q: k = q(q+1)/2 + p.
__device__ __forceinline__ void band_pair(int k, int& p, int& q) {
    int qq = (int)((sqrt(8.0 * (double)k + 1.0) - 1.0) * 0.5);
    while ((qq + 1) * (qq + 2) / 2 <= k) qq++;
    while (qq * (qq + 1) / 2 > k) qq--;
    q = qq;
    p = k - qq * (qq + 1) / 2;
}

// Geometry of a tile pair: displacement of J's centre from I's (FP64, minimum
// image), whether any pair needs per-pair folding, whether any pair can be
// within the damping range.
struct TileGeom {
    double dcx, dcy, dcz;
    bool fold;
    bool near;
    unsigned fmask;   // dimensions in which some pair may need folding (bit k: dimension k)
};

__device__ __forceinline__ TileGeom tile_geom(const PairParams& P, double4 cA, double4 eA, double4 cB, double4 eB) {
    TileGeom g;
    g.dcx = cB.x - cA.x;
    g.dcy = cB.y - cA.y;
    g.dcz = cB.z - cA.z;
    g.fold = false;
    g.fmask = 0u;
    if (P.periodic) {
        g.dcx = fold_d(g.dcx, P.box[0], P.inv_box[0]);
        g.dcy = fold_d(g.dcy, P.box[1], P.inv_box[1]);
        g.dcz = fold_d(g.dcz, P.box[2], P.inv_box[2]);
        g.fmask = (fabs(g.dcx) + eA.x + eB.x >= P.half_box_tol[0] ? 1u : 0u) |
                  (fabs(g.dcy) + eA.y + eB.y >= P.half_box_tol[1] ? 2u : 0u) |
                  (fabs(g.dcz) + eA.z + eB.z >= P.half_box_tol[2] ? 4u : 0u);
        g.fold = fabs(g.dcx) + eA.x + eB.x >= P.half_box_tol[0] || fabs(g.dcy) + eA.y + eB.y >= P.half_box_tol[1] ||
                 fabs(g.dcz) + eA.z + eB.z >= P.half_box_tol[2];
    }
    // Smallest minimum-image distance any pair of the two tiles can have: per
    // dimension the periodic distance is a metric, so it is at least the
    // centres' folded distance minus both extents.
    double gx = fmax(fabs(g.dcx) - eA.x - eB.x, 0.0);
    double gy = fmax(fabs(g.dcy) - eA.y - eB.y, 0.0);
    double gz = fmax(fabs(g.dcz) - eA.z - eB.z, 0.0);
    g.near = gx * gx + gy * gy + gz * gz < (double)P.damp_r2;
    return g;
}

// Exact FP64 minimum-image displacement p_j - p_i (the reference's own
// arithmetic), for FP32 pairs near the half-box.
__device__ __forceinline__ d3 exact_delta(const PairParams& P, const double* __restrict__ pos, int i, int j) {
    d3 d = ld3(pos + 3 * j) - ld3(pos + 3 * i);
    if (P.periodic) {
        d.x = fold_d(d.x, P.box[0], P.inv_box[0]);
        d.y = fold_d(d.y, P.box[1], P.inv_box[1]);
        d.z = fold_d(d.z, P.box[2], P.inv_box[2]);
    }
    return d;
}

// p_j - p_i from j's record (its own tile frame) and i's record shifted into
// that frame.
template <class R, bool FOLD>
__device__ __forceinline__ void pair_delta(const PairParams& P, const double* __restrict__ pos, int i, int j, R pjx,
                                           R pjy, R pjz, R oix, R oiy, R oiz, R& dx, R& dy, R& dz) {
    dx = pjx - oix;
    dy = pjy - oiy;
    dz = pjz - oiz;
    if (FOLD) {
        if (sizeof(R) == 4) {
            dx = (R)fold_f((float)dx, (float)P.box[0], (float)P.inv_box[0]);
            dy = (R)fold_f((float)dy, (float)P.box[1], (float)P.inv_box[1]);
            dz = (R)fold_f((float)dz, (float)P.box[2], (float)P.inv_box[2]);
            if ((fabs(dx) > (R)P.half_box_tol[0] || fabs(dy) > (R)P.half_box_tol[1] ||
                 fabs(dz) > (R)P.half_box_tol[2]) && i < P.n && j < P.n) {
                d3 e = exact_delta(P, pos, i, j);
                dx = (R)e.x;
                dy = (R)e.y;
                dz = (R)e.z;
            }
        } else {
            dx = (R)fold_d((double)dx, P.box[0], P.inv_box[0]);
            dy = (R)fold_d((double)dy, P.box[1], P.inv_box[1]);
            dz = (R)fold_d((double)dz, P.box[2], P.inv_box[2]);
        }
    }
}

// The record of an I-tile atom shifted into J's frame.  FP32: offsets from the
// tile centres, shifted by the minimum-image centre displacement; FP64:
// absolute positions, shifted by the whole-box image the tile pair chose.
template <class R>
__device__ __forceinline__ void shift_into(const TileGeom& g, double4 cA, double4 cB, R px, R py, R pz, R& ox, R& oy,
                                           R& oz) {
    if (sizeof(R) == 4) {
        ox = px - (R)g.dcx;
        oy = py - (R)g.dcy;
        oz = pz - (R)g.dcz;
    } else {
        ox = px + (R)((cB.x - cA.x) - g.dcx);
        oy = py + (R)((cB.y - cA.y) - g.dcy);
        oz = pz + (R)((cB.z - cA.z) - g.dcz);
    }
}

// Pairs of the diagonal walk that are left out: self, padding, listed
// partners, and on the diagonal tile the second visit of every pair (steps
// 17..31 and the upper half of step 16 repeat steps 15..1 and 16).
__device__ __forceinline__ bool skip_pair(int s, int lane, int i, int j, int n, unsigned partners, int jj, bool diag) {
    bool skip = i >= n || j >= n || ((partners >> jj) & 1u);
    if (diag) skip = skip || s == 0 || s > 16 || (s == 16 && lane >= 16);
    return skip;
}

// Bits of the J-tile atoms listed as covalent partners of atom i.
__device__ __forceinline__ unsigned partner_bits(const int* __restrict__ exc_j, int e0, int e1, int jbase) {
    unsigned b = 0u;
    for (int e = e0; e < e1; e++) {
        unsigned off = (unsigned)(exc_j[e] - jbase);
        if (off < 32u) b |= 1u << off;
    }
    return b;
}

// 64-bit fixed-point accumulator of the mixed form (Dev::fixacc).
struct FixAcc {
    unsigned long long* acc;
    int* err;
    double scale, limit;
};

// Adds v to the accumulator word; a sum at or beyond the limit (or not finite)
// flags the error instead of wrapping.
__device__ __forceinline__ void fix_add(const FixAcc& F, size_t k, double v) {
    if (v == 0.0) return;
    if (!(fabs(v) < F.limit)) {
        atomicExch(F.err, 1);
        return;
    }
    atomicAdd(F.acc + k, (unsigned long long)__double2ll_rn(v * F.scale));
}

// ---------------------------------------------------------------------------
// Field kernels: KIND 0 = permanent field (records: posq + lab dipole/thole),
// KIND 1 = mutual-field matvec T*v (records: posq + v/thole).
// ---------------------------------------------------------------------------
template <class R, int KIND, bool FOLD, bool SLOW, bool DAMP>
__device__ __forceinline__ void field_walk(const PairParams& P, const double* __restrict__ pos,
                                           const typename Vec4T<R>::type* __restrict__ sp,
                                           const typename Vec4T<R>::type* __restrict__ sv, int lane, int i, int jbase,
                                           R oix, R oiy, R oiz, R qi, typename Vec4T<R>::type vi, bool diag,
                                           unsigned partners, R damp_r2, R& fx, R& fy, R& fz, R& gx, R& gy, R& gz) {
    const int nxt = (lane + 1) & 31;
#pragma unroll 2
    for (int s = 0; s < 32; s++) {
        const int jj = (lane + s) & 31;
        const typename Vec4T<R>::type pj = sp[jj];
        const typename Vec4T<R>::type vj = sv[jj];
        const int j = jbase + jj;
        R dx, dy, dz;
        pair_delta<R, FOLD>(P, pos, i, j, pj.x, pj.y, pj.z, oix, oiy, oiz, dx, dy, dz);
        R r2 = dx * dx + dy * dy + dz * dz;
        if (SLOW && skip_pair(s, lane, i, j, P.n, partners, jj, diag)) r2 = (R)INFINITY;
        if (KIND == 0)
            pair_fixed2<R, DAMP>(dx, dy, dz, r2, qi, vi.x, vi.y, vi.z, pj.w, vj.x, vj.y, vj.z, vi.w, vj.w, damp_r2, fx,
                                 fy, fz, gx, gy, gz);
        else
            pair_matvec2<R, DAMP>(dx, dy, dz, r2, vi.x, vi.y, vi.z, vj.x, vj.y, vj.z, vi.w, vj.w, damp_r2, fx, fy, fz,
                                  gx, gy, gz);
        gx = __shfl_sync(kFull, gx, nxt);
        gy = __shfl_sync(kFull, gy, nxt);
        gz = __shfl_sync(kFull, gz, nxt);
    }
}

// Two I tiles against the same J tile: every J record read from shared
// memory and every shuffle of the J-side sums serves two pairs, and the two
// pair evaluations are independent instruction streams.
template <class R, int KIND, bool FOLD, bool SLOW, bool DAMP>
__device__ __forceinline__ void field_walk2(const PairParams& P, const double* __restrict__ pos,
                                            const typename Vec4T<R>::type* __restrict__ sp,
                                            const typename Vec4T<R>::type* __restrict__ sv, int lane, int jbase,
                                            int ia, R oax, R oay, R oaz, R qa, typename Vec4T<R>::type va, bool diag_a,
                                            unsigned part_a, int ib, R obx, R oby, R obz, R qb,
                                            typename Vec4T<R>::type vb, bool diag_b, unsigned part_b, R damp_r2,
                                            R* fa, R* fb, R* g) {
    const int nxt = (lane + 1) & 31;
#pragma unroll 2
    for (int s = 0; s < 32; s++) {
        const int jj = (lane + s) & 31;
        const typename Vec4T<R>::type pj = sp[jj];
        const typename Vec4T<R>::type vj = sv[jj];
        const int j = jbase + jj;
        R dax, day, daz, dbx, dby, dbz;
        pair_delta<R, FOLD>(P, pos, ia, j, pj.x, pj.y, pj.z, oax, oay, oaz, dax, day, daz);
        pair_delta<R, FOLD>(P, pos, ib, j, pj.x, pj.y, pj.z, obx, oby, obz, dbx, dby, dbz);
        R ra = dax * dax + day * day + daz * daz;
        R rb = dbx * dbx + dby * dby + dbz * dbz;
        if (SLOW) {
            if (skip_pair(s, lane, ia, j, P.n, part_a, jj, diag_a)) ra = (R)INFINITY;
            if (skip_pair(s, lane, ib, j, P.n, part_b, jj, diag_b)) rb = (R)INFINITY;
        }
        if (KIND == 0) {
            pair_fixed2<R, DAMP>(dax, day, daz, ra, qa, va.x, va.y, va.z, pj.w, vj.x, vj.y, vj.z, va.w, vj.w,
                                 damp_r2, fa[0], fa[1], fa[2], g[0], g[1], g[2]);
            pair_fixed2<R, DAMP>(dbx, dby, dbz, rb, qb, vb.x, vb.y, vb.z, pj.w, vj.x, vj.y, vj.z, vb.w, vj.w,
                                 damp_r2, fb[0], fb[1], fb[2], g[0], g[1], g[2]);
        } else {
            pair_matvec2<R, DAMP>(dax, day, daz, ra, va.x, va.y, va.z, vj.x, vj.y, vj.z, va.w, vj.w, damp_r2, fa[0],
                                  fa[1], fa[2], g[0], g[1], g[2]);
            pair_matvec2<R, DAMP>(dbx, dby, dbz, rb, vb.x, vb.y, vb.z, vj.x, vj.y, vj.z, vb.w, vj.w, damp_r2, fb[0],
                                  fb[1], fb[2], g[0], g[1], g[2]);
        }
        g[0] = __shfl_sync(kFull, g[0], nxt);
        g[1] = __shfl_sync(kFull, g[1], nxt);
        g[2] = __shfl_sync(kFull, g[2], nxt);
    }
}

// ---------------------------------------------------------------------------
// Packed FP32 walk over J-atom pairs: the halves of every 64-bit register are
// J atoms m and m + 16 of the tile (records pair-interleaved in a per-warp
// shared tile), so the I-side operands are loop-invariant broadcasts and the
// J-side sums stay packed.  Lane l takes pair m = (l + s) & 15 at step s and
// passes its packed J-side sums one lane on; lanes l and l ^ 16 hold two
// partial copies of the same pair, added by one xor-16 exchange at the end.
// Each lane carries one or two I atoms (slots a and b), each with the pair
// arithmetic of pair_delta + pair_matvec2 / pair_fixed2 per half.
// ---------------------------------------------------------------------------
struct FPackedTile {
    float4 p0[16], p1[16];   // (x, x', y, y'), (z, z', q, q')   (' = atom m + 16)
    float4 v0[16], v1[16];   // (vx, vx', vy, vy'), (vz, vz', t, t')
};

__device__ __forceinline__ void stage_fpacked(FPackedTile& T, int lane, float4 p, float4 v) {
    const int m = lane & 15, h = lane >> 4;
    float* p0 = reinterpret_cast<float*>(&T.p0[m]);
    float* p1 = reinterpret_cast<float*>(&T.p1[m]);
    float* v0 = reinterpret_cast<float*>(&T.v0[m]);
    float* v1 = reinterpret_cast<float*>(&T.v1[m]);
    p0[h] = p.x;
    p0[2 + h] = p.y;
    p1[h] = p.z;
    p1[2 + h] = p.w;
    v0[h] = v.x;
    v0[2 + h] = v.y;
    v1[h] = v.z;
    v1[2 + h] = v.w;
}

// Loop-invariant operands of one I atom.
struct XSlot {
    f2 OX, OY, OZ, VX, VY, VZ, NQ;   // NQ = -q
    float t;
    int i;
};

__device__ __forceinline__ XSlot xslot(int i, float ox, float oy, float oz, float q, float4 v) {
    XSlot x;
    x.OX = bc2(ox);
    x.OY = bc2(oy);
    x.OZ = bc2(oz);
    x.VX = bc2(v.x);
    x.VY = bc2(v.y);
    x.VZ = bc2(v.z);
    x.NQ = bc2(-q);
    x.t = v.w;
    x.i = i;
    return x;
}

// One I atom against J atoms (m, m + 16): I-side sums into F*, J-side into G*,
// both with the opposite sign of the field (the walk's caller flips them), so
// that every term is a plain product-sum with -rr5.
template <int KIND, bool FOLD, bool DAMP>
__device__ __forceinline__ void xslot_pairs(const PairParams& P, const double* __restrict__ pos, const XSlot& x,
                                            int ja, f2 PX, f2 PY, f2 PZ, f2 QJ, f2 VJX, f2 VJY, f2 VJZ, float tja,
                                            float tjb, unsigned fm, f2 Lx, f2 Ly, f2 Lz, f2 Ix, f2 Iy, f2 Iz,
                                            f2 NTx, f2 NTy, f2 NTz, float damp_r2, f2& FX, f2& FY, f2& FZ,
                                            f2& GX, f2& GY, f2& GZ) {
    f2 DX = sub2(PX, x.OX), DY = sub2(PY, x.OY), DZ = sub2(PZ, x.OZ);
    if (FOLD) {
        // Fold the dimensions of fm.  Q = d^2 - t^2 (t = half a box minus 16
        // ulp) is negative unless the pair lies within the margin of half a
        // box; AND-ing the Q words keeps sign bits 31 (low half) and 63 (high
        // half) set only if every Q of that half is negative.
        f2 neg = ~0ull;
        if (fm & 1u) {
            DX = fold2(DX, Lx, Ix);
            neg &= fma2(DX, DX, NTx);
        }
        if (fm & 2u) {
            DY = fold2(DY, Ly, Iy);
            neg &= fma2(DY, DY, NTy);
        }
        if (fm & 4u) {
            DZ = fold2(DZ, Lz, Iz);
            neg &= fma2(DZ, DZ, NTz);
        }
        const f2 flag = ~neg & 0x8000000080000000ull;
        if (flag) {
            const bool amb_a = (flag >> 31) & 1ull, amb_b = (flag >> 63) != 0ull;
            float ax, bx, ay, by, az, bz;
            un2(DX, ax, bx);
            un2(DY, ay, by);
            un2(DZ, az, bz);
            // Within 16 ulp of half a box: the reference's FP64 minimum image.
            if (amb_a && x.i < P.n && ja < P.n) {
                d3 e = exact_delta(P, pos, x.i, ja);
                ax = (float)e.x;
                ay = (float)e.y;
                az = (float)e.z;
            }
            if (amb_b && x.i < P.n && ja + 16 < P.n) {
                d3 e = exact_delta(P, pos, x.i, ja + 16);
                bx = (float)e.x;
                by = (float)e.y;
                bz = (float)e.z;
            }
            DX = pk2(ax, bx);
            DY = pk2(ay, by);
            DZ = pk2(az, bz);
        }
    }
    const f2 R2 = fma2(DX, DX, fma2(DY, DY, mul2(DZ, DZ)));
    float r2a, r2b;
    un2(R2, r2a, r2b);
    const f2 RINV = pk2(rsqrt_r(r2a), rsqrt_r(r2b));
    const f2 RINV2 = mul2(RINV, RINV);
    f2 RR3 = mul2(RINV, RINV2);
    f2 NRR5 = mul2(RR3, mul2(RINV2, bc2(-3.0f)));   // -rr5
    if (DAMP) {
        if (r2a < damp_r2 || r2b < damp_r2) {
            float ra, rb, r3a, r3b, r5a, r5b;
            un2(RINV, ra, rb);
            un2(RR3, r3a, r3b);
            un2(NRR5, r5a, r5b);
            r5a = -r5a;
            r5b = -r5b;
            damp_field<float>(r2a, ra, x.t, tja, damp_r2, r3a, r5a);
            damp_field<float>(r2b, rb, x.t, tjb, damp_r2, r3b, r5b);
            RR3 = pk2(r3a, r3b);
            NRR5 = pk2(-r5a, -r5b);
        }
    }
    if (KIND == 1) {
        // pair_matvec2 with both sums negated: -f_i += rr3 v_j - (rr5 v_j.d) d,
        // -f_j += rr3 v_i - (rr5 v_i.d) d.
        const f2 DDJ = mul2(NRR5, fma2(VJX, DX, fma2(VJY, DY, mul2(VJZ, DZ))));
        const f2 DDI = mul2(NRR5, fma2(x.VX, DX, fma2(x.VY, DY, mul2(x.VZ, DZ))));
        FX = fma2(RR3, VJX, fma2(DDJ, DX, FX));
        FY = fma2(RR3, VJY, fma2(DDJ, DY, FY));
        FZ = fma2(RR3, VJZ, fma2(DDJ, DZ, FZ));
        GX = fma2(RR3, x.VX, fma2(DDI, DX, GX));
        GY = fma2(RR3, x.VY, fma2(DDI, DY, GY));
        GZ = fma2(RR3, x.VZ, fma2(DDI, DZ, GZ));
    } else {
        // pair_fixed2: a = rr3 q_j - rr5 m_j.d, b = rr3 q_i + rr5 m_i.d;
        // -f_i += d a + m_j rr3;  -f_j += m_i rr3 - d b, with nb = -b.
        const f2 A = fma2(NRR5, fma2(VJX, DX, fma2(VJY, DY, mul2(VJZ, DZ))), mul2(RR3, QJ));
        const f2 NB = fma2(NRR5, fma2(x.VX, DX, fma2(x.VY, DY, mul2(x.VZ, DZ))), mul2(RR3, x.NQ));
        FX = fma2(VJX, RR3, fma2(DX, A, FX));
        FY = fma2(VJY, RR3, fma2(DY, A, FY));
        FZ = fma2(VJZ, RR3, fma2(DZ, A, FZ));
        GX = fma2(x.VX, RR3, fma2(DX, NB, GX));
        GY = fma2(x.VY, RR3, fma2(DY, NB, GY));
        GZ = fma2(x.VZ, RR3, fma2(DZ, NB, GZ));
    }
}

template <int KIND, bool FOLD, bool DAMP>
__device__ __forceinline__ void field_walk_x4(const PairParams& P, const double* __restrict__ pos,
                                              const FPackedTile& T, int lane, int jbase, const XSlot& xa,
                                              const XSlot& xb, bool two, unsigned fm, float damp_r2, float* fa,
                                              float* fb, float* g) {
    const int nxt = (lane + 1) & 31;
    f2 Lx = 0, Ly = 0, Lz = 0, Ix = 0, Iy = 0, Iz = 0, NTx = 0, NTy = 0, NTz = 0;
    if (FOLD) {
        Lx = bc2(-(float)P.box[0]);
        Ly = bc2(-(float)P.box[1]);
        Lz = bc2(-(float)P.box[2]);
        Ix = bc2((float)P.inv_box[0]);
        Iy = bc2((float)P.inv_box[1]);
        Iz = bc2((float)P.inv_box[2]);
        NTx = bc2(-(float)(P.half_box_tol[0] * P.half_box_tol[0]));
        NTy = bc2(-(float)(P.half_box_tol[1] * P.half_box_tol[1]));
        NTz = bc2(-(float)(P.half_box_tol[2] * P.half_box_tol[2]));
    }
    f2 FXA = 0, FYA = 0, FZA = 0, FXB = 0, FYB = 0, FZB = 0;   // I side, packed over (m, m + 16)
    f2 GX = 0, GY = 0, GZ = 0;                                 // J side (packed atoms m, m + 16)
    // One step is already four independent pairs: no unrolling (the walk's
    // variants must stay small enough for the instruction cache).
#pragma unroll 1
    for (int s = 0; s < 16; s++) {
        const int m = (lane + s) & 15;
        const float4 a = T.p0[m], b = T.p1[m], c = T.v0[m], d = T.v1[m];
        const f2 PX = pk2(a.x, a.y), PY = pk2(a.z, a.w), PZ = pk2(b.x, b.y), QJ = pk2(b.z, b.w);
        const f2 VJX = pk2(c.x, c.y), VJY = pk2(c.z, c.w), VJZ = pk2(d.x, d.y);
        xslot_pairs<KIND, FOLD, DAMP>(P, pos, xa, jbase + m, PX, PY, PZ, QJ, VJX, VJY, VJZ, d.z, d.w, fm, Lx, Ly,
                                      Lz, Ix, Iy, Iz, NTx, NTy, NTz, damp_r2, FXA, FYA, FZA, GX, GY, GZ);
        if (two)
            xslot_pairs<KIND, FOLD, DAMP>(P, pos, xb, jbase + m, PX, PY, PZ, QJ, VJX, VJY, VJZ, d.z, d.w, fm, Lx, Ly,
                                          Lz, Ix, Iy, Iz, NTx, NTy, NTz, damp_r2, FXB, FYB, FZB, GX, GY, GZ);
        GX = __shfl_sync(kFull, GX, nxt);
        GY = __shfl_sync(kFull, GY, nxt);
        GZ = __shfl_sync(kFull, GZ, nxt);
    }
    // F and G hold the negated sums (xslot_pairs).
    float lo, hi;
    un2(FXA, lo, hi);
    fa[0] -= lo + hi;
    un2(FYA, lo, hi);
    fa[1] -= lo + hi;
    un2(FZA, lo, hi);
    fa[2] -= lo + hi;
    if (two) {
        un2(FXB, lo, hi);
        fb[0] -= lo + hi;
        un2(FYB, lo, hi);
        fb[1] -= lo + hi;
        un2(FZB, lo, hi);
        fb[2] -= lo + hi;
    }
    // Lane l now holds (atom l & 15, atom (l & 15) + 16); lane l ^ 16 the other copy.
    const f2 Js[3] = {GX, GY, GZ};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        un2(Js[k], lo, hi);
        const float olo = __shfl_xor_sync(kFull, lo, 16), ohi = __shfl_xor_sync(kFull, hi, 16);
        g[k] -= lane < 16 ? lo + olo : hi + ohi;
    }
}

// Partner pairs of a SLOW tile pair, each side once with its scale (M for
// the permanent field, I for the matvec): lane l adds, for its I atom, the
// partners in J, and for atom l of J (not on the diagonal tile), the partners
// in I.
template <class R, int KIND, bool FOLD>
__device__ __forceinline__ void field_partners(const PairParams& P, const double* __restrict__ pos,
                                               const typename Vec4T<R>::type* __restrict__ posq,
                                               const typename Vec4T<R>::type* __restrict__ jvec,
                                               const typename Vec4T<R>::type* __restrict__ sp,
                                               const typename Vec4T<R>::type* __restrict__ sv,
                                               const int* __restrict__ exc_off, const int* __restrict__ exc_j,
                                               const double* __restrict__ exc_m, const double* __restrict__ exc_s,
                                               const TileGeom& g, double4 cA, double4 cB, int lane, int i, int ibase,
                                               int jbase, int e0, int e1, R oix, R oiy, R oiz, R qi,
                                               typename Vec4T<R>::type vi, bool diag, R damp_r2, R& fx, R& fy, R& fz,
                                               R& gx, R& gy, R& gz,
                                               const typename Vec4T<R>::type* __restrict__ lab = nullptr) {
    typedef typename Vec4T<R>::type V4;
    // With lab (the fused start of a warm-started solve, KIND 0) the operand
    // is P = m + mu0 and a partner pair adds M * field(q, P) + (I - M) * T mu0
    // = M * field(q, m) + I * T mu0, with mu0 = P - m.
    const bool fused = KIND == 0 && lab != nullptr;
#pragma unroll 1
    for (int e = e0; e < e1; e++) {
        unsigned off = (unsigned)(exc_j[e] - jbase);
        if (off >= 32u) continue;
        R sc = (R)(KIND == 0 ? exc_m[e] : exc_s[e]);
        const R si = (R)exc_s[e];
        if (sc == R(0) && (!fused || si == R(0))) continue;
        const V4 pj = sp[off], vj = sv[off];
        R dx, dy, dz;
        pair_delta<R, FOLD>(P, pos, i, jbase + off, pj.x, pj.y, pj.z, oix, oiy, oiz, dx, dy, dz);
        R r2 = dx * dx + dy * dy + dz * dz;
        R tx = 0, ty = 0, tz = 0;
        if (KIND == 0) pair_fixed<R, true>(dx, dy, dz, r2, pj.w, vj.x, vj.y, vj.z, vi.w, vj.w, damp_r2, tx, ty, tz);
        else pair_matvec<R, true>(dx, dy, dz, r2, vj.x, vj.y, vj.z, vi.w, vj.w, damp_r2, tx, ty, tz);
        fx += sc * tx;
        fy += sc * ty;
        fz += sc * tz;
        if (fused && si != sc) {
            const V4 mj = lab[jbase + off];
            R ux = 0, uy = 0, uz = 0;
            pair_matvec<R, true>(dx, dy, dz, r2, vj.x - mj.x, vj.y - mj.y, vj.z - mj.z, vi.w, vj.w, damp_r2, ux, uy,
                                 uz);
            fx += (si - sc) * ux;
            fy += (si - sc) * uy;
            fz += (si - sc) * uz;
        }
    }
    if (diag) return;
    const int jl = jbase + lane;
    if (jl >= P.n) return;
    const V4 pl = sp[lane], vl = sv[lane];
#pragma unroll 1
    for (int e = exc_off[jl]; e < exc_off[jl + 1]; e++) {
        const int a = exc_j[e];
        if ((unsigned)(a - ibase) >= 32u) continue;
        R sc = (R)(KIND == 0 ? exc_m[e] : exc_s[e]);
        const R si = (R)exc_s[e];
        if (sc == R(0) && (!fused || si == R(0))) continue;
        const V4 pa = posq[a], va = jvec[a];
        R ox, oy, oz;
        shift_into<R>(g, cA, cB, pa.x, pa.y, pa.z, ox, oy, oz);
        R dx, dy, dz;  // p_a - p_jl
        pair_delta<R, FOLD>(P, pos, jl, a, ox, oy, oz, pl.x, pl.y, pl.z, dx, dy, dz);
        R r2 = dx * dx + dy * dy + dz * dz;
        R tx = 0, ty = 0, tz = 0;
        if (KIND == 0) pair_fixed<R, true>(dx, dy, dz, r2, pa.w, va.x, va.y, va.z, vl.w, va.w, damp_r2, tx, ty, tz);
        else pair_matvec<R, true>(dx, dy, dz, r2, va.x, va.y, va.z, vl.w, va.w, damp_r2, tx, ty, tz);
        gx += sc * tx;
        gy += sc * ty;
        gz += sc * tz;
        if (fused && si != sc) {
            const V4 ma = lab[a];
            R ux = 0, uy = 0, uz = 0;
            pair_matvec<R, true>(dx, dy, dz, r2, va.x - ma.x, va.y - ma.y, va.z - ma.z, vl.w, va.w, damp_r2, ux, uy,
                                 uz);
            gx += (si - sc) * ux;
            gy += (si - sc) * uy;
            gz += (si - sc) * uz;
        }
    }
}

// One I tile of a warp (lane = atom) and its state against the current J
// tile.  The tile's centre and extent stay in shared memory (s_ic, s_ie).
template <class R>
struct ISlot {
    typename Vec4T<R>::type pi, vi;
    int2 et;
    int Il, I, i, e0, e1;
    bool act;
    // Against the current J tile.
    bool valid, diag, slow, fold, near;
    unsigned partners, fmask;
    R ox, oy, oz;
};

template <class R>
__device__ __forceinline__ void load_slot(ISlot<R>& a, const PairParams& P, int p, int BT, int Il, int lane,
                                          const typename Vec4T<R>::type* __restrict__ posq,
                                          const typename Vec4T<R>::type* __restrict__ jvec,
                                          const int* __restrict__ exc_off, const int2* __restrict__ exc_tiles) {
    a.Il = Il;
    a.I = p * BT + Il;
    a.act = Il < BT && a.I < P.n_tiles;
    a.i = a.I * 32 + lane;
    a.pi = {};
    a.vi = {};
    a.et = make_int2(1 << 30, -1);
    a.e0 = a.e1 = 0;
    if (a.act) {
        a.pi = posq[a.i];
        a.vi = jvec[a.i];
        a.et = exc_tiles[a.I];
        if (a.i < P.n) {
            a.e0 = exc_off[a.i];
            a.e1 = exc_off[a.i + 1];
        }
    }
}

template <class R>
__device__ __forceinline__ void slot_against(ISlot<R>& a, const PairParams& P, bool same_band, int J, int Jl,
                                             double4 cA, double4 eA, double4 cB, double4 eB,
                                             const int* __restrict__ exc_j) {
    a.valid = a.act && J < P.n_tiles && (!same_band || Jl >= a.Il);
    if (!a.valid) return;
    const TileGeom g = tile_geom(P, cA, eA, cB, eB);
    shift_into<R>(g, cA, cB, a.pi.x, a.pi.y, a.pi.z, a.ox, a.oy, a.oz);
    a.fold = g.fold;
    a.fmask = g.fmask;
    a.near = g.near;
    a.diag = a.I == J;
    a.slow = a.diag || (J == P.n_tiles - 1 && (P.n & 31)) || (J >= a.et.x && J <= a.et.y);
    a.partners = a.slow ? partner_bits(exc_j, a.e0, a.e1, J * 32) : 0u;
}

// The same from the tile pair's geometry computed beforehand (FP32 form):
// centre displacement dc in FP32 and flags fmask | fold << 3 | near << 4.
template <class R>
__device__ __forceinline__ void slot_against_pre(ISlot<R>& a, const PairParams& P, bool same_band, int J, int Jl,
                                                 float dcx, float dcy, float dcz, unsigned fl,
                                                 const int* __restrict__ exc_j) {
    a.valid = a.act && J < P.n_tiles && (!same_band || Jl >= a.Il);
    if (!a.valid) return;
    a.ox = a.pi.x - (R)dcx;
    a.oy = a.pi.y - (R)dcy;
    a.oz = a.pi.z - (R)dcz;
    a.fmask = fl & 7u;
    a.fold = (fl >> 3) & 1u;
    a.near = (fl >> 4) & 1u;
    a.diag = a.I == J;
    a.slow = a.diag || (J == P.n_tiles - 1 && (P.n & 31)) || (J >= a.et.x && J <= a.et.y);
    a.partners = a.slow ? partner_bits(exc_j, a.e0, a.e1, J * 32) : 0u;
}

// FP32: 4 CTAs per SM at 128 registers; FP64: 3 CTAs per SM (168 registers),
// which halves the FP64 walks' register spills (measured 2-4 % faster).
template <class R, int KIND>
__global__ void __launch_bounds__(kSymThreads, sizeof(R) == 4 ? 4 : 3) k_field_sym(
    PairParams P, const typename Vec4T<R>::type* __restrict__ posq, const typename Vec4T<R>::type* __restrict__ jvec,
    const double4* __restrict__ tctr, const double4* __restrict__ text, const double* __restrict__ pos,
    const int* __restrict__ exc_off, const int* __restrict__ exc_j, const double* __restrict__ exc_m,
    const double* __restrict__ exc_s, const int2* __restrict__ exc_tiles, int n_pad, double* __restrict__ partial,
    FixAcc fix, const typename Vec4T<R>::type* __restrict__ lab) {
    typedef typename Vec4T<R>::type V4;
    extern __shared__ __align__(16) unsigned char smem[];
    const int BT = P.band_tiles, NA = BT * 32;
    double* s_iacc = reinterpret_cast<double*>(smem);              // 6 * kSymThreads: I-side sums, two slots
    double4* s_ctr = reinterpret_cast<double4*>(s_iacc + 6 * kSymThreads);  // BT
    double4* s_ext = s_ctr + BT;                                   // BT
    double4* s_ic = s_ext + BT;                                    // 2 * kSymWarps: the warps' I tiles
    double4* s_ie = s_ic + 2 * kSymWarps;
    V4* s_pos = reinterpret_cast<V4*>(s_ie + 2 * kSymWarps);       // NA
    V4* s_vec = s_pos + NA;                                        // NA
    R* s_acc = reinterpret_cast<R*>(s_vec + NA);                   // kSymWarps * 3 * NA: J-side sums per warp
    FPackedTile* s_fpt = reinterpret_cast<FPackedTile*>(s_acc + kSymWarps * 3 * NA);  // kSymWarps (FP32 only)

    int p, q;
    band_pair(blockIdx.x, p, q);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int qa0 = q * NA;
    for (int k = threadIdx.x; k < NA; k += kSymThreads) {
        s_pos[k] = posq[qa0 + k];
        s_vec[k] = jvec[qa0 + k];
    }
    for (int k = threadIdx.x; k < kSymWarps * 3 * NA; k += kSymThreads) s_acc[k] = R(0);
    for (int k = threadIdx.x; k < BT; k += kSymThreads) {
        s_ctr[k] = tctr[q * BT + k];
        s_ext[k] = text[q * BT + k];
    }
    double* my = s_iacc + 6 * threadIdx.x;
    R* wacc = s_acc + warp * 3 * NA;
    __syncthreads();

    // Each warp sums its J-side contributions in its own area, so the warps
    // never wait for one another until the final combination.
    const R damp_r2 = (R)P.damp_r2;
    const int stride = BT >= kSymWarps ? BT / kSymWarps : 1;
    // A warp's I tiles are warp, warp + 4, warp + 8, ...; a round takes two of them.
    const int rounds = (BT + 2 * kSymWarps - 1) / (2 * kSymWarps);
    for (int r = 0; r < rounds; r++) {
        ISlot<R> a, b;
        load_slot<R>(a, P, p, BT, warp + 2 * kSymWarps * r, lane, posq, jvec, exc_off, exc_tiles);
        load_slot<R>(b, P, p, BT, warp + 2 * kSymWarps * r + kSymWarps, lane, posq, jvec, exc_off, exc_tiles);
        __syncwarp();
        if (lane < 2) {
            const ISlot<R>& s1 = lane == 0 ? a : b;
            s_ic[2 * warp + lane] = s1.act ? tctr[s1.I] : make_double4(0, 0, 0, 0);
            s_ie[2 * warp + lane] = s1.act ? text[s1.I] : make_double4(0, 0, 0, 0);
        }
        __syncwarp();
        // FP32 form: the round's 2 x BT tile-pair geometries (FP64 arithmetic),
        // one per lane, instead of every lane repeating each of them.
        float gdx = 0.f, gdy = 0.f, gdz = 0.f;
        unsigned gfl = 0u;
        if constexpr (sizeof(R) == 4) {
            if (lane < 2 * BT) {
                const int k = lane / BT, Jl = lane - k * BT;
                const TileGeom g = tile_geom(P, s_ic[2 * warp + k], s_ie[2 * warp + k], s_ctr[Jl], s_ext[Jl]);
                gdx = (float)g.dcx;
                gdy = (float)g.dcy;
                gdz = (float)g.dcz;
                gfl = g.fmask | (g.fold ? 8u : 0u) | (g.near ? 16u : 0u);
            }
        }
        for (int c = 0; c < 6; c++) my[c] = 0.0;
        for (int t = 0; t < BT; t++) {
            const int Jl = (t + warp * stride) % BT;
            const int J = q * BT + Jl;
            const double4 cB = s_ctr[Jl], eB = s_ext[Jl];
            if constexpr (sizeof(R) == 4) {
                const int la = Jl, lb = BT + Jl;
                const float ax = __shfl_sync(kFull, gdx, la), ay = __shfl_sync(kFull, gdy, la),
                            az = __shfl_sync(kFull, gdz, la);
                const float bx = __shfl_sync(kFull, gdx, lb), by = __shfl_sync(kFull, gdy, lb),
                            bz = __shfl_sync(kFull, gdz, lb);
                const unsigned af = __shfl_sync(kFull, gfl, la), bf = __shfl_sync(kFull, gfl, lb);
                slot_against_pre<R>(a, P, p == q, J, Jl, ax, ay, az, af, exc_j);
                slot_against_pre<R>(b, P, p == q, J, Jl, bx, by, bz, bf, exc_j);
            } else {
                slot_against<R>(a, P, p == q, J, Jl, s_ic[2 * warp], s_ie[2 * warp], cB, eB, exc_j);
                slot_against<R>(b, P, p == q, J, Jl, s_ic[2 * warp + 1], s_ie[2 * warp + 1], cB, eB, exc_j);
            }
            if (!(a.valid || b.valid)) continue;
            const int jbase = J * 32;
            const V4* sp = s_pos + Jl * 32;
            const V4* sv = s_vec + Jl * 32;
            R fa[3] = {0, 0, 0}, fb[3] = {0, 0, 0}, g[3] = {0, 0, 0};
            bool packed = false;
            if constexpr (sizeof(R) == 4) {
                // Non-SLOW tile pairs: the packed walk over J-atom pairs, one or both slots.
                const bool two = a.valid && b.valid;
                if (two ? !(a.slow || b.slow) : !(a.valid ? a.slow : b.slow)) {
                    packed = true;
                    __syncwarp();
                    stage_fpacked(s_fpt[warp], lane, sp[lane], sv[lane]);
                    __syncwarp();
                    const ISlot<R>& s1 = a.valid ? a : b;
                    const ISlot<R>& s2 = two ? b : s1;
                    float* f1 = a.valid ? fa : fb;
                    const XSlot x1 = xslot(s1.i, s1.ox, s1.oy, s1.oz, s1.pi.w, s1.vi);
                    const XSlot x2 = xslot(s2.i, s2.ox, s2.oy, s2.oz, s2.pi.w, s2.vi);
                    const unsigned fm = s1.fmask | s2.fmask;
                    const bool fold = s1.fold || s2.fold, near = s1.near || s2.near;
// One inlined copy per slot count (the count is a constant inside each).
#define TDP_FWALKX4(F, D)                                                                                        \
    do {                                                                                                         \
        if (two)                                                                                                 \
            field_walk_x4<KIND, F, D>(P, pos, s_fpt[warp], lane, jbase, x1, x2, true, fm, damp_r2, f1, fb, g);  \
        else                                                                                                     \
            field_walk_x4<KIND, F, D>(P, pos, s_fpt[warp], lane, jbase, x1, x2, false, fm, damp_r2, f1, fb, g); \
    } while (0)
                    if (fold) {
                        if (near) TDP_FWALKX4(true, true);
                        else TDP_FWALKX4(true, false);
                    } else if (near) {
                        TDP_FWALKX4(false, true);
                    } else {
                        TDP_FWALKX4(false, false);
                    }
#undef TDP_FWALKX4
                }
            }
            if (packed) {
            } else if (a.valid && b.valid) {
                const bool slow = a.slow || b.slow, fold = a.fold || b.fold;
                const bool near = a.near || b.near;
#define TDP_FWALK2(F, S, D)                                                                                        \
    field_walk2<R, KIND, F, S, D>(P, pos, sp, sv, lane, jbase, a.i, a.ox, a.oy, a.oz, a.pi.w, a.vi, a.diag,     \
                                  a.partners, b.i, b.ox, b.oy, b.oz, b.pi.w, b.vi, b.diag, b.partners, damp_r2, fa, \
                                  fb, g)
                if (slow) {
                    if (fold) TDP_FWALK2(true, true, true);
                    else TDP_FWALK2(false, true, true);
                } else if (fold) {
                    if (near) TDP_FWALK2(true, false, true);
                    else TDP_FWALK2(true, false, false);
                } else if (near) {
                    TDP_FWALK2(false, false, true);
                } else {
                    TDP_FWALK2(false, false, false);
                }
#undef TDP_FWALK2
            } else {
                const ISlot<R>& s1 = a.valid ? a : b;
                R* f1 = a.valid ? fa : fb;
#define TDP_FWALK(F, S, D)                                                                                        \
    field_walk<R, KIND, F, S, D>(P, pos, sp, sv, lane, s1.i, jbase, s1.ox, s1.oy, s1.oz, s1.pi.w, s1.vi, s1.diag, \
                                 s1.partners, damp_r2, f1[0], f1[1], f1[2], g[0], g[1], g[2])
                if (s1.slow) {
                    if (s1.fold) TDP_FWALK(true, true, true);
                    else TDP_FWALK(false, true, true);
                } else if (s1.fold) {
                    if (s1.near) TDP_FWALK(true, false, true);
                    else TDP_FWALK(true, false, false);
                } else if (s1.near) {
                    TDP_FWALK(false, false, true);
                } else {
                    TDP_FWALK(false, false, false);
                }
#undef TDP_FWALK
            }
            // Partner pairs of each SLOW slot, each side once.
            for (int k = 0; k < 2; k++) {
                const ISlot<R>& s1 = k == 0 ? a : b;
                if (!s1.valid || !s1.slow) continue;
                R* f1 = k == 0 ? fa : fb;
                const double4 cA = s_ic[2 * warp + k];
                const TileGeom g1 = tile_geom(P, cA, s_ie[2 * warp + k], cB, eB);
                if (s1.fold)
                    field_partners<R, KIND, true>(P, pos, posq, jvec, sp, sv, exc_off, exc_j, exc_m, exc_s, g1, cA,
                                                  cB, lane, s1.i, s1.I * 32, jbase, s1.e0, s1.e1, s1.ox, s1.oy, s1.oz,
                                                  s1.pi.w, s1.vi, s1.diag, damp_r2, f1[0], f1[1], f1[2], g[0], g[1],
                                                  g[2], lab);
                else
                    field_partners<R, KIND, false>(P, pos, posq, jvec, sp, sv, exc_off, exc_j, exc_m, exc_s, g1, cA,
                                                   cB, lane, s1.i, s1.I * 32, jbase, s1.e0, s1.e1, s1.ox, s1.oy,
                                                   s1.oz, s1.pi.w, s1.vi, s1.diag, damp_r2, f1[0], f1[1], f1[2], g[0],
                                                   g[1], g[2], lab);
            }
            R* acc = wacc + 3 * (Jl * 32 + lane);
            for (int c = 0; c < 3; c++) {
                acc[c] += g[c];
                my[c] += (double)fa[c];
                my[3 + c] += (double)fb[c];
            }
        }
        // I-side sums: slot q of band p; on the diagonal band, slot p, where
        // the J-side sums of the same atoms are added below.
        // (Mixed form: added into the fixed-point accumulator instead.)
        for (int k = 0; k < 2; k++) {
            const ISlot<R>& s1 = k == 0 ? a : b;
            if (!s1.act) continue;
            if (sizeof(R) == 4) {
                for (int c = 0; c < 3; c++) fix_add(fix, (size_t)c * n_pad + s1.i, my[3 * k + c]);
            } else {
                const size_t base = (size_t)q * 3 * n_pad;
                for (int c = 0; c < 3; c++) partial[base + (size_t)c * n_pad + s1.i] = my[3 * k + c];
            }
        }
    }
    __syncthreads();
    const size_t base = (size_t)p * 3 * n_pad;
    for (int k = threadIdx.x; k < NA; k += kSymThreads) {
        const int a = qa0 + k;
        const bool own = p == q && (a >> 5) < P.n_tiles;
        for (int c = 0; c < 3; c++) {
            double v = 0.0;
            for (int w = 0; w < kSymWarps; w++) v += (double)s_acc[w * 3 * NA + 3 * k + c];
            if (sizeof(R) == 4) {
                fix_add(fix, (size_t)c * n_pad + a, v);
            } else {
                if (own) v += partial[base + (size_t)c * n_pad + a];
                partial[base + (size_t)c * n_pad + a] = v;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Energy / force / torque kernel (index order: within a tile pair I < J every
// lane's atom has the lower index, the reference's orientation I = lower).
// ---------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ EAtom<R> eatom(typename Vec4T<R>::type pq, typename Vec4T<R>::type d,
                                          typename Vec4T<R>::type u) {
    EAtom<R> a;
    a.q = pq.w;
    a.mx = d.x;
    a.my = d.y;
    a.mz = d.z;
    a.t = d.w;
    a.ux = u.x;
    a.uy = u.y;
    a.uz = u.z;
    return a;
}

// formQIRotationMatrix's test on the raw positions, pI.y != pK.y || pI.z !=
// pK.z (RTDF.cpp:584): displacements above 1e-5 nm decide it; below that the
// raw FP64 coordinates are compared.
template <class R>
__device__ __forceinline__ bool yz_differ(R dy, R dz, const double2* __restrict__ yz, int i, int j, int nmax) {
    bool d = fabs(dy) > R(1e-5) || fabs(dz) > R(1e-5);
    if (!d) {
        const double2 a = yz[min(i, nmax)], b = yz[min(j, nmax)];
        d = (a.x != b.x) || (a.y != b.y);
    }
    return d;
}

// LAB (non-SLOW tile pairs beyond the damping range only): pair_energy_lab.
template <class R, bool FOLD, bool SLOW, bool LAB = false>
__device__ __forceinline__ void energy_walk(const PairParams& P, const double* __restrict__ pos,
                                            const double2* __restrict__ yz,
                                            const typename Vec4T<R>::type* __restrict__ sp,
                                            const typename Vec4T<R>::type* __restrict__ sd,
                                            const typename Vec4T<R>::type* __restrict__ su, int lane, int i,
                                            int jbase, R oix, R oiy, R oiz, const EAtom<R>& me, bool diag,
                                            unsigned partners, R damp_r2, R rv4p, R rv4f, R f[6], R g[6], R& en) {
    const int nxt = (lane + 1) & 31;
    const int nmax = P.n_tiles * 32 - 1;
    // LAB: the walk sums V_ij (I side) and V_ji (J side, rotating with the
    // J atoms) and turns them into torques once at the end (pair_energy_lab).
    R vi[3] = {0, 0, 0}, vj[3] = {0, 0, 0};
#pragma unroll 1
    for (int s = 0; s < 32; s++) {
        const int jj = (lane + s) & 31;
        const int j = jbase + jj;
        const EAtom<R> other = eatom<R>(sp[jj], sd[jj], su[jj]);
        R dx, dy, dz;
        pair_delta<R, FOLD>(P, pos, i, j, sp[jj].x, sp[jj].y, sp[jj].z, oix, oiy, oiz, dx, dy, dz);
        R r2 = dx * dx + dy * dy + dz * dz;
        if (SLOW && skip_pair(s, lane, i, j, P.n, partners, jj, diag)) r2 = (R)INFINITY;
        const bool yzd = yz_differ<R>(dy, dz, yz, i, j, nmax);
        if (LAB) {
            pair_energy_lab<R, true>(dx, dy, dz, r2, yzd, me, other, P.mutual ? R(1) : R(-1), f[0], f[1], f[2], vi[0],
                                     vi[1], vi[2], g[0], g[1], g[2], vj[0], vj[1], vj[2], en);
        } else if (!SLOW || !diag) {
            pair_energy_sides<R, 3>(dx, dy, dz, r2, yzd, me, other, R(1), R(1), damp_r2, rv4p, rv4f, P.mutual != 0,
                                    f[0], f[1], f[2], f[3], f[4], f[5], g[0], g[1], g[2], g[3], g[4], g[5], en);
        } else {
            // Diagonal tile: the lane's atom is the lower index iff lane + s < 32.
            const bool lo = lane + s < 32;
            const EAtom<R> A = lo ? me : other;
            const EAtom<R> B = lo ? other : me;
            const R sg = lo ? R(1) : R(-1);
            R a[6] = {0, 0, 0, 0, 0, 0}, b[6] = {0, 0, 0, 0, 0, 0};
            pair_energy_sides<R, 3>(sg * dx, sg * dy, sg * dz, r2, yzd, A, B, R(1), R(1), damp_r2, rv4p, rv4f,
                                    P.mutual != 0, a[0], a[1], a[2], a[3], a[4], a[5], b[0], b[1], b[2], b[3], b[4],
                                    b[5], en);
#pragma unroll
            for (int c = 0; c < 6; c++) {
                f[c] += lo ? a[c] : b[c];
                g[c] += lo ? b[c] : a[c];
            }
        }
        if (LAB) {
            // g[3..5] are untouched by this walk (a full rotation is the identity).
#pragma unroll
            for (int c = 0; c < 3; c++) {
                g[c] = __shfl_sync(kFull, g[c], nxt);
                vj[c] = __shfl_sync(kFull, vj[c], nxt);
            }
        } else {
#pragma unroll
            for (int c = 0; c < 6; c++) g[c] = __shfl_sync(kFull, g[c], nxt);
        }
    }
    if (LAB) {
        // tau = -perm(m x sum V) and the dipole energy 0.5 m.sum V: the lane's
        // I atom, and J atom jbase + lane.
        const typename Vec4T<R>::type mj = sd[lane];
        en += R(0.5) * (me.mx * vi[0] + me.my * vi[1] + me.mz * vi[2] + mj.x * vj[0] + mj.y * vj[1] + mj.z * vj[2]);
        f[3] -= me.mz * vi[0] - me.mx * vi[2];
        f[4] -= me.mx * vi[1] - me.my * vi[0];
        f[5] -= me.my * vi[2] - me.mz * vi[1];
        g[3] -= mj.z * vj[0] - mj.x * vj[2];
        g[4] -= mj.x * vj[1] - mj.y * vj[0];
        g[5] -= mj.y * vj[2] - mj.z * vj[1];
    }
}

// ---------------------------------------------------------------------------
// Packed FP32 energy walk (mixed form, non-SLOW tile pairs): the lane's I
// atom against J atoms m and m + 16 of the tile at once (m = (lane + s) & 15,
// s = 0..15), the pair routine of pair_energy_sides<R, 3> in f32x2 halves.
// The J-side sums ride packed (lo: atom m, hi: atom m + 16) and rotate one
// lane per step; after 16 steps lanes l and l ^ 16 hold the two copies of the
// sums of atoms l & 15 and (l & 15) + 16, added by one xor-16 shuffle.
// ---------------------------------------------------------------------------
struct EPackedTile {
    float4 p0[16], p1[16];   // (x, x', y, y'), (z, z', q, q')   (' = atom m + 16)
    float4 d0[16], d1[16];   // (mx, mx', my, my'), (mz, mz', t, t')
    float4 u0[16], u1[16];   // (ux, ux', uy, uy'), (uz, uz', 1/t, 1/t')
};

__device__ __forceinline__ void stage_epacked(EPackedTile& T, int lane, float4 p, float4 d, float4 u) {
    const int m = lane & 15, h = lane >> 4;
    float* p0 = reinterpret_cast<float*>(&T.p0[m]);
    float* p1 = reinterpret_cast<float*>(&T.p1[m]);
    float* d0 = reinterpret_cast<float*>(&T.d0[m]);
    float* d1 = reinterpret_cast<float*>(&T.d1[m]);
    float* u0 = reinterpret_cast<float*>(&T.u0[m]);
    float* u1 = reinterpret_cast<float*>(&T.u1[m]);
    p0[h] = p.x;
    p0[2 + h] = p.y;
    p1[h] = p.z;
    p1[2 + h] = p.w;
    d0[h] = d.x;
    d0[2 + h] = d.y;
    d1[h] = d.z;
    d1[2 + h] = d.w;
    u0[h] = u.x;
    u0[2 + h] = u.y;
    u1[h] = u.z;
    u1[2 + h] = 1.0f / d.w;
}


template <bool FOLD>
__device__ __forceinline__ void energy_walk_x2(const PairParams& P, const double* __restrict__ pos,
                                               const double2* __restrict__ yz, const EPackedTile& T, int lane,
                                               int i, int jbase, float oix, float oiy, float oiz, float4 pi,
                                               float4 di, float4 ui, unsigned fm, float damp_r2, float rv4p,
                                               float rv4f, bool mutual, float f[6], float gg[6], float& en) {
    const int nxt = (lane + 1) & 31;
    const int nmax = P.n_tiles * 32 - 1;
    const f2 OX = bc2(oix), OY = bc2(oiy), OZ = bc2(oiz);
    const f2 QI0 = bc2(pi.w), MIX = bc2(di.x), MIY = bc2(di.y), MIZ = bc2(di.z);
    const f2 UIX = bc2(ui.x), UIY = bc2(ui.y), UIZ = bc2(ui.z);
    const float ti = di.w, iti = 1.0f / di.w;
    const f2 ITI = bc2(iti), ONE = bc2(1.0f), HALF = bc2(0.5f);
    const f2 RV4P = bc2(rv4p), RV4F = bc2(rv4f);
    f2 Lx = 0, Ly = 0, Lz = 0, Ix = 0, Iy = 0, Iz = 0, NTx = 0, NTy = 0, NTz = 0;
    if (FOLD) {
        Lx = bc2(-(float)P.box[0]);
        Ly = bc2(-(float)P.box[1]);
        Lz = bc2(-(float)P.box[2]);
        Ix = bc2((float)P.inv_box[0]);
        Iy = bc2((float)P.inv_box[1]);
        Iz = bc2((float)P.inv_box[2]);
        NTx = bc2(-(float)(P.half_box_tol[0] * P.half_box_tol[0]));
        NTy = bc2(-(float)(P.half_box_tol[1] * P.half_box_tol[1]));
        NTz = bc2(-(float)(P.half_box_tol[2] * P.half_box_tol[2]));
    }
    // Torques from summed V (pair_energy_lab, VSUM): TX.. sum V_ij, UX.. V_ji.
    f2 FX = 0, FY = 0, FZ = 0, TX = 0, TY = 0, TZ = 0, EN = 0;        // I side
    f2 GX = 0, GY = 0, GZ = 0, UX = 0, UY = 0, UZ = 0;                // J side (packed atoms m, m + 16)
#pragma unroll 1
    for (int s = 0; s < 16; s++) {
        const int m = (lane + s) & 15;
        const float4 a = T.p0[m], b = T.p1[m], c = T.d0[m], d = T.d1[m], e = T.u0[m], h = T.u1[m];
        f2 DX = sub2(pk2(a.x, a.y), OX), DY = sub2(pk2(a.z, a.w), OY), DZ = sub2(pk2(b.x, b.y), OZ);
        const int ja = jbase + m, jb = ja + 16;
        if (FOLD) {
            // As in xslot_pairs: one sign-bit AND of the d^2 - t^2 words flags
            // the pairs within the margin of half a box.
            f2 neg = ~0ull;
            if (fm & 1u) {
                DX = fold2(DX, Lx, Ix);
                neg &= fma2(DX, DX, NTx);
            }
            if (fm & 2u) {
                DY = fold2(DY, Ly, Iy);
                neg &= fma2(DY, DY, NTy);
            }
            if (fm & 4u) {
                DZ = fold2(DZ, Lz, Iz);
                neg &= fma2(DZ, DZ, NTz);
            }
            const f2 flag = ~neg & 0x8000000080000000ull;
            if (flag) {
                const bool amb_a = (flag >> 31) & 1ull, amb_b = (flag >> 63) != 0ull;
                float ax, bx, ay, by, az, bz;
                un2(DX, ax, bx);
                un2(DY, ay, by);
                un2(DZ, az, bz);
                if (amb_a) {
                    d3 q = exact_delta(P, pos, i, ja);
                    ax = (float)q.x;
                    ay = (float)q.y;
                    az = (float)q.z;
                }
                if (amb_b) {
                    d3 q = exact_delta(P, pos, i, jb);
                    bx = (float)q.x;
                    by = (float)q.y;
                    bz = (float)q.z;
                }
                DX = pk2(ax, bx);
                DY = pk2(ay, by);
                DZ = pk2(az, bz);
            }
        }
        const f2 R2 = dot2(DX, DY, DZ, DX, DY, DZ);
        float r2a, r2b, dya, dyb, dza, dzb;
        un2(R2, r2a, r2b);
        un2(DY, dya, dyb);
        un2(DZ, dza, dzb);
        const bool yza = yz_differ<float>(dya, dza, yz, i, ja, nmax);
        const bool yzb = yz_differ<float>(dyb, dzb, yz, i, jb, nmax);
        const f2 RINV = pk2(rsqrtf(r2a), rsqrtf(r2b));
        // QI frame: Z along d; X from Z + x^ or y^ (the reference's yz test), Gram-Schmidt; Y = Z x X.
        const f2 ZX = mul2(DX, RINV), ZY = mul2(DY, RINV), ZZ = mul2(DZ, RINV);
        f2 XX = add2(ZX, pk2(yza ? 1.0f : 0.0f, yzb ? 1.0f : 0.0f));
        f2 XY = add2(ZY, pk2(yza ? 0.0f : 1.0f, yzb ? 0.0f : 1.0f));
        f2 XZ = ZZ;
        const f2 NDT = neg2(dot2(ZX, ZY, ZZ, XX, XY, XZ));
        XX = fma2(ZX, NDT, XX);
        XY = fma2(ZY, NDT, XY);
        XZ = fma2(ZZ, NDT, XZ);
        float xna, xnb;
        un2(dot2(XX, XY, XZ, XX, XY, XZ), xna, xnb);
        const f2 SN = pk2(xna > 0.0f ? rsqrtf(xna) : 1.0f, xnb > 0.0f ? rsqrtf(xnb) : 1.0f);
        XX = mul2(XX, SN);
        XY = mul2(XY, SN);
        XZ = mul2(XZ, SN);
        const f2 YX = fma2(ZY, XZ, neg2(mul2(ZZ, XY)));
        const f2 YY = fma2(ZZ, XX, neg2(mul2(ZX, XZ)));
        const f2 YZ = fma2(ZX, XY, neg2(mul2(ZY, XX)));
        // Rotated multipoles.
        const f2 UJX = pk2(e.x, e.y), UJY = pk2(e.z, e.w), UJZ = pk2(h.x, h.y);
        const f2 MJX = pk2(c.x, c.y), MJY = pk2(c.z, c.w), MJZ = pk2(d.x, d.y);
        const f2 uI0 = dot2(XX, XY, XZ, UIX, UIY, UIZ), uI1 = dot2(YX, YY, YZ, UIX, UIY, UIZ),
                 uI2 = dot2(ZX, ZY, ZZ, UIX, UIY, UIZ);
        const f2 uJ0 = dot2(XX, XY, XZ, UJX, UJY, UJZ), uJ1 = dot2(YX, YY, YZ, UJX, UJY, UJZ),
                 uJ2 = dot2(ZX, ZY, ZZ, UJX, UJY, UJZ);
        const f2 QJ0 = pk2(b.z, b.w);
        const f2 QI1 = dot2(XX, XY, XZ, MIX, MIY, MIZ), QI2 = dot2(YX, YY, YZ, MIX, MIY, MIZ),
                 QI3 = dot2(ZX, ZY, ZZ, MIX, MIY, MIZ);
        const f2 QJ1 = dot2(XX, XY, XZ, MJX, MJY, MJZ), QJ2 = dot2(YX, YY, YZ, MJX, MJY, MJZ),
                 QJ3 = dot2(ZX, ZY, ZZ, MJX, MJY, MJZ);
        const f2 rv1 = RINV, rv2 = mul2(RINV, RINV), rv3 = mul2(rv2, RINV);
        const f2 rv4 = fma2(RV4P, mul2(rv3, RINV), RV4F);
        // Thole factors (1 beyond damp_r2 or where t_i t_j <= 1e-5, as the reference).
        f2 tc = ONE, td0 = ONE, td1 = ONE, dtc = ONE, dtd0 = ONE, dtd1 = ONE;
        if (r2a < damp_r2 || r2b < damp_r2) {
            const f2 R = mul2(R2, RINV);
            const f2 U = mul2(mul2(R, ITI), pk2(h.z, h.w));
            const f2 AM = pk2(fminf(ti, d.z), fminf(ti, d.w));
            const f2 AU3 = mul2(AM, mul2(U, mul2(U, U)));
            float xa, xb;
            un2(AU3, xa, xb);
            const bool da = r2a < damp_r2 && fabsf(ti * d.z) > 1.0e-5f;
            const bool db = r2b < damp_r2 && fabsf(ti * d.w) > 1.0e-5f;
            const f2 EX = pk2(da ? __expf(-xa) : 0.0f, db ? __expf(-xb) : 0.0f);
            const f2 AUs = pk2(da ? xa : 0.0f, db ? xb : 0.0f);   // no inf/NaN into the products
            const f2 NEX = neg2(EX);
            tc = add2(ONE, NEX);
            td1 = tc;
            td0 = fma2(NEX, fma2(bc2(1.5f), AUs, ONE), ONE);
            dtc = td0;
            dtd0 = fma2(NEX, fma2(mul2(bc2(1.5f), AUs), AUs, add2(ONE, AUs)), ONE);
            dtd1 = fma2(NEX, add2(ONE, AUs), ONE);
        }
        // Interaction terms (mS = iS = 1).
        f2 eP = rv1, dP = mul2(bc2(-0.5f), rv2);
        f2 Vij0 = mul2(eP, QJ0), Vji0 = mul2(eP, QI0), VijR0 = mul2(dP, QJ0), VjiR0 = mul2(dP, QI0);
        eP = rv2;
        f2 eU = mul2(rv2, tc);
        dP = neg2(rv3);
        f2 dU = mul2(mul2(bc2(-2.0f), rv3), dtc);
        Vij0 = sub2(Vij0, fma2(eP, QJ1, mul2(eU, uJ0)));
        const f2 Vji1n = mul2(eP, QI0);   // -Vji1 so far (subtracted below: exact)
        VijR0 = sub2(VijR0, fma2(dP, QJ1, mul2(dU, uJ0)));
        f2 VjiR1 = mul2(rv3, QI0);        // -(dP QI0), dP = -rv3: exact
        f2 Vjid0 = neg2(mul2(eU, QI0));
        f2 Vij1 = mul2(eP, QJ0);
        Vji0 = add2(Vji0, fma2(eP, QI1, mul2(eU, uI0)));
        f2 VijR1 = mul2(dP, QJ0);
        VjiR0 = add2(VjiR0, fma2(dP, QI1, mul2(dU, uI0)));
        f2 Vijd0 = mul2(eU, QJ0);
        eP = mul2(bc2(-2.0f), rv3);
        eU = mul2(eP, td0);
        dP = mul2(bc2(3.0f), rv4);
        dU = mul2(mul2(bc2(6.0f), rv4), dtd0);
        Vij1 = add2(Vij1, fma2(eP, QJ1, mul2(eU, uJ0)));
        f2 Vji1 = sub2(fma2(eP, QI1, mul2(eU, uI0)), Vji1n);
        VijR1 = add2(VijR1, fma2(dP, QJ1, mul2(dU, uJ0)));
        VjiR1 = add2(VjiR1, fma2(dP, QI1, mul2(dU, uI0)));
        Vijd0 = fma2(eU, QJ1, Vijd0);
        Vjid0 = fma2(eU, QI1, Vjid0);
        eP = rv3;
        eU = mul2(rv3, td1);
        dP = mul2(bc2(-1.5f), rv4);
        dU = mul2(mul2(bc2(-3.0f), rv4), dtd1);
        const f2 Vij2 = fma2(eP, QJ2, mul2(eU, uJ1)), Vji2 = fma2(eP, QI2, mul2(eU, uI1));
        const f2 VijR2 = fma2(dP, QJ2, mul2(dU, uJ1)), VjiR2 = fma2(dP, QI2, mul2(dU, uI1));
        const f2 Vijd1 = mul2(eU, QJ2), Vjid1 = mul2(eU, QI2);
        const f2 Vij3 = fma2(eP, QJ3, mul2(eU, uJ2)), Vji3 = fma2(eP, QI3, mul2(eU, uI2));
        const f2 VijR3 = fma2(dP, QJ3, mul2(dU, uJ2)), VjiR3 = fma2(dP, QI3, mul2(dU, uI2));
        const f2 Vijd2 = mul2(eU, QJ3), Vjid2 = mul2(eU, QI3);

        f2 fIZ = fma2(QI0, VijR0, fma2(QI1, VijR1, fma2(QI2, VijR2, mul2(QI3, VijR3))));
        f2 fJZ = fma2(QJ0, VjiR0, fma2(QJ1, VjiR1, fma2(QJ2, VjiR2, mul2(QJ3, VjiR3))));
        const f2 EIX = sub2(mul2(QI3, Vij1), mul2(QI1, Vij3));
        const f2 EIY = sub2(mul2(QI1, Vij2), mul2(QI2, Vij1));
        const f2 EJX = sub2(mul2(QJ3, Vji1), mul2(QJ1, Vji3));
        const f2 EJY = sub2(mul2(QJ1, Vji2), mul2(QJ2, Vji1));
        f2 iEIX = sub2(mul2(uI2, Vijd0), mul2(uI0, Vijd2));
        f2 iEJX = sub2(mul2(uJ2, Vjid0), mul2(uJ0, Vjid2));
        f2 iEIY = sub2(mul2(uI0, Vijd1), mul2(uI1, Vijd0));
        f2 iEJY = sub2(mul2(uJ0, Vjid1), mul2(uJ1, Vjid0));
        if (mutual) {
            f2 eC = mul2(mul2(bc2(-4.0f), rv3), td0);
            f2 dC = mul2(mul2(bc2(6.0f), rv4), dtd0);
            iEIX = fma2(mul2(eC, uI2), uJ0, iEIX);
            iEJX = fma2(mul2(eC, uJ2), uI0, iEJX);
            iEIY = sub2(iEIY, mul2(mul2(eC, uI1), uJ0));
            iEJY = sub2(iEJY, mul2(mul2(eC, uJ1), uI0));
            fIZ = fma2(mul2(dC, uI0), uJ0, fIZ);
            fJZ = fma2(mul2(dC, uJ0), uI0, fJZ);
            eC = mul2(mul2(bc2(2.0f), rv3), td1);
            dC = mul2(mul2(bc2(-3.0f), rv4), dtd1);
            iEIX = sub2(iEIX, mul2(mul2(eC, uI0), uJ2));
            iEJX = sub2(iEJX, mul2(mul2(eC, uJ0), uI2));
            iEIY = fma2(mul2(eC, uI0), uJ1, iEIY);
            iEJY = fma2(mul2(eC, uJ0), uI1, iEJY);
            const f2 uu = fma2(uI1, uJ1, mul2(uI2, uJ2));
            fIZ = fma2(dC, uu, fIZ);
            fJZ = fma2(dC, uu, fJZ);
        }
        // nqf = -qf (the QI-frame force); every sign flip below is exact.
        const f2 nqf0 = neg2(mul2(RINV, add2(add2(EIY, EJY), add2(iEIY, iEJY))));
        const f2 nqf1 = mul2(RINV, add2(add2(EIX, EJX), add2(iEIX, iEJX)));
        const f2 nqf2 = add2(fJZ, fIZ);
        // Back rotation with the reference's permuted matrix: nfv = -fv.
        const f2 nfvx = fma2(YY, nqf0, fma2(ZY, nqf1, mul2(XY, nqf2)));
        const f2 nfvy = fma2(YZ, nqf0, fma2(ZZ, nqf1, mul2(XZ, nqf2)));
        const f2 nfvz = fma2(YX, nqf0, fma2(ZX, nqf1, mul2(XX, nqf2)));
        {
            const f2 EIZ = sub2(mul2(QI2, Vij3), mul2(QI3, Vij2));
            // Torque of the QI-frame vector -E_I, rotated back (sign folded into the sub).
            TX = sub2(TX, fma2(YY, EIX, fma2(ZY, EIY, mul2(XY, EIZ))));
            TY = sub2(TY, fma2(YZ, EIX, fma2(ZZ, EIY, mul2(XZ, EIZ))));
            TZ = sub2(TZ, fma2(YX, EIX, fma2(ZX, EIY, mul2(XX, EIZ))));
            FX = add2(FX, nfvx);
            FY = add2(FY, nfvy);
            FZ = add2(FZ, nfvz);
            f2 eq = fma2(QI0, Vij0, mul2(QJ0, Vji0));
            eq = fma2(QI1, Vij1, fma2(QJ1, Vji1, eq));
            eq = fma2(QI2, Vij2, fma2(QJ2, Vji2, eq));
            eq = fma2(QI3, Vij3, fma2(QJ3, Vji3, eq));
            EN = fma2(HALF, eq, EN);
        }
        {
            const f2 EJZ = sub2(mul2(QJ2, Vji3), mul2(QJ3, Vji2));
            UX = sub2(UX, fma2(YY, EJX, fma2(ZY, EJY, mul2(XY, EJZ))));
            UY = sub2(UY, fma2(YZ, EJX, fma2(ZZ, EJY, mul2(XZ, EJZ))));
            UZ = sub2(UZ, fma2(YX, EJX, fma2(ZX, EJY, mul2(XX, EJZ))));
            GX = sub2(GX, nfvx);
            GY = sub2(GY, nfvy);
            GZ = sub2(GZ, nfvz);
        }
        // Rotate the packed J-side sums one lane (64-bit shuffles).
        GX = __shfl_sync(kFull, GX, nxt);
        GY = __shfl_sync(kFull, GY, nxt);
        GZ = __shfl_sync(kFull, GZ, nxt);
        UX = __shfl_sync(kFull, UX, nxt);
        UY = __shfl_sync(kFull, UY, nxt);
        UZ = __shfl_sync(kFull, UZ, nxt);
    }
    float lo, hi;
    const f2* Is[7] = {&FX, &FY, &FZ, &TX, &TY, &TZ, &EN};
    float* Io[7] = {&f[0], &f[1], &f[2], &f[3], &f[4], &f[5], &en};
#pragma unroll
    for (int k = 0; k < 7; k++) {
        un2(*Is[k], lo, hi);
        *Io[k] += lo + hi;
    }
    // Lane l now holds (atom l & 15, atom (l & 15) + 16); lane l ^ 16 the other copy.
    const f2 Js[6] = {GX, GY, GZ, UX, UY, UZ};
#pragma unroll
    for (int k = 0; k < 6; k++) {
        un2(Js[k], lo, hi);
        const float olo = __shfl_xor_sync(kFull, lo, 16), ohi = __shfl_xor_sync(kFull, hi, 16);
        gg[k] += lane < 16 ? lo + olo : hi + ohi;
    }
}

// ---------------------------------------------------------------------------
// Packed FP32 energy walk for tile pairs that no Thole damping reaches (every
// damping factor 1), with unit scales and rInvVec[4] = 0 (the default, see
// TDP_FLAG_DD_FORCE_R4).  It computes the reference's pair routine
// (RTDF.cpp:129-366) in the lab frame.  With all damping factors 1 the
// permanent and induced coefficients of calculateElectrostaticPairIxn merge
// and every rInvVec[4] term vanishes; what is left of the quasi-internal
// frame is its X row, the axis its multipole algebra treats as the bond axis
// (component 0).  With P = m + u and W = m + 2u (W = m without the
// induced-induced terms, i.e. unless Mutual), X-components written _0:
//   E   = q_i q_j / r + (q_j (P_i0 + m_i0) - q_i (P_j0 + m_j0)) / (2 r^2)
//         + (m_i.P_j + m_j.P_i - 3 (m_i0 P_j0 + m_j0 P_i0)) / (2 r^3)
//   V_ij = (q_j/r^2 - 3 P_j0/r^3) X + P_j/r^3,  V_ji = (-q_i/r^2 - 3 P_i0/r^3) X + P_i/r^3
//   Vd_ij, Vd_ji: the same with W for P
//   S   = m_i x V_ij + m_j x V_ji + u_i x Vd_ij + u_j x Vd_ji
//   f   = (S x X) / r + (q_i q_j / r^2 - 2 (q_i P_j0 - q_j P_i0) / r^3) X
//   F_i -= perm(f), F_j += perm(f), tau_i = -perm(m_i x V_ij), tau_j = -perm(m_j x V_ji)
// where perm(v) = (v_y, v_z, v_x) is the reference's permuted back rotation
// (:150-159).  This is an exact rewrite (FP64 transcriptions of both agree to
// rounding), with X from the frame test as there: X = (x^ - Z_x Z)/|.| when
// the pair's y or z coordinates differ (:584), written here as
// (d_y^2 + d_z^2, -d_x d_y, -d_x d_z) / (r sqrt(d_y^2 + d_z^2)); pairs within
// 1e-5 nm of the x axis take the reference's test and Gram-Schmidt as is.
// ---------------------------------------------------------------------------
__device__ __forceinline__ f2 xneg2(f2 a) { return a ^ 0x8000000080000000ull; }


// X row of formQIRotationMatrix (RTDF.cpp:580-593) for one pair, as the
// general walk forms it.
__device__ __forceinline__ void qi_frame_x(float dx, float dy, float dz, float rinv, bool yzd, float& xx, float& xy,
                                           float& xz) {
    const float zx = dx * rinv, zy = dy * rinv, zz = dz * rinv;
    xx = zx + (yzd ? 1.0f : 0.0f);
    xy = zy + (yzd ? 0.0f : 1.0f);
    xz = zz;
    const float dt = zx * xx + zy * xy + zz * xz;
    xx -= zx * dt;
    xy -= zy * dt;
    xz -= zz * dt;
    const float n2 = xx * xx + xy * xy + xz * xz;
    const float s = n2 > 0.0f ? rsqrtf(n2) : 1.0f;
    xx *= s;
    xy *= s;
    xz *= s;
}

template <bool FOLD>
__device__ __forceinline__ void energy_walk_x2_fast(const PairParams& P, const double* __restrict__ pos,
                                                    const double2* __restrict__ yz, const EPackedTile& T, int lane,
                                                    int i, int jbase, float oix, float oiy, float oiz, float4 pi,
                                                    float4 di, float4 ui, unsigned fm, bool mutual, float f[6],
                                                    float gg[6], float& en) {
    const int nxt = (lane + 1) & 31;
    const int nmax = P.n_tiles * 32 - 1;
    const f2 OX = bc2(oix), OY = bc2(oiy), OZ = bc2(oiz);
    const float kap = mutual ? 1.0f : -1.0f;   // W = P + kap u
    const f2 KAP = bc2(kap);
    const f2 QI0 = bc2(pi.w), NQI0 = bc2(-pi.w);
    const f2 MIX = bc2(di.x), MIY = bc2(di.y), MIZ = bc2(di.z);
    const f2 UIX = bc2(ui.x), UIY = bc2(ui.y), UIZ = bc2(ui.z);
    const float pix = di.x + ui.x, piy = di.y + ui.y, piz = di.z + ui.z;
    const f2 PIX = bc2(pix), PIY = bc2(piy), PIZ = bc2(piz);
    const f2 HALF = bc2(0.5f), NTHREE = bc2(-3.0f), NTWO = bc2(-2.0f);
    f2 Lx = 0, Ly = 0, Lz = 0, Ix = 0, Iy = 0, Iz = 0, NTx = 0, NTy = 0, NTz = 0;
    if (FOLD) {
        Lx = bc2(-(float)P.box[0]);
        Ly = bc2(-(float)P.box[1]);
        Lz = bc2(-(float)P.box[2]);
        Ix = bc2((float)P.inv_box[0]);
        Iy = bc2((float)P.inv_box[1]);
        Iz = bc2((float)P.inv_box[2]);
        NTx = bc2(-(float)(P.half_box_tol[0] * P.half_box_tol[0]));
        NTy = bc2(-(float)(P.half_box_tol[1] * P.half_box_tol[1]));
        NTz = bc2(-(float)(P.half_box_tol[2] * P.half_box_tol[2]));
    }
    // Torques from summed V (pair_energy_lab, VSUM): TX.. sum V_ij, UX.. V_ji.
    f2 FX = 0, FY = 0, FZ = 0, TX = 0, TY = 0, TZ = 0, EN = 0;        // I side
    f2 GX = 0, GY = 0, GZ = 0, UX = 0, UY = 0, UZ = 0;                // J side (packed atoms m, m + 16)
#pragma unroll 1
    for (int s = 0; s < 16; s++) {
        const int m = (lane + s) & 15;
        const float4 a = T.p0[m], b = T.p1[m], c = T.d0[m], d = T.d1[m], e = T.u0[m], h = T.u1[m];
        f2 DX = sub2(pk2(a.x, a.y), OX), DY = sub2(pk2(a.z, a.w), OY), DZ = sub2(pk2(b.x, b.y), OZ);
        const int ja = jbase + m, jb = ja + 16;
        if (FOLD) {
            f2 neg = ~0ull;
            if (fm & 1u) {
                DX = fold2(DX, Lx, Ix);
                neg &= fma2(DX, DX, NTx);
            }
            if (fm & 2u) {
                DY = fold2(DY, Ly, Iy);
                neg &= fma2(DY, DY, NTy);
            }
            if (fm & 4u) {
                DZ = fold2(DZ, Lz, Iz);
                neg &= fma2(DZ, DZ, NTz);
            }
            const f2 flag = ~neg & 0x8000000080000000ull;
            if (flag) {
                const bool amb_a = (flag >> 31) & 1ull, amb_b = (flag >> 63) != 0ull;
                float ax, bx, ay, by, az, bz;
                un2(DX, ax, bx);
                un2(DY, ay, by);
                un2(DZ, az, bz);
                if (amb_a) {
                    d3 q = exact_delta(P, pos, i, ja);
                    ax = (float)q.x;
                    ay = (float)q.y;
                    az = (float)q.z;
                }
                if (amb_b) {
                    d3 q = exact_delta(P, pos, i, jb);
                    bx = (float)q.x;
                    by = (float)q.y;
                    bz = (float)q.z;
                }
                DX = pk2(ax, bx);
                DY = pk2(ay, by);
                DZ = pk2(az, bz);
            }
        }
        float r2a, r2b, ra, rb;
        un2(dot2(DX, DY, DZ, DX, DY, DZ), r2a, r2b);
        const f2 RINV = pk2(rsqrtf(r2a), rsqrtf(r2b));
        const f2 RHO2 = fma2(DY, DY, mul2(DZ, DZ));
        un2(RHO2, ra, rb);
        // Frame X row (see above).
        const f2 XS = mul2(RINV, pk2(rsqrtf(ra), rsqrtf(rb)));
        const f2 NDXS = mul2(xneg2(DX), XS);
        f2 XX = mul2(RHO2, XS), XY = mul2(NDXS, DY), XZ = mul2(NDXS, DZ);
        if (ra <= 1.0e-10f || rb <= 1.0e-10f) {
            float dxa, dxb, dya, dyb, dza, dzb, rva, rvb, xxa, xxb, xya, xyb, xza, xzb;
            un2(DX, dxa, dxb);
            un2(DY, dya, dyb);
            un2(DZ, dza, dzb);
            un2(RINV, rva, rvb);
            un2(XX, xxa, xxb);
            un2(XY, xya, xyb);
            un2(XZ, xza, xzb);
            if (ra <= 1.0e-10f) qi_frame_x(dxa, dya, dza, rva, yz_differ<float>(dya, dza, yz, i, ja, nmax), xxa, xya, xza);
            if (rb <= 1.0e-10f) qi_frame_x(dxb, dyb, dzb, rvb, yz_differ<float>(dyb, dzb, yz, i, jb, nmax), xxb, xyb, xzb);
            XX = pk2(xxa, xxb);
            XY = pk2(xya, xyb);
            XZ = pk2(xza, xzb);
        }
        const f2 QJ0 = pk2(b.z, b.w);
        const f2 MJX = pk2(c.x, c.y), MJY = pk2(c.z, c.w), MJZ = pk2(d.x, d.y);
        const f2 UJX = pk2(e.x, e.y), UJY = pk2(e.z, e.w), UJZ = pk2(h.x, h.y);
        const f2 PJX = add2(MJX, UJX), PJY = add2(MJY, UJY), PJZ = add2(MJZ, UJZ);
        const f2 PI0 = dot2(XX, XY, XZ, PIX, PIY, PIZ), UI0 = dot2(XX, XY, XZ, UIX, UIY, UIZ);
        const f2 PJ0 = dot2(XX, XY, XZ, PJX, PJY, PJZ), UJ0 = dot2(XX, XY, XZ, UJX, UJY, UJZ);
        const f2 rv2 = mul2(RINV, RINV), rv3 = mul2(rv2, RINV);
        const f2 NR3X3 = mul2(NTHREE, rv3);
        // Energy: the charge terms here; the dipole terms 0.5 (m_i.V_ij +
        // m_j.V_ji) come from the V sums after the walk (pair_energy_lab, VSUM).
        {
            const f2 qq = mul2(QI0, QJ0);
            const f2 cp = fma2(QJ0, PI0, mul2(NQI0, PJ0));
            EN = fma2(RINV, qq, fma2(mul2(HALF, rv2), cp, EN));
        }
        const f2 rv2QJ0 = mul2(rv2, QJ0), rv2NQI0 = mul2(rv2, NQI0);
        // S = K x X with K = a m_i + b m_j + c u_i + d u_j (pair_energy_lab):
        // the torques need m_i x V_ij and m_j x V_ji, the force only K.
        const f2 aJ = fma2(NR3X3, PJ0, rv2QJ0);
        const f2 bI = fma2(NR3X3, PI0, rv2NQI0);
        // V_ij (I torque) and V_ji (J torque), summed; the cross products with
        // m_i and m_j come once per atom after the walk.
        TX = fma2(aJ, XX, fma2(rv3, PJX, TX));
        TY = fma2(aJ, XY, fma2(rv3, PJY, TY));
        TZ = fma2(aJ, XZ, fma2(rv3, PJZ, TZ));
        UX = fma2(bI, XX, fma2(rv3, PIX, UX));
        UY = fma2(bI, XY, fma2(rv3, PIY, UY));
        UZ = fma2(bI, XZ, fma2(rv3, PIZ, UZ));
        {
            const f2 cJ = fma2(NR3X3, fma2(KAP, UJ0, PJ0), rv2QJ0);
            const f2 dI = fma2(NR3X3, fma2(KAP, UI0, PI0), rv2NQI0);
            const f2 KX = fma2(aJ, MIX, fma2(bI, MJX, fma2(cJ, UIX, mul2(dI, UJX))));
            const f2 KY = fma2(aJ, MIY, fma2(bI, MJY, fma2(cJ, UIY, mul2(dI, UJY))));
            const f2 KZ = fma2(aJ, MIZ, fma2(bI, MJZ, fma2(cJ, UIZ, mul2(dI, UJZ))));
            const f2 qf2 = fma2(mul2(NTWO, rv3), fma2(QI0, PJ0, xneg2(mul2(QJ0, PI0))), mul2(rv2QJ0, QI0));
            // f = (S x X) / r + qf2 X = (rinv K.X + qf2) X - rinv K.
            const f2 CF = fma2(RINV, dot2(KX, KY, KZ, XX, XY, XZ), qf2);
            const f2 NRINV = xneg2(RINV);
            const f2 FVX = fma2(CF, XX, mul2(NRINV, KX)), FVY = fma2(CF, XY, mul2(NRINV, KY)),
                     FVZ = fma2(CF, XZ, mul2(NRINV, KZ));
            FX = sub2(FX, FVY);
            FY = sub2(FY, FVZ);
            FZ = sub2(FZ, FVX);
            GX = add2(GX, FVY);
            GY = add2(GY, FVZ);
            GZ = add2(GZ, FVX);
        }
        GX = __shfl_sync(kFull, GX, nxt);
        GY = __shfl_sync(kFull, GY, nxt);
        GZ = __shfl_sync(kFull, GZ, nxt);
        UX = __shfl_sync(kFull, UX, nxt);
        UY = __shfl_sync(kFull, UY, nxt);
        UZ = __shfl_sync(kFull, UZ, nxt);
    }
    float lo, hi;
    const f2* Is[4] = {&FX, &FY, &FZ, &EN};
    float* Io[4] = {&f[0], &f[1], &f[2], &en};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        un2(*Is[k], lo, hi);
        *Io[k] += lo + hi;
    }
    float v[3];
    const f2 Vs[3] = {TX, TY, TZ};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        un2(Vs[k], lo, hi);
        v[k] = lo + hi;
    }
    // tau_I = -perm(m_i x sum V_ij); dipole energy 0.5 m_i.sum V_ij.
    en += 0.5f * (di.x * v[0] + di.y * v[1] + di.z * v[2]);
    f[3] -= di.z * v[0] - di.x * v[2];
    f[4] -= di.x * v[1] - di.y * v[0];
    f[5] -= di.y * v[2] - di.z * v[1];
    const f2 Js[6] = {GX, GY, GZ, UX, UY, UZ};
    float w[6];
#pragma unroll
    for (int k = 0; k < 6; k++) {
        un2(Js[k], lo, hi);
        const float olo = __shfl_xor_sync(kFull, lo, 16), ohi = __shfl_xor_sync(kFull, hi, 16);
        w[k] = lane < 16 ? lo + olo : hi + ohi;
    }
    gg[0] += w[0];
    gg[1] += w[1];
    gg[2] += w[2];
    // Lane l now holds J atom l: tau_J = -perm(m_j x sum V_ji).
    const int m = lane & 15, h = lane >> 4;
    const float mjx = reinterpret_cast<const float*>(&T.d0[m])[h];
    const float mjy = reinterpret_cast<const float*>(&T.d0[m])[2 + h];
    const float mjz = reinterpret_cast<const float*>(&T.d1[m])[h];
    gg[3] -= mjz * w[3] - mjx * w[5];
    gg[4] -= mjx * w[4] - mjy * w[3];
    gg[5] -= mjy * w[5] - mjz * w[4];
    en += 0.5f * (mjx * w[3] + mjy * w[4] + mjz * w[5]);
}

// Partner pairs of a SLOW tile pair with their (M, I) scales, each side once:
// the lane's I atom with its partners in J (the pair energy is counted on the
// lower-index side), and atom l of J (off the diagonal) with its partners in I.
template <class R, bool FOLD>
__device__ __forceinline__ void energy_partners(
    const PairParams& P, const double* __restrict__ pos, const double2* __restrict__ yz,
    const typename Vec4T<R>::type* __restrict__ posq, const typename Vec4T<R>::type* __restrict__ dipt,
    const typename Vec4T<R>::type* __restrict__ indv, const typename Vec4T<R>::type* __restrict__ sp,
    const typename Vec4T<R>::type* __restrict__ sd, const typename Vec4T<R>::type* __restrict__ su,
    const int* __restrict__ exc_off, const int* __restrict__ exc_j, const double* __restrict__ exc_m,
    const double* __restrict__ exc_s, const TileGeom& geo, double4 cA, double4 cB, int lane, int i, int ibase,
    int jbase, int e0, int e1, R oix, R oiy, R oiz, const EAtom<R>& me, bool diag, R damp_r2, R rv4p, R rv4f, R f[6],
    R g[6], R& en) {
    typedef typename Vec4T<R>::type V4;
    const int nmax = P.n_tiles * 32 - 1;
#pragma unroll 1
    for (int e = e0; e < e1; e++) {
        unsigned off = (unsigned)(exc_j[e] - jbase);
        if (off >= 32u) continue;
        const R mS = (R)exc_m[e], iS = (R)exc_s[e];
        if (mS == R(0) && iS == R(0)) continue;
        const int j = jbase + (int)off;
        const EAtom<R> other = eatom<R>(sp[off], sd[off], su[off]);
        R dx, dy, dz;
        pair_delta<R, FOLD>(P, pos, i, j, sp[off].x, sp[off].y, sp[off].z, oix, oiy, oiz, dx, dy, dz);
        const R r2 = dx * dx + dy * dy + dz * dz;
        const bool yzd = yz_differ<R>(dy, dz, yz, i, j, nmax);
        if (j > i)
            pair_energy<R, true>(dx, dy, dz, r2, yzd, me, other, mS, iS, damp_r2, rv4p, rv4f, P.mutual != 0, f[0],
                                 f[1], f[2], f[3], f[4], f[5], en);
        else
            pair_energy<R, false>(-dx, -dy, -dz, r2, yzd, other, me, mS, iS, damp_r2, rv4p, rv4f, P.mutual != 0,
                                  f[0], f[1], f[2], f[3], f[4], f[5], en);
    }
    if (diag) return;
    const int jl = jbase + lane;
    if (jl >= P.n) return;
    const EAtom<R> mine = eatom<R>(sp[lane], sd[lane], su[lane]);
    R dummy = 0;
#pragma unroll 1
    for (int e = exc_off[jl]; e < exc_off[jl + 1]; e++) {
        const int a = exc_j[e];
        if ((unsigned)(a - ibase) >= 32u) continue;
        const R mS = (R)exc_m[e], iS = (R)exc_s[e];
        if (mS == R(0) && iS == R(0)) continue;
        const V4 pa = posq[a];
        const EAtom<R> A = eatom<R>(pa, dipt[a], indv[a]);
        R ox, oy, oz;
        shift_into<R>(geo, cA, cB, pa.x, pa.y, pa.z, ox, oy, oz);
        R dx, dy, dz;  // p_jl - p_a: a (tile I < J) is the lower index
        pair_delta<R, FOLD>(P, pos, a, jl, sp[lane].x, sp[lane].y, sp[lane].z, ox, oy, oz, dx, dy, dz);
        const R r2 = dx * dx + dy * dy + dz * dz;
        const bool yzd = yz_differ<R>(dy, dz, yz, a, jl, nmax);
        pair_energy<R, false>(dx, dy, dz, r2, yzd, A, mine, mS, iS, damp_r2, rv4p, rv4f, P.mutual != 0, g[0], g[1],
                              g[2], g[3], g[4], g[5], dummy);
    }
}

template <class R>
__global__ void __launch_bounds__(kSymThreads, 3) k_energy_sym(
    PairParams P, const typename Vec4T<R>::type* __restrict__ posq, const typename Vec4T<R>::type* __restrict__ dipt,
    const typename Vec4T<R>::type* __restrict__ indv, const double2* __restrict__ yz, const double4* __restrict__ tctr,
    const double4* __restrict__ text, const double* __restrict__ pos, const int* __restrict__ exc_off,
    const int* __restrict__ exc_j, const double* __restrict__ exc_m, const double* __restrict__ exc_s,
    const int2* __restrict__ exc_tiles, int n_pad, double* __restrict__ partial, double* __restrict__ energy_partial,
    FixAcc fix) {
    typedef typename Vec4T<R>::type V4;
    extern __shared__ __align__(16) unsigned char smem[];
    const int BT = P.band_tiles, NA = BT * 32;
    double* s_acc = reinterpret_cast<double*>(smem);              // 6 * NA: J-side sums of band q
    double* s_iacc = s_acc + 6 * NA;                               // 7 * kSymThreads: I-side sums and energy
    double4* s_ctr = reinterpret_cast<double4*>(s_iacc + 7 * kSymThreads);
    double4* s_ext = s_ctr + BT;
    V4* s_pos = reinterpret_cast<V4*>(s_ext + BT);
    V4* s_dip = s_pos + NA;
    V4* s_ind = s_dip + NA;
    __shared__ EPackedTile s_ept[sizeof(R) == 4 ? kSymWarps : 1];   // packed walk's J tile (mixed form)

    int p, q;
    band_pair(blockIdx.x, p, q);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int qa0 = q * NA;
    for (int k = threadIdx.x; k < NA; k += kSymThreads) {
        s_pos[k] = posq[qa0 + k];
        s_dip[k] = dipt[qa0 + k];
        s_ind[k] = indv[qa0 + k];
        for (int c = 0; c < 6; c++) s_acc[6 * k + c] = 0.0;
    }
    for (int k = threadIdx.x; k < BT; k += kSymThreads) {
        s_ctr[k] = tctr[q * BT + k];
        s_ext[k] = text[q * BT + k];
    }
    double* my = s_iacc + 7 * threadIdx.x;
    my[6] = 0.0;
    __syncthreads();

    const R damp_r2 = (R)P.damp_r2;
    const R rv4p = (R)P.rinv4_power, rv4f = (R)P.rinv4_fill;
    const int stride = BT >= kSymWarps ? BT / kSymWarps : 1;
    const int rounds = (BT + kSymWarps - 1) / kSymWarps;
    for (int r = 0; r < rounds; r++) {
        const int Il = warp + kSymWarps * r;
        const int I = p * BT + Il;
        const bool wact = Il < BT && I < P.n_tiles;
        const int ibase = I * 32;
        const int i = ibase + lane;
        V4 pi = {}, di = {}, ui = {};
        double4 cA = {}, eA = {};
        int2 et = make_int2(1 << 30, -1);
        int e0 = 0, e1 = 0;
        if (wact) {
            pi = posq[i];
            di = dipt[i];
            ui = indv[i];
            cA = tctr[I];
            eA = text[I];
            et = exc_tiles[I];
            if (i < P.n) {
                e0 = exc_off[i];
                e1 = exc_off[i + 1];
            }
        }
        const EAtom<R> me = eatom<R>(pi, di, ui);
        // FP32 form: the round's BT tile-pair geometries (FP64 arithmetic), one
        // per lane, read by shuffles instead of every lane repeating each.
        float gdx = 0.f, gdy = 0.f, gdz = 0.f;
        unsigned gfl = 0u;
        if constexpr (sizeof(R) == 4) {
            if (wact && lane < BT) {
                const TileGeom g0 = tile_geom(P, cA, eA, s_ctr[lane], s_ext[lane]);
                gdx = (float)g0.dcx;
                gdy = (float)g0.dcy;
                gdz = (float)g0.dcz;
                gfl = g0.fmask | (g0.fold ? 8u : 0u) | (g0.near ? 16u : 0u);
            }
        }
        for (int c = 0; c < 6; c++) my[c] = 0.0;
        for (int t = 0; t < BT; t++) {
            const int Jl = (t + warp * stride) % BT;
            const int J = q * BT + Jl;
            if (wact && J < P.n_tiles && (p != q || Jl >= Il)) {
                const double4 cB = s_ctr[Jl];
                const bool diag = I == J;
                const bool slow = diag || (J == P.n_tiles - 1 && (P.n & 31)) || (J >= et.x && J <= et.y);
                TileGeom g;
                R oix, oiy, oiz;
                if constexpr (sizeof(R) == 4) {
                    const float dx = __shfl_sync(kFull, gdx, Jl), dy = __shfl_sync(kFull, gdy, Jl),
                                dz = __shfl_sync(kFull, gdz, Jl);
                    const unsigned fl = __shfl_sync(kFull, gfl, Jl);
                    oix = pi.x - dx;
                    oiy = pi.y - dy;
                    oiz = pi.z - dz;
                    if (slow) {
                        g = tile_geom(P, cA, eA, cB, s_ext[Jl]);   // the partner walk's FP64 geometry
                    } else {
                        g.fmask = fl & 7u;
                        g.fold = (fl >> 3) & 1u;
                        g.near = (fl >> 4) & 1u;
                    }
                } else {
                    g = tile_geom(P, cA, eA, cB, s_ext[Jl]);
                    shift_into<R>(g, cA, cB, pi.x, pi.y, pi.z, oix, oiy, oiz);
                }
                const int jbase = J * 32;
                const V4* sp = s_pos + Jl * 32;
                const V4* sd = s_dip + Jl * 32;
                const V4* su = s_ind + Jl * 32;
                const unsigned partners = slow ? partner_bits(exc_j, e0, e1, jbase) : 0u;
                R f[6] = {0, 0, 0, 0, 0, 0}, gg[6] = {0, 0, 0, 0, 0, 0}, en = 0;
                bool packed = false;
                if constexpr (sizeof(R) == 4) {
                    if (!slow) {
                        packed = true;
                        __syncwarp();
                        stage_epacked(s_ept[warp], lane, sp[lane], sd[lane], su[lane]);
                        __syncwarp();
                        if (!g.near && P.lab_energy) {
                            if (g.fold)
                                energy_walk_x2_fast<true>(P, pos, yz, s_ept[warp], lane, i, jbase, oix, oiy, oiz, pi,
                                                          di, ui, g.fmask, P.mutual != 0, f, gg, en);
                            else
                                energy_walk_x2_fast<false>(P, pos, yz, s_ept[warp], lane, i, jbase, oix, oiy, oiz, pi,
                                                           di, ui, g.fmask, P.mutual != 0, f, gg, en);
                        } else if (g.fold)
                            energy_walk_x2<true>(P, pos, yz, s_ept[warp], lane, i, jbase, oix, oiy, oiz, pi, di, ui,
                                                 g.fmask, damp_r2, rv4p, rv4f, P.mutual != 0, f, gg, en);
                        else
                            energy_walk_x2<false>(P, pos, yz, s_ept[warp], lane, i, jbase, oix, oiy, oiz, pi, di, ui,
                                                  g.fmask, damp_r2, rv4p, rv4f, P.mutual != 0, f, gg, en);
                    }
                }
                if (packed) {
                } else if (slow) {
                    if (g.fold) {
                        energy_walk<R, true, true>(P, pos, yz, sp, sd, su, lane, i, jbase, oix, oiy, oiz, me, diag,
                                                   partners, damp_r2, rv4p, rv4f, f, gg, en);
                        energy_partners<R, true>(P, pos, yz, posq, dipt, indv, sp, sd, su, exc_off, exc_j, exc_m,
                                                 exc_s, g, cA, cB, lane, i, ibase, jbase, e0, e1, oix, oiy, oiz, me,
                                                 diag, damp_r2, rv4p, rv4f, f, gg, en);
                    } else {
                        energy_walk<R, false, true>(P, pos, yz, sp, sd, su, lane, i, jbase, oix, oiy, oiz, me, diag,
                                                    partners, damp_r2, rv4p, rv4f, f, gg, en);
                        energy_partners<R, false>(P, pos, yz, posq, dipt, indv, sp, sd, su, exc_off, exc_j, exc_m,
                                                  exc_s, g, cA, cB, lane, i, ibase, jbase, e0, e1, oix, oiy, oiz, me,
                                                  diag, damp_r2, rv4p, rv4f, f, gg, en);
                    }
                } else if (!g.near && P.lab_energy) {
                    if (g.fold)
                        energy_walk<R, true, false, true>(P, pos, yz, sp, sd, su, lane, i, jbase, oix, oiy, oiz, me,
                                                          diag, partners, damp_r2, rv4p, rv4f, f, gg, en);
                    else
                        energy_walk<R, false, false, true>(P, pos, yz, sp, sd, su, lane, i, jbase, oix, oiy, oiz, me,
                                                           diag, partners, damp_r2, rv4p, rv4f, f, gg, en);
                } else if (g.fold) {
                    energy_walk<R, true, false>(P, pos, yz, sp, sd, su, lane, i, jbase, oix, oiy, oiz, me, diag,
                                                partners, damp_r2, rv4p, rv4f, f, gg, en);
                } else {
                    energy_walk<R, false, false>(P, pos, yz, sp, sd, su, lane, i, jbase, oix, oiy, oiz, me, diag,
                                                 partners, damp_r2, rv4p, rv4f, f, gg, en);
                }
                double* acc = s_acc + 6 * (Jl * 32 + lane);
                for (int c = 0; c < 6; c++) {
                    acc[c] += (double)gg[c];
                    my[c] += (double)f[c];
                }
                my[6] += (double)en;
            }
            // Within a window of `stride` steps the warps' J tiles are
            // disjoint ((t + warp * stride) % BT), so the shared J-side sums
            // need a barrier only between windows; the windows' order fixes the
            // order of the additions (deterministic).
            if ((t + 1) % stride == 0 || t + 1 == BT) __syncthreads();
        }
        if (wact) {
            if (p == q) {
                double* acc = s_acc + 6 * (Il * 32 + lane);
                for (int c = 0; c < 6; c++) acc[c] += my[c];
            } else if (sizeof(R) == 4) {
                for (int c = 0; c < 6; c++) fix_add(fix, (size_t)c * n_pad + i, my[c]);
            } else {
                const size_t b = (size_t)q * 6 * n_pad;
                for (int c = 0; c < 6; c++) partial[b + (size_t)c * n_pad + i] = my[c];
            }
        }
        __syncthreads();
    }
    const size_t b = (size_t)p * 6 * n_pad;
    for (int k = threadIdx.x; k < NA; k += kSymThreads)
        for (int c = 0; c < 6; c++) {
            if (sizeof(R) == 4) fix_add(fix, (size_t)c * n_pad + qa0 + k, s_acc[6 * k + c]);
            else partial[b + (size_t)c * n_pad + qa0 + k] = s_acc[6 * k + c];
        }
    // CTA energy, summed in thread order (padding atoms contribute exactly 0).
    double e = warp_sum(my[6]);
    __shared__ double s_red[kSymWarps];
    if (lane == 0) s_red[warp] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kSymWarps; w++) s += s_red[w];
        energy_partial[blockIdx.x] = s;
    }
}

template <class R>
size_t field_smem(int BT) {
    const int NA = 32 * BT;
    return sizeof(double) * 6 * kSymThreads + sizeof(double4) * (2 * BT + 4 * kSymWarps) +
           sizeof(typename Vec4T<R>::type) * 2 * NA + sizeof(R) * kSymWarps * 3 * NA +
           (sizeof(R) == 4 ? sizeof(FPackedTile) * kSymWarps : 0);
}

template <class R>
size_t energy_smem(int BT) {
    const int NA = 32 * BT;
    return sizeof(double) * (6 * NA + 7 * kSymThreads) + sizeof(double4) * 2 * BT +
           sizeof(typename Vec4T<R>::type) * 3 * NA;
}

int band_pairs(const Dev& d) { return d.pp.n_bands * (d.pp.n_bands + 1) / 2; }

// Fixed-point accumulator -> partial slot 0 (ncomp components of n_pad), clearing it.
__global__ void k_fix_flush(size_t count, unsigned long long* __restrict__ acc, double inv_scale,
                            double* __restrict__ out) {
    size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    long long v = (long long)acc[k];
    acc[k] = 0ull;
    out[k] = (double)v * inv_scale;
}

FixAcc fix_of(const Dev& d) { return FixAcc{d.fixacc, d.fix_err, d.fix_scale, d.fix_limit}; }

void fix_flush(const Dev& d, int ncomp, cudaStream_t st) {
    if (!d.fixacc) return;
    const size_t count = (size_t)ncomp * d.n_pad;
    k_fix_flush<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(count, d.fixacc, 1.0 / d.fix_scale, d.partial);
}

}  // namespace

// kind 0: permanent field (operand: the lab dipoles); kind 1: mutual-field
// matvec (operand: vec); kind 2: the start of a warm-started solve, the
// permanent field plus T mu0 in one walk (operand vec = m + mu0, see
// field_partners).
template <class R>
void launch_field(const Dev& d, int kind, cudaStream_t st) {
    typedef typename Vec4T<R>::type V4;
    const size_t smem = field_smem<R>(d.pp.band_tiles);
    // Field kernels run on the spatially sorted records.
    if (kind == 0 || kind == 2) {
        cudaFuncSetAttribute(k_field_sym<R, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_field_sym<R, 0><<<band_pairs(d), kSymThreads, smem, st>>>(
            d.pp, (const V4*)d.posq_s, (const V4*)(kind == 0 ? d.dipt_s : d.vec_s), d.tctr_s, d.text_s, d.pos_s,
            d.exs_off, d.exs_j, d.exs_m, d.exs_s, d.exs_tiles, d.n_pad, d.partial, fix_of(d),
            kind == 2 ? (const V4*)d.dipt_s : nullptr);
    } else {
        cudaFuncSetAttribute(k_field_sym<R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_field_sym<R, 1><<<band_pairs(d), kSymThreads, smem, st>>>(
            d.pp, (const V4*)d.posq_s, (const V4*)d.vec_s, d.tctr_s, d.text_s, d.pos_s, d.exs_off, d.exs_j, d.exs_m,
            d.exs_s, d.exs_tiles, d.n_pad, d.partial, fix_of(d), nullptr);
    }
    if (sizeof(R) == 4) fix_flush(d, 3, st);
}

template <class R>
void launch_energy(const Dev& d, cudaStream_t st) {
    typedef typename Vec4T<R>::type V4;
    const size_t smem = energy_smem<R>(d.pp.band_tiles);
    cudaFuncSetAttribute(k_energy_sym<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_energy_sym<R><<<band_pairs(d), kSymThreads, smem, st>>>(
        d.pp, (const V4*)d.posq, (const V4*)d.dipt, (const V4*)d.ind, d.yz, d.tctr, d.text, d.pos, d.exc_off, d.exc_j,
        d.exc_m, d.exc_s, d.exc_tiles, d.n_pad, d.partial, d.energy_partial, fix_of(d));
    if (sizeof(R) == 4) fix_flush(d, 6, st);
}

template void launch_field<float>(const Dev&, int, cudaStream_t);
template void launch_field<double>(const Dev&, int, cudaStream_t);
template void launch_energy<float>(const Dev&, cudaStream_t);
template void launch_energy<double>(const Dev&, cudaStream_t);

}  // namespace tdp
