// sgm_step.cuh -- one step of the SGM path recurrence, disparities across lanes.
//
// Reference semantics (src/sgbm_kernels.cu:338-360, identical in all eight
// path kernels), all values uint16 with wrap on every assignment:
//   C       = (u16)(cost * costScale)
//   L[d]    = (u16)(C + min(L'[d], (u16)(L'[d-1]+P1), (u16)(L'[d+1]+P1),
//                           (u16)(minL' + P2adj)) - minL')
// with L'[-1] and L'[D] contributing 0xFFFF.
//
// Layout: a warp owns one pixel of one path; lane l holds disparities
// [2*KW*l, 2*KW*l + 2*KW) as KW packed uint16x2 words (low half = even d).
// The neighbour words (L'[d-1], L'[d]) are built with one byte-permute per
// word plus one shuffle each way at the lane edges, so a step costs two
// shuffles and one warp min-reduction (redux.sync) regardless of KW.
//
// Two arithmetic modes, both bit-exact to the reference:
//  * WRAP  = true : per-halfword modular arithmetic (__vadd2/__vsub2), valid
//    for any parameters.
//  * WRAP  = false: plain 32-bit integer adds on the packed words.  The host
//    selects it only when it has proved that no halfword can leave [0, 65535]
//    (255*costScale + max(P1+1, P2) + P1 <= 65535, P1 >= 0 and the summed
//    paths fit), in which case the modular and the integer results coincide
//    and carries never cross halves.  L >= minL' holds there, so
//    L = min(...) + C - minL' is one IADD3 with no borrow.
// Boundary neighbours: the half holding L'[-1] (lane 0) or L'[D] is replaced
// by (0xFFFF - P1) mod 2^16 before P1 is added, which yields the reference's
// 0xFFFF exactly in both modes.  Disparities d >= D (padding) are forced to
// 0xFFFF after each step so they never win the minimum.
#pragma once
#include "common.cuh"

namespace lumen {

constexpr unsigned kFull = kFullMask;

template <int KW>
struct LaneMasks {
    uint32_t nbMask[KW + 1];  // halves of nb[j] replaced by the boundary stand-in
    uint32_t padMask[KW];     // halves of word i with d >= D
};

// Per-lane masks for a team lane `lane` holding d = 2*KW*lane + (0..2KW-1).
template <int KW>
__device__ __forceinline__ void make_lane_masks(int lane, int D, LaneMasks<KW>& m) {
    const int base = 2 * KW * lane;
#pragma unroll
    for (int j = 0; j <= KW; ++j) {
        // nb[j] = (L'[base+2j-1], L'[base+2j])
        uint32_t mk = 0;
        if (base + 2 * j - 1 == -1) mk |= 0x0000FFFFu;         // left of d = 0
        if (base + 2 * j - 1 == D) mk |= 0x0000FFFFu;          // right of d = D-1 (D-1 even)
        if (base + 2 * j == D) mk |= 0xFFFF0000u;              // right of d = D-1 (D-1 odd)
        m.nbMask[j] = mk;
    }
#pragma unroll
    for (int i = 0; i < KW; ++i) {
        uint32_t pm = 0;
        if (base + 2 * i >= D) pm |= 0x0000FFFFu;
        if (base + 2 * i + 1 >= D) pm |= 0xFFFF0000u;
        m.padMask[i] = pm;
    }
}

// Scaled cost words from packed cost bytes (two disparities per word).
template <bool WRAP>
__device__ __forceinline__ uint32_t scale_cost(uint32_t pk, int costScale) {
    if (!WRAP) return pk * (uint32_t)costScale;  // host proved 255*costScale <= 65535
    const uint32_t lo = ((pk & 0xFFFFu) * (uint32_t)costScale) & 0xFFFFu;
    const uint32_t hi = ((pk >> 16) * (uint32_t)costScale) << 16;
    return lo | hi;
}

// min over the lane's words and both halves, then across the team of T lanes
// (T = 32: one redux.sync; T < 32: xor butterfly inside the T-lane segment).
template <int KW, int T = 32>
__device__ __forceinline__ uint32_t warp_min_u16(const uint32_t (&L)[KW]) {
    uint32_t m = L[0];
#pragma unroll
    for (int i = 1; i < KW; ++i) m = __vminu2(m, L[i]);
    m = min(m & 0xFFFFu, m >> 16);
    if constexpr (T == 32) {
        return __reduce_min_sync(kFull, m);
    } else {
#pragma unroll
        for (int o = T / 2; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(kFull, m, o));
        return m;
    }
}

// One recurrence step.  Lp: previous path costs; Cw: scaled matching costs of
// the current pixel; minPrev: min over d of Lp; p2: P2adj of this step;
// bsub: (0xFFFF - P1) in both halves (mod 2^16); p1x2: P1 in both halves.
// T: lanes per pixel (the team); lanes of a team are a contiguous, aligned
// segment of the warp and every lane of the warp executes the step.
template <int KW, bool WRAP, bool FULL, int T = 32>
__device__ __forceinline__ void sgm_step(const uint32_t (&Lp)[KW], const uint32_t (&Cw)[KW],
                                         uint32_t minPrev, int p2, uint32_t p1x2, uint32_t bsub,
                                         const LaneMasks<KW>& mk, uint32_t (&Ln)[KW]) {
    const uint32_t up = __shfl_up_sync(kFull, Lp[KW - 1], 1, T);
    const uint32_t dn = __shfl_down_sync(kFull, Lp[0], 1, T);
    uint32_t nb[KW + 1];
    nb[0] = __byte_perm(up, Lp[0], 0x5432);
#pragma unroll
    for (int j = 1; j < KW; ++j) nb[j] = __byte_perm(Lp[j - 1], Lp[j], 0x5432);
    nb[KW] = __byte_perm(Lp[KW - 1], dn, 0x5432);
    if (FULL) {
        // Only L'[-1] (team lane 0, nb[0] low) and L'[D] (last team lane, nb[KW] high) occur.
        nb[0] = (nb[0] & ~mk.nbMask[0]) | (bsub & mk.nbMask[0]);
        nb[KW] = (nb[KW] & ~mk.nbMask[KW]) | (bsub & mk.nbMask[KW]);
    } else {
#pragma unroll
        for (int j = 0; j <= KW; ++j) nb[j] = (nb[j] & ~mk.nbMask[j]) | (bsub & mk.nbMask[j]);
    }
    const uint32_t mpx2 = minPrev * 0x10001u;
    if (!WRAP) {
        const uint32_t mp2 = (minPrev + (uint32_t)p2) * 0x10001u;
#pragma unroll
        for (int i = 0; i < KW; ++i) {
            const uint32_t t = __vminu2(nb[i], nb[i + 1]) + p1x2;
            const uint32_t m = __vminu2(__vminu2(t, Lp[i]), mp2);
            uint32_t l = m + Cw[i] - mpx2;
            if (!FULL) l |= mk.padMask[i];
            Ln[i] = l;
        }
    } else {
        const uint32_t mp2 = ((minPrev + (uint32_t)p2) & 0xFFFFu) * 0x10001u;
#pragma unroll
        for (int i = 0; i < KW; ++i) {
            const uint32_t c1 = __vadd2(nb[i], p1x2);
            const uint32_t c2 = __vadd2(nb[i + 1], p1x2);
            const uint32_t m = __vminu2(__vminu2(Lp[i], c1), __vminu2(c2, mp2));
            uint32_t l = __vsub2(__vadd2(Cw[i], m), mpx2);
            if (!FULL) l |= mk.padMask[i];
            Ln[i] = l;
        }
    }
}

// ---- per-lane loads/stores of KW words (cost: 2 bytes per word; agg: 4) ----

// Cost bytes of the lane's 2*KW disparities -> KW packed uint16x2 words.
template <int KW>
__device__ __forceinline__ void load_cost_words(const uint8_t* p, uint32_t (&w)[KW]) {
    if (KW == 1) {
        const uint32_t v = *reinterpret_cast<const uint16_t*>(p);
        w[0] = bytes_lo(v);
    } else if (KW == 2) {
        const uint32_t v = *reinterpret_cast<const uint32_t*>(p);
        w[0] = bytes_lo(v);
        w[1 % KW] = bytes_hi(v);
    } else if (KW % 4 == 0) {
#pragma unroll
        for (int q = 0; q < KW / 4; ++q) {
            const uint2 v = reinterpret_cast<const uint2*>(p)[q];
            w[(4 * q + 0) % KW] = bytes_lo(v.x);
            w[(4 * q + 1) % KW] = bytes_hi(v.x);
            w[(4 * q + 2) % KW] = bytes_lo(v.y);
            w[(4 * q + 3) % KW] = bytes_hi(v.y);
        }
    } else if (KW % 2 == 0) {
#pragma unroll
        for (int q = 0; q < KW / 2; ++q) {
            const uint32_t v = reinterpret_cast<const uint32_t*>(p)[q];
            w[(2 * q) % KW] = bytes_lo(v);
            w[(2 * q + 1) % KW] = bytes_hi(v);
        }
    } else {
#pragma unroll
        for (int i = 0; i < KW; ++i) w[i] = bytes_lo(reinterpret_cast<const uint16_t*>(p)[i]);
    }
}

template <int KW>
__device__ __forceinline__ void load_words(const uint16_t* p, uint32_t (&w)[KW]) {
    if (KW % 4 == 0) {
#pragma unroll
        for (int q = 0; q < KW / 4; ++q) {
            const uint4 v = reinterpret_cast<const uint4*>(p)[q];
            w[(4 * q + 0) % KW] = v.x; w[(4 * q + 1) % KW] = v.y;
            w[(4 * q + 2) % KW] = v.z; w[(4 * q + 3) % KW] = v.w;
        }
    } else if (KW % 2 == 0) {
#pragma unroll
        for (int q = 0; q < KW / 2; ++q) {
            const uint2 v = reinterpret_cast<const uint2*>(p)[q];
            w[(2 * q) % KW] = v.x; w[(2 * q + 1) % KW] = v.y;
        }
    } else {
#pragma unroll
        for (int i = 0; i < KW; ++i) w[i] = reinterpret_cast<const uint32_t*>(p)[i];
    }
}

template <int KW>
__device__ __forceinline__ void store_words(uint16_t* p, const uint32_t (&w)[KW]) {
    if (KW % 4 == 0) {
#pragma unroll
        for (int q = 0; q < KW / 4; ++q)
            reinterpret_cast<uint4*>(p)[q] = make_uint4(w[(4 * q) % KW], w[(4 * q + 1) % KW],
                                                        w[(4 * q + 2) % KW], w[(4 * q + 3) % KW]);
    } else if (KW % 2 == 0) {
#pragma unroll
        for (int q = 0; q < KW / 2; ++q)
            reinterpret_cast<uint2*>(p)[q] = make_uint2(w[(2 * q) % KW], w[(2 * q + 1) % KW]);
    } else {
#pragma unroll
        for (int i = 0; i < KW; ++i) reinterpret_cast<uint32_t*>(p)[i] = w[i];
    }
}

}  // namespace lumen
