// Epilogue building blocks shared by the exact-search kernels: per-thread
// running top-2 of one query row and the pruned scan of 32 accumulator
// columns (see exact2nn.cu for the pruning argument).
#pragma once
#include <climits>
#include <cstdint>

namespace sift {
namespace {

__device__ __forceinline__ int max8(const uint32_t* v) {
    int m = __vimax3_s32(static_cast<int>(v[0]), static_cast<int>(v[1]), static_cast<int>(v[2]));
    m = __vimax3_s32(m, static_cast<int>(v[3]), static_cast<int>(v[4]));
    m = __vimax3_s32(m, static_cast<int>(v[5]), static_cast<int>(v[6]));
    return max(m, static_cast<int>(v[7]));
}

// An f32 accumulator holding an integer multiple of 1/dscale (dscale a power
// of two; exact, see the FP16 kernel) -> the integer dot product.
__device__ __forceinline__ int f32_dot(uint32_t bits, float dscale) {
    return __float2int_rn(__uint_as_float(bits) * dscale);
}

// Per-thread running top-2 of one query row over base rows visited in
// increasing index order (strict '<' keeps the lower index on ties).
struct Top2 {
    int k1, i1, k2, i2;
    int thr;  // prune bound: rows with key > thr cannot enter the final top-2
};

__device__ __forceinline__ void top2_update(Top2& s, int key, int idx) {
    if (key < s.k2) {
        if (key < s.k1) {
            s.k2 = s.k1; s.i2 = s.i1;
            s.k1 = key; s.i1 = idx;
        } else {
            s.k2 = key; s.i2 = idx;
        }
        s.thr = min(s.thr, s.k2 - 1);
    }
}

// One group of 32 consecutive base rows [row0, row0 + 32) for this thread's
// query row; v[c] = q.b(row0 + c) as s32, or (F32) as the f32 accumulator of
// the FP16 kernel, q.b / dscale. Those are never negative (inputs are
// integers in [0, 255] times 2^-s), so their bit patterns, compared as int32,
// order like the values (-0.0 only below +0.0, and both convert to 0): the
// max trees run on the raw bits, and only the four subgroup maxima and the
// values of passing subgroups are converted. nrm points at the group's 32 norms in the
// shared-memory record, gm8 at its four 8-row minima. Each 8-row subgroup is
// bounded from below by gm8[k] - 2 max(v[8k..8k+8)) (no key of its rows is
// smaller), so a subgroup whose bound exceeds the thread's threshold holds no
// candidate; the four bounds are tested with one vote. A passing subgroup
// forms its 8 exact keys and updates the top-2 only when their minimum is
// within the threshold (a key above it cannot reach the final top-2: the
// threshold never exceeds the final second-best key).
template <bool F32 = false>
__device__ __forceinline__ void scan_group(const uint32_t (&v)[32], int row0, const int32_t* nrm, const int32_t* gm8,
                                           Top2& s, float dscale = 1.0f) {
    int mx[4];
    #pragma unroll
    for (int k = 0; k < 4; ++k) {
        mx[k] = max8(v + 8 * k);
        if constexpr (F32) mx[k] = f32_dot(static_cast<uint32_t>(mx[k]), dscale);
    }
    const int4 g8 = *reinterpret_cast<const int4*>(gm8);
    const int bnd[4] = {g8.x - 2 * mx[0], g8.y - 2 * mx[1], g8.z - 2 * mx[2], g8.w - 2 * mx[3]};
    const int bmin = min(__vimin3_s32(bnd[0], bnd[1], bnd[2]), bnd[3]);
    if (__any_sync(0xffffffffu, bmin <= s.thr)) {
        #pragma unroll
        for (int k = 0; k < 4; ++k) {
            const bool ps = bnd[k] <= s.thr;
            if (__any_sync(0xffffffffu, ps)) {
                if (ps) {
                    const int4 na = *reinterpret_cast<const int4*>(nrm + 8 * k);
                    const int4 nb = *reinterpret_cast<const int4*>(nrm + 8 * k + 4);
                    const int nr[8] = {na.x, na.y, na.z, na.w, nb.x, nb.y, nb.z, nb.w};
                    int key[8];
                    #pragma unroll
                    for (int e = 0; e < 8; ++e)
                        key[e] = nr[e] - 2 * (F32 ? f32_dot(v[8 * k + e], dscale) : static_cast<int>(v[8 * k + e]));
                    // Exact keys first; the (rare) updates only when one can enter.
                    int mk = __vimin3_s32(key[0], key[1], key[2]);
                    mk = __vimin3_s32(mk, key[3], key[4]);
                    mk = __vimin3_s32(mk, key[5], key[6]);
                    mk = min(mk, key[7]);
                    if (mk <= s.thr) {
                        const int base = row0 + 8 * k;
                        #pragma unroll
                        for (int e = 0; e < 8; ++e) top2_update(s, key[e], base + e);
                    }
                }
            }
        }
    }
}

// Accumulator kinds of scan16 / bound16 / exact8.
enum AccKind : int {
    kAccS32 = 0,    // s32 dot products (u8 kernel)
    kAccF32Int = 1, // f32 accumulators holding integer dot products / dscale (FP16 kernel)
    kAccFloat = 2,  // f32 dot products of general floats (float keys, float norms)
};

// The pruned scan of 16 consecutive base rows [row0, row0 + 16) in one pass:
// the two 8-row subgroups of scan_group (same bounds, same keys), a warp vote
// per chunk, exact keys formed at once from the registers (the form for
// batches of small problems, whose bounds pass often).
// nrm: the 16 norms, gm8: the two 8-row minima (8-byte aligned).
template <int KIND>
__device__ __forceinline__ void scan16(const uint32_t (&v)[16], int row0, const int32_t* nrm, const int32_t* gm8,
                                       Top2& s, float dscale) {
    const int2 g8 = *reinterpret_cast<const int2*>(gm8);
    int bnd[2];
    #pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int g = k ? g8.y : g8.x;
        if constexpr (KIND == kAccFloat) {
            float m = __uint_as_float(v[8 * k]);
            #pragma unroll
            for (int e = 1; e < 8; ++e) m = fmaxf(m, __uint_as_float(v[8 * k + e]));
            bnd[k] = float_key(fmaf(-2.0f, m, __int_as_float(g)));
        } else {
            int m = max8(v + 8 * k);
            if constexpr (KIND == kAccF32Int) m = f32_dot(static_cast<uint32_t>(m), dscale);
            bnd[k] = g - 2 * m;
        }
    }
    if (__any_sync(0xffffffffu, min(bnd[0], bnd[1]) <= s.thr)) {
        #pragma unroll
        for (int k = 0; k < 2; ++k) {
            const bool ps = bnd[k] <= s.thr;
            if (__any_sync(0xffffffffu, ps)) {
                if (ps) {
                    const int4 na = *reinterpret_cast<const int4*>(nrm + 8 * k);
                    const int4 nb = *reinterpret_cast<const int4*>(nrm + 8 * k + 4);
                    const int nr[8] = {na.x, na.y, na.z, na.w, nb.x, nb.y, nb.z, nb.w};
                    int key[8];
                    #pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        if constexpr (KIND == kAccFloat)
                            key[e] = float_key(fmaf(-2.0f, __uint_as_float(v[8 * k + e]), __int_as_float(nr[e])));
                        else if constexpr (KIND == kAccF32Int)
                            key[e] = nr[e] - 2 * f32_dot(v[8 * k + e], dscale);
                        else
                            key[e] = nr[e] - 2 * static_cast<int>(v[8 * k + e]);
                    }
                    int mk = __vimin3_s32(key[0], key[1], key[2]);
                    mk = __vimin3_s32(mk, key[3], key[4]);
                    mk = __vimin3_s32(mk, key[5], key[6]);
                    mk = min(mk, key[7]);
                    if (mk <= s.thr) {
                        const int base = row0 + 8 * k;
                        #pragma unroll
                        for (int e = 0; e < 8; ++e) top2_update(s, key[e], base + e);
                    }
                }
            }
        }
    }
}

// The pruned scan of a TMEM slot in two passes, so that an epilogue can bound
// every 8-row subgroup with no vote and no branch and form exact keys only
// where a bound passes.
//
// bound16: the pass bits of the chunk's two 8-row subgroups (bit k set when
// subgroup k's lower bound, the 8-row minimum gm8[k] minus twice the largest
// q.b of its rows, is within thr; the same bound as scan_group). gm8: the two
// 8-row minima (8-byte aligned).
template <int KIND>
__device__ __forceinline__ uint32_t bound16(const uint32_t (&v)[16], const int32_t* gm8, int thr, float dscale) {
    const int2 g8 = *reinterpret_cast<const int2*>(gm8);
    uint32_t bits = 0;
    #pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int g = k ? g8.y : g8.x;
        int bnd;
        if constexpr (KIND == kAccFloat) {
            float m = __uint_as_float(v[8 * k]);
            #pragma unroll
            for (int e = 1; e < 8; ++e) m = fmaxf(m, __uint_as_float(v[8 * k + e]));
            bnd = float_key(fmaf(-2.0f, m, __int_as_float(g)));
        } else {
            int m = max8(v + 8 * k);
            if constexpr (KIND == kAccF32Int) m = f32_dot(static_cast<uint32_t>(m), dscale);
            bnd = g - 2 * m;
        }
        bits |= (bnd <= thr ? 1u : 0u) << k;
    }
    return bits;
}

// fold_bits16: the pass bits of a chunk's two 8-row subgroups in the fold
// variant, whose accumulators hold q.b - c and whose keys are r - 2 acc with
// residuals r >= -1: subgroup k may hold a key within thr only when its
// largest accumulator reaches vt = -floor((thr + 1) / 2).
__device__ __forceinline__ uint32_t fold_bits16(const uint32_t (&v)[16], int vt) {
    return (max8(v) >= vt ? 1u : 0u) | (max8(v + 8) >= vt ? 2u : 0u);
}

// exact8: the exact keys of one 8-row subgroup [row0, row0 + 8) (v: its
// accumulators, nrm: its 8 norms, 16-byte aligned); they update the running
// top-2 only when their minimum is within the thread's current threshold (a
// key above it cannot reach the final top-2).
template <int KIND>
__device__ __forceinline__ void exact8(const uint32_t (&v)[8], int row0, const int32_t* nrm, Top2& s,
                                       float dscale) {
    const int4 na = *reinterpret_cast<const int4*>(nrm);
    const int4 nb = *reinterpret_cast<const int4*>(nrm + 4);
    const int nr[8] = {na.x, na.y, na.z, na.w, nb.x, nb.y, nb.z, nb.w};
    int key[8];
    #pragma unroll
    for (int e = 0; e < 8; ++e) {
        if constexpr (KIND == kAccFloat)
            key[e] = float_key(fmaf(-2.0f, __uint_as_float(v[e]), __int_as_float(nr[e])));
        else if constexpr (KIND == kAccF32Int)
            key[e] = nr[e] - 2 * f32_dot(v[e], dscale);
        else
            key[e] = nr[e] - 2 * static_cast<int>(v[e]);
    }
    int mk = __vimin3_s32(key[0], key[1], key[2]);
    mk = __vimin3_s32(mk, key[3], key[4]);
    mk = __vimin3_s32(mk, key[5], key[6]);
    mk = min(mk, key[7]);
    if (mk <= s.thr) {
        #pragma unroll
        for (int e = 0; e < 8; ++e) top2_update(s, key[e], row0 + e);
    }
}

}  // namespace
}  // namespace sift
