// swb_device.cuh -- device helpers shared by the SW kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "swb_internal.h"

namespace swb {

// One base of a task span (see the SWB_* flags in swb_cuda.h).  `pac` is
// the resident forward strand in .pac layout: base p lives in byte p>>2,
// bits (3-(p&3))*2 (PackedReference.swift:34-38).
__device__ __forceinline__ uint32_t span_base(const uint8_t *__restrict__ bases,
                                              const uint8_t *__restrict__ pac, uint64_t off,
                                              int k, int len, uint32_t flags, bool is_target) {
    const bool rev = is_target ? (flags & SWB_T_REVERSE) : (flags & SWB_Q_REVERSE);
    const uint64_t idx = off + (uint64_t)(rev ? (len - 1 - k) : k);
    uint32_t b;
    if (is_target && (flags & SWB_T_FROM_REF)) {
        b = (pac[idx >> 2] >> ((3 - (uint32_t)(idx & 3)) << 1)) & 3u;
    } else {
        b = bases[idx];
    }
    if (is_target && (flags & SWB_T_COMPLEMENT) && b < 4u) b = 3u - b;   // N stays N
    return b;
}

// Score table of one target base t as 8 signed bytes (query codes 0-4):
// a on the diagonal, -b off it, -1 in the N row/column
// (ScoringParameters.swift:65-73).  lo holds codes 0-3, hi code 4.
struct RowTable {
    uint32_t lo, hi;
};

__device__ __forceinline__ RowTable row_table(const DevScoring &sc, uint32_t t) {
    const uint32_t A = (uint32_t)(uint8_t)(int8_t)sc.a;
    const uint32_t B = (uint32_t)(uint8_t)(int8_t)(-sc.b);
    const uint32_t N = 0xFFu;
    RowTable r;
    if (t >= 4) {
        r.lo = 0xFFFFFFFFu;
    } else {
        r.lo = (B * 0x01010101u);
        r.lo = (r.lo & ~(0xFFu << (8 * t))) | (A << (8 * t));
    }
    r.hi = N;
    return r;
}

// prmt.b32 in its default mode: each selector nibble picks one of the 8
// input bytes (low 3 bits) and, when its msb is set, replicates that
// byte's sign bit instead of copying it.
__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
    uint32_t d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
    return d;
}

// Signed score of query code q (0-4) against the row's target base: one
// byte permute, sign-extended from byte q.
__device__ __forceinline__ int row_score(const RowTable &r, uint32_t q) {
    return (int)prmt(r.lo, r.hi, q * 0x1111u + 0x8880u);
}

// Saturating-free helpers.
__host__ __device__ __forceinline__ int imax(int a, int b) { return a > b ? a : b; }
__host__ __device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }

}  // namespace swb
