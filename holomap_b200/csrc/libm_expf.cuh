// libm_expf.cuh -- device port of the libm crate's expf (libm 0.2.16, the
// FreeBSD msun e_expf method) used by smooth-kNN (src/fmath.rs:119-122 via
// src/smooth_knn.rs:46) and the fuzzy graph (src/fuzzy.rs:44): the same
// constants and the same sequence of binary32 operations as the oracle's
// restatement, each rounded to nearest.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hm {

__device__ __forceinline__ float scalbnf_dev(float y, int n) {
    if (n > 127) {
        y = __fmul_rn(y, __uint_as_float(0x7f000000u));
        n -= 127;
        if (n > 127) {
            y = __fmul_rn(y, __uint_as_float(0x7f000000u));
            n -= 127;
            if (n > 127) n = 127;
        }
    } else if (n < -126) {
        y = __fmul_rn(y, __uint_as_float(0x0c800000u));  // 2^-102
        n += 102;
        if (n < -126) {
            y = __fmul_rn(y, __uint_as_float(0x0c800000u));
            n += 102;
            if (n < -126) n = -126;
        }
    }
    return __fmul_rn(y, __uint_as_float((uint32_t)(0x7f + n) << 23));
}

__device__ __forceinline__ float expf_libm(float x) {
    const float ln2_hi = __uint_as_float(0x3f317200u);
    const float ln2_lo = __uint_as_float(0x35bfbe8eu);
    const float inv_ln2 = __uint_as_float(0x3fb8aa3bu);
    const float p1 = __uint_as_float(0x3e2aaa8fu);
    const float p2 = __uint_as_float(0xbb355215u);

    const uint32_t bits = __float_as_uint(x);
    const bool neg = (bits >> 31) != 0;
    const uint32_t mag = bits & 0x7fffffffu;

    if (mag >= 0x42aeac50u) {
        if (mag > 0x7f800000u) return x;
        if (!neg && mag >= 0x42b17218u) return __fmul_rn(x, __uint_as_float(0x7f000000u));
        if (neg && mag >= 0x42cff1b5u) return 0.0f;
    }
    float hi, lo, r;
    int k;
    if (mag > 0x3eb17218u) {
        if (mag > 0x3f851592u) {
            float t = __fmul_rn(inv_ln2, x);
            t = __fadd_rn(t, neg ? -0.5f : 0.5f);
            k = __float2int_rz(t);
        } else {
            k = neg ? -1 : 1;
        }
        const float kf = __int2float_rn(k);
        hi = __fsub_rn(x, __fmul_rn(kf, ln2_hi));
        lo = __fmul_rn(kf, ln2_lo);
        r = __fsub_rn(hi, lo);
    } else if (mag > 0x39000000u) {
        k = 0;
        hi = x;
        lo = 0.0f;
        r = x;
    } else {
        return __fadd_rn(1.0f, x);
    }
    const float rr = __fmul_rn(r, r);
    float poly = __fmul_rn(rr, p2);
    poly = __fadd_rn(p1, poly);
    poly = __fmul_rn(rr, poly);
    const float c = __fsub_rn(r, poly);
    const float num = __fmul_rn(r, c);
    const float den = __fsub_rn(2.0f, c);
    float q = __fdiv_rn(num, den);
    q = __fsub_rn(q, lo);
    q = __fadd_rn(q, hi);
    const float y = __fadd_rn(1.0f, q);
    return k == 0 ? y : scalbnf_dev(y, k);
}

}  // namespace hm
