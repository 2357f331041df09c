/* bg_expfn.h -- functions of generated synaptic code that must give the
 * same bits on the GPU and in the CPU restatement: the same IEEE operations
 * in the same order (no contraction on either side: -fmad=false,
 * -ffp-contract=off), so the results agree exactly.
 *
 * bg_exp: exp(x) by the classic reduction x = k ln2 + r, |r| <= ln2/2 (ln2
 * split into a 32-bit head, so k*ln2_hi is exact, and a tail), the Taylor
 * series of exp(r) to degree 13 (truncation error below 2^-60) in Horner
 * form, and an exact scaling by 2^k.  Within one ulp of exp.
 * bg_clip: numpy.clip(x, lo, hi) for scalars (NaN stays NaN). */
#ifndef BG_EXPFN_H
#define BG_EXPFN_H

#if defined(__CUDACC__) || defined(__CUDACC_RTC__)
#define BG_HD __host__ __device__ __forceinline__
#else
#define BG_HD static inline
#endif

BG_HD double bg_clip(double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); }

BG_HD double bg_exp(double x) {
    if (x != x) return x;
    if (x > 709.79) return x * 0x1p1023 * 0x1p1023;          /* +inf */
    if (x < -745.2) return 0.0;
    const double k = rint(x * 0x1.71547652b82fep+0);          /* x / ln2, nearest */
    const double r = (x - k * 0x1.62e42fee00000p-1) - k * 0x1.a39ef35793c76p-33;
    double p = 0x1.6124613a86d09p-33;                          /* 1/13! */
    p = p * r + 0x1.1eed8eff8d898p-29;                         /* 1/12! */
    p = p * r + 0x1.ae64567f544e4p-26;
    p = p * r + 0x1.27e4fb7789f5cp-22;
    p = p * r + 0x1.71de3a556c734p-19;
    p = p * r + 0x1.a01a01a01a01ap-16;
    p = p * r + 0x1.a01a01a01a01ap-13;
    p = p * r + 0x1.6c16c16c16c17p-10;
    p = p * r + 0x1.1111111111111p-7;
    p = p * r + 0x1.5555555555555p-5;
    p = p * r + 0x1.5555555555555p-3;
    p = p * r + 0x1p-1;
    p = p * r + 1.0;
    p = p * r + 1.0;
    return ldexp(p, (int)k);
}

#endif
