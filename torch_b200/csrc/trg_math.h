/*
 * Portable double-precision exp / log / log10 / pow built only from IEEE
 * +, -, *, / (no fused multiply-add), so that host code compiled with
 * -ffp-contract=off and device code compiled with --fmad=false produce
 * bit-identical results.
 *
 * Why: the reference's radiation and cooling step amplifies one-ulp
 * differences between two math libraries (a thermal sub-cycle count is a
 * ceil(), the implicit ionisation solve stops on a relative-change test) until
 * they reach the 1e-10 level after a few tens of steps.  The FP64 GPU kernels
 * and the CPU oracle therefore share this one implementation, which turns
 * "GPU versus CPU" into a bit-for-bit comparison of the step algorithm.
 *
 * Methods (textbook):
 *   exp  : x = k ln2 + r with a two-part ln2 (Cody & Waite), |r| <= ln2/2,
 *          exp(r) by its Taylor series to r^14/14! (truncation < 2e-17),
 *          then an exact scaling by 2^k.
 *   log  : x = m 2^e with m in [sqrt(1/2), sqrt(2)), f = (m-1)/(m+1),
 *          log m = 2 atanh f = 2 (f + f^3/3 + ... + f^23/23) (|f| <= 0.1716,
 *          truncation < 1e-19), log x = e ln2_hi + (log m + e ln2_lo).
 *   log10: log(x) / ln 10.
 *   pow  : exp(y log x) for x > 0 (relative error grows with |y log x|,
 *          about 1e-14 for the arguments of the cooling functions).
 * The split constants are ln 2 and 1/ln 2, sqrt(1/2), 1/ln 10 rounded to
 * double, with LN2_HI = ln 2 with its low 21 significand bits cleared (so that
 * k * LN2_HI is exact for |k| < 2^21) and LN2_LO = ln 2 - LN2_HI.
 * Accuracy is a few ulp for exp/log/log10, checked in tests/test_math.py
 * against the host libm.
 */
#ifndef TRG_MATH_H
#define TRG_MATH_H

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define TRG_MATH_FN static __host__ __device__ __forceinline__
#else
#define TRG_MATH_FN static inline
#endif

TRG_MATH_FN double trg_bits_to_double(uint64_t u) {
	double d;
	memcpy(&d, &u, sizeof(d));
	return d;
}
TRG_MATH_FN uint64_t trg_double_to_bits(double d) {
	uint64_t u;
	memcpy(&u, &d, sizeof(u));
	return u;
}

/* 2^k for -1022 <= k <= 1023, exact. */
TRG_MATH_FN double trg_pow2i(int k) { return trg_bits_to_double((uint64_t)(k + 1023) << 52); }

TRG_MATH_FN double trg_exp(double x) {
	const double LN2_HI = 6.93147180369123816490e-01; /* ln 2 rounded to 33 bits (k * LN2_HI exact) */
	const double LN2_LO = 1.90821492927058770002e-10; /* ln 2 - LN2_HI */
	const double INV_LN2 = 1.44269504088896338700e+00;
	if (x != x) return x;
	if (x > 709.782712893384) return trg_bits_to_double(0x7ff0000000000000ULL);
	if (x < -745.2) return 0.0;
	double kd = x * INV_LN2;
	kd = kd >= 0 ? (double)(int64_t)(kd + 0.5) : -(double)(int64_t)(-kd + 0.5);
	int k = (int)kd;
	double r = (x - kd * LN2_HI) - kd * LN2_LO;
	/* Taylor series of exp(r) - 1 in Horner form, highest term first */
	double p = 1.0 / 87178291200.0;               /* 1/14! */
	p = 1.0 / 6227020800.0 + r * p;               /* 1/13! */
	p = 1.0 / 479001600.0 + r * p;                /* 1/12! */
	p = 1.0 / 39916800.0 + r * p;                 /* 1/11! */
	p = 1.0 / 3628800.0 + r * p;                  /* 1/10! */
	p = 1.0 / 362880.0 + r * p;                   /* 1/9!  */
	p = 1.0 / 40320.0 + r * p;                    /* 1/8!  */
	p = 1.0 / 5040.0 + r * p;                     /* 1/7!  */
	p = 1.0 / 720.0 + r * p;                      /* 1/6!  */
	p = 1.0 / 120.0 + r * p;                      /* 1/5!  */
	p = 1.0 / 24.0 + r * p;                       /* 1/4!  */
	p = 1.0 / 6.0 + r * p;                        /* 1/3!  */
	p = 0.5 + r * p;                              /* 1/2!  */
	p = r + (r * r) * p;                          /* exp(r) - 1 */
	double e = 1.0 + p;
	if (k > 1023) return e * trg_pow2i(1023) * trg_pow2i(k - 1023);
	if (k < -1022) return (e * trg_pow2i(k + 1000)) * trg_pow2i(-1000);
	return e * trg_pow2i(k);
}

TRG_MATH_FN double trg_log(double x) {
	const double LN2_HI = 6.93147180369123816490e-01;
	const double LN2_LO = 1.90821492927058770002e-10;
	const double SQRT_HALF = 0.70710678118654752440;
	if (x != x) return x;
	if (x < 0) return trg_bits_to_double(0x7ff8000000000000ULL);
	if (x == 0) return -trg_bits_to_double(0x7ff0000000000000ULL);
	if (x == trg_bits_to_double(0x7ff0000000000000ULL)) return x;
	int e = 0;
	if (x < 2.2250738585072014e-308) { /* subnormal: scale into the normal range */
		x *= trg_pow2i(54);
		e = -54;
	}
	uint64_t u = trg_double_to_bits(x);
	e += (int)((u >> 52) & 0x7ff) - 1023;
	double m = trg_bits_to_double((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL); /* [1, 2) */
	if (m > 2.0 * SQRT_HALF) {
		m = m * 0.5;
		e += 1;
	}
	double f = (m - 1.0) / (m + 1.0);
	double f2 = f * f;
	double s = 1.0 / 23.0;
	s = 1.0 / 21.0 + f2 * s;
	s = 1.0 / 19.0 + f2 * s;
	s = 1.0 / 17.0 + f2 * s;
	s = 1.0 / 15.0 + f2 * s;
	s = 1.0 / 13.0 + f2 * s;
	s = 1.0 / 11.0 + f2 * s;
	s = 1.0 / 9.0 + f2 * s;
	s = 1.0 / 7.0 + f2 * s;
	s = 1.0 / 5.0 + f2 * s;
	s = 1.0 / 3.0 + f2 * s;
	double logm = 2.0 * f + (2.0 * f) * (f2 * s);
	double ed = (double)e;
	return ed * LN2_HI + (logm + ed * LN2_LO);
}

TRG_MATH_FN double trg_log10(double x) { return trg_log(x) * 0.43429448190325182765; }

TRG_MATH_FN double trg_pow(double x, double y) {
	if (y == 0) return 1.0;
	if (x == 1.0) return 1.0;
	if (x != x || y != y) return x + y;
	if (x == 0) return y > 0 ? 0.0 : trg_bits_to_double(0x7ff0000000000000ULL);
	if (x < 0) return trg_bits_to_double(0x7ff8000000000000ULL);
	return trg_exp(y * trg_log(x));
}

#endif /* TRG_MATH_H */
