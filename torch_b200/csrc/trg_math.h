/*
 * Double-precision exp / log / log10 / pow for the FP64 form, shared by the
 * FP64 GPU kernels and the CPU oracle's portable-math twin, built only from
 * IEEE operations (+, -, *, /, and explicit fused multiply-adds through
 * fma()), so that host code compiled with -ffp-contract=off and device code
 * compiled with --fmad=false produce bit-identical results.
 *
 * Why these functions are nearly correctly rounded: the reference's
 * radiation and cooling step amplifies one-ulp differences between math
 * libraries (a thermal sub-cycle count is a ceil(), the implicit ionisation
 * solve stops on a relative-change test) until they reach the 1e-10 level
 * after a few tens of steps.  The host glibc's exp, log and pow round to
 * nearest in all but a small fraction of cases (error bounds just above half
 * an ulp), so functions that are correctly rounded except where the exact
 * value lies within ~2^-20 ulp of a rounding boundary return glibc's results
 * almost everywhere; tests/test_math.py measures the remaining differences.
 *
 * Methods (each result is formed as an unevaluated double-double sum with a
 * relative error below about 2^-75, then rounded once):
 *   exp  : x = k ln2/128 + r (|r| <= ln2/256), ln2/128 in three parts (the
 *          first with 35 bits, k * part exact), r as a double-double;
 *          exp(r) - 1 = r + r^2/2 (double-double) + r^3 (1/6 + ... + r^5/8!)
 *          (double); 2^(j/128) from a double-double table, j = k mod 128;
 *          scaled by 2^((k - j)/128), with the last rounding done on the
 *          subnormal grid when the result is below 2^-1022.
 *   log  : x = 2^e m with m in [0.75, 1.5); m in one of 96 intervals of width
 *          1/128, c ~ 1/mid of the interval; r = m c - 1 exactly as a
 *          double-double (two-product, Sterbenz subtraction; c = 1 next to
 *          m = 1); log(1 + r) = r - r^2/2 + r^3/3 (double-double) + r^4
 *          (-1/4 + r/5 - ... + r^8/12) (double); plus -log(c) (double-double
 *          table) and e ln2 (three parts, the first with 42 bits).
 *   log10: the classical reduction of fdlibm: n = exponent of x (plus one
 *          when negative), m = x 2^-n, log10(x) = n log10_2hi +
 *          (n log10_2lo + log(m) / ln 10), with log10_2hi the leading 40 bits
 *          of log10(2).
 *   pow  : exp(y log x), log as a double-double, the product y log x as a
 *          double-double argument of exp.
 * Tables and split constants: trg_math_tables.h (make_math_tables.py).
 */
#ifndef TRG_MATH_H
#define TRG_MATH_H

#include <math.h>
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define TRG_MATH_FN static __host__ __device__ __forceinline__
#else
#define TRG_MATH_FN static inline
#endif

/* host copies of the tables, and device copies (global memory, read through
   the read-only data cache) */
#define TRG_MATH_TABLE(name, n) static const double name##_h[n]
#include "trg_math_tables.h"
#undef TRG_MATH_TABLE
#if defined(__CUDACC__)
#define TRG_MATH_TABLE(name, n) static __device__ const double name##_d[n]
#include "trg_math_tables.h"
#undef TRG_MATH_TABLE
#endif
#if defined(__CUDA_ARCH__)
#define TRG_TAB(name, i) __ldg(&name##_d[i])
#else
#define TRG_TAB(name, i) (name##_h[i])
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

#define TRG_INF trg_bits_to_double(0x7ff0000000000000ULL)
#define TRG_NAN trg_bits_to_double(0x7ff8000000000000ULL)

/* Error-free transformations: a + b = s + e, a * b = p + e exactly. */
TRG_MATH_FN void trg_two_sum(double a, double b, double* s, double* e) {
	const double x = a + b, bb = x - a;
	*s = x;
	*e = (a - (x - bb)) + (b - bb);
}
TRG_MATH_FN void trg_two_prod(double a, double b, double* p, double* e) {
	const double x = a * b;
	*p = x;
	*e = fma(a, b, -x);
}

/* exp(xh + xl), |xl| at most a few ulp of xh. */
TRG_MATH_FN double trg_exp_dd(double xh, double xl) {
	if (xh != xh) return xh + xh;
	if (xh > 709.79) return TRG_INF;
	if (xh < -745.2) return 0.0;
	const double shift = 0x1.8p52;
	const double kd = (xh * TRG_EXP_INV_LN2_128 + shift) - shift; /* nearest integer */
	const int k = (int)kd;
	/* r = x - k ln2/128 as a double-double */
	const double t1 = xh - kd * TRG_EXP_LN2_128_1; /* exact: kd * part exact, Sterbenz */
	double p, pe, rh, rl;
	trg_two_prod(kd, TRG_EXP_LN2_128_2, &p, &pe);
	trg_two_sum(t1, -p, &rh, &rl);
	rl = ((rl - pe) - kd * TRG_EXP_LN2_128_3) + xl;
	trg_two_sum(rh, rl, &rh, &rl);
	/* exp(r) - 1 = a + tail */
	double s2h, s2l;
	trg_two_prod(rh, rh, &s2h, &s2l);
	s2l += 2.0 * rh * rl;
	double q = 1.0 / 40320.0;
	q = 1.0 / 5040.0 + rh * q;
	q = 1.0 / 720.0 + rh * q;
	q = 1.0 / 120.0 + rh * q;
	q = 1.0 / 24.0 + rh * q;
	q = 1.0 / 6.0 + rh * q;
	q = (s2h * rh) * q;
	double a, ea;
	trg_two_sum(rh, 0.5 * s2h, &a, &ea);
	const double tail = (ea + rl) + (0.5 * s2l + q);
	/* 2^(j/128) (1 + a + tail) */
	const int j = k & 127;
	const int ex = (k - j) / 128;
	const double th = TRG_TAB(trg_exp_tab, 2 * j), tl = TRG_TAB(trg_exp_tab, 2 * j + 1);
	double m, me, s, se;
	trg_two_prod(th, a, &m, &me);
	const double small = (me + th * tail) + (tl + tl * a);
	trg_two_sum(th, m, &s, &se);
	trg_two_sum(s, se + small, &s, &se); /* s: the result rounded, se: the rest */
	if (ex > -1022 || (ex == -1022 && s > 1.0)) {
		if (ex > 1023) return (s * 0x1p1023) * trg_pow2i(ex - 1023);
		return s * trg_pow2i(ex);
	}
	/* below 2^-1022: round once on the subnormal grid (spacing 2^-1074),
	   which is the integer grid after scaling by 2^(ex + 1074) */
	const double sc = trg_pow2i(ex + 1074);
	const double U = s * sc, L = se * sc;
	const double grid = 0x1p52; /* U + grid stays in [2^52, 2^53]: integer spacing */
	double z, ze;
	trg_two_sum(U, grid, &z, &ze);
	z = z + (ze + L);
	return (z - grid) * 0x1p-1074;
}

TRG_MATH_FN double trg_exp(double x) { return trg_exp_dd(x, 0.0); }

/* log(x) as a double-double hi + lo (hi the rounded result), x > 0 finite. */
TRG_MATH_FN void trg_log_dd(double x, double* hi, double* lo) {
	int e = 0;
	if (x < 0x1p-1022) { /* subnormal: scale into the normal range */
		x *= 0x1p54;
		e = -54;
	}
	const uint64_t u = trg_double_to_bits(x);
	e += (int)((u >> 52) & 0x7ff) - 1023;
	double m = trg_bits_to_double((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL); /* [1, 2) */
	if (m >= 1.5) {
		m *= 0.5;
		e += 1;
	}
	const int i = (int)((m - 0.75) * 128.0); /* exact: Sterbenz, power of two */
	const double c = TRG_TAB(trg_log_tab, 3 * i), th = TRG_TAB(trg_log_tab, 3 * i + 1),
	             tl = TRG_TAB(trg_log_tab, 3 * i + 2);
	double rh, rl;
	if (c == 1.0) {
		rh = m - 1.0; /* exact */
		rl = 0.0;
	} else {
		double ph, pl;
		trg_two_prod(m, c, &ph, &pl);
		trg_two_sum(ph - 1.0, pl, &rh, &rl); /* ph - 1 exact: ph within 2^-7 of 1 */
	}
	/* log(1 + r) = b + tail */
	double s2h, s2l, s3h, s3l, t3h, t3l;
	trg_two_prod(rh, rh, &s2h, &s2l);
	s2l += 2.0 * rh * rl;
	trg_two_prod(s2h, rh, &s3h, &s3l);
	s3l += s2l * rh + s2h * rl;
	trg_two_prod(s3h, TRG_LOG_THIRD_HI, &t3h, &t3l);
	t3l += s3l * TRG_LOG_THIRD_HI + s3h * TRG_LOG_THIRD_LO;
	double q = -1.0 / 12.0;
	q = 1.0 / 11.0 + rh * q;
	q = -1.0 / 10.0 + rh * q;
	q = 1.0 / 9.0 + rh * q;
	q = -1.0 / 8.0 + rh * q;
	q = 1.0 / 7.0 + rh * q;
	q = -1.0 / 6.0 + rh * q;
	q = 1.0 / 5.0 + rh * q;
	q = -1.0 / 4.0 + rh * q;
	q = (s2h * s2h) * q;
	double a, ea, b, eb;
	trg_two_sum(rh, -0.5 * s2h, &a, &ea);
	trg_two_sum(a, t3h, &b, &eb);
	const double tail = ((ea + eb) + (rl - 0.5 * s2l)) + (t3l + q);
	/* e ln2 - log(c) + log(1 + r) */
	const double ed = (double)e;
	double u1, eu1, u2, eu2;
	trg_two_sum(ed * TRG_LOG_LN2_1, th, &u1, &eu1); /* ed * part exact */
	trg_two_sum(u1, b, &u2, &eu2);
	const double rest = (eu1 + eu2) + ((ed * TRG_LOG_LN2_2 + tl) + (tail + ed * TRG_LOG_LN2_3));
	trg_two_sum(u2, rest, hi, lo);
}

TRG_MATH_FN double trg_log(double x) {
	if (x != x) return x;
	if (x < 0) return TRG_NAN;
	if (x == 0) return -TRG_INF;
	if (x == TRG_INF) return x;
	double hi, lo;
	trg_log_dd(x, &hi, &lo);
	return hi;
}

TRG_MATH_FN double trg_log10(double x) {
	if (x != x) return x;
	if (x < 0) return TRG_NAN;
	if (x == 0) return -TRG_INF;
	if (x == TRG_INF) return x;
	int k = 0;
	if (x < 0x1p-1022) {
		x *= 0x1p54;
		k = -54;
	}
	const uint64_t u = trg_double_to_bits(x);
	k += (int)((u >> 52) & 0x7ff) - 1023;
	const int neg = k < 0;
	/* mantissa in [1, 2), or in [0.5, 1) for x < 1 */
	const double m = trg_bits_to_double((u & 0x000fffffffffffffULL) | ((uint64_t)(0x3ff - neg) << 52));
	const double n = (double)(k + neg);
	const double z = n * TRG_LOG10_2LO + TRG_LOG10_IVLN10 * trg_log(m);
	return z + n * TRG_LOG10_2HI;
}

TRG_MATH_FN double trg_pow(double x, double y) {
	if (y == 0) return 1.0;
	if (x == 1.0) return 1.0;
	if (x != x || y != y) return x + y;
	double sign = 1.0;
	if (x < 0) { /* defined for integer y only */
		const double ay = y < 0 ? -y : y;
		if (ay < 0x1p62) {
			const int64_t iy = (int64_t)y;
			if ((double)iy != y) return TRG_NAN;
			if (iy & 1) sign = -1.0;
		}
		x = -x;
	}
	if (x == 0) return y > 0 ? 0.0 * sign : sign * TRG_INF;
	if (y == TRG_INF || y == -TRG_INF) {
		if (x == 1.0) return 1.0;
		return (x < 1.0) == (y > 0) ? 0.0 : TRG_INF;
	}
	if (x == TRG_INF) return y > 0 ? sign * TRG_INF : 0.0 * sign;
	double lh, ll, zh, zl;
	trg_log_dd(x, &lh, &ll);
	trg_two_prod(y, lh, &zh, &zl);
	zl += y * ll;
	return sign * trg_exp_dd(zh, zl);
}

#endif /* TRG_MATH_H */
