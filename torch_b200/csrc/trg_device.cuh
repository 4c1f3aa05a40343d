// Device-side types and FP64 physics shared by the kernels of torch_b200.
//
// Every routine restates a reference TORCH routine (cited beside it) with the
// same operation order; the translation units that include this header are
// compiled with --fmad=false so that each a*b+c rounds twice, as on the
// reference's x86-64 build.  Transcendentals come from trg_math.h.
#pragma once

#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "trg_math.h"
#include "trg_types.h"
#include "../../include/torch_b200.h"

// Transcendentals of the radiation and cooling kernels.  The exact build
// (FP64 form) uses the correctly rounded functions of trg_math.h, shared with
// the CPU oracle; the fast build (FP32 form, compiled with TRG_FAST_MATH and FMA
// contraction) uses CUDA's double-precision library.
#ifdef TRG_FAST_MATH
#define d_exp(x) exp(x)
#define d_log(x) log(x)
#define d_log10(x) log10(x)
#define d_pow(x, y) pow(x, y)
#else
#define d_exp(x) trg_exp(x)
#define d_log(x) trg_log(x)
#define d_log10(x) trg_log10(x)
#define d_pow(x, y) trg_pow(x, y)
#endif

namespace trg {

#define FLD(a, f, i) ((a)[(long long)(f) * P.N + (i)])
// radiation and thermodynamics fields (layouts in trg_types.h)
#define RFLD(a, f, i) ((a)[r_index(P.N, (f), (i))])
#define TFLD(a, f, i) ((a)[t_index(P.N, (f), (i))])

__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }

__device__ __forceinline__ void cell_ijk(const Params& P, long long id, int* ijk) {
	if (P.N <= 0x7fffffffLL) {  // 32-bit division: a fraction of the cost of the 64-bit one
		unsigned u = (unsigned)id, nx = (unsigned)P.nx, ny = (unsigned)P.ny;
		unsigned q = u / nx;
		ijk[0] = (int)(u - q * nx);
		unsigned r = q / ny;
		ijk[1] = (int)(q - r * ny);
		ijk[2] = (int)r;
		return;
	}
	ijk[0] = (int)(id % P.nx);
	ijk[1] = (int)((id / P.nx) % P.ny);
	ijk[2] = (int)(id / ((long long)P.nx * P.ny));
}
__device__ __forceinline__ long long flat_id(const Params& P, int i, int j, int k) {
	return i + (long long)P.nx * (j + (long long)P.ny * k);
}
// Grid::buildCells (Grid.cpp:525-548): centre at index + 0.5 for dims < nd, 0 beyond.
__device__ __forceinline__ void cell_xc(const Params& P, const int* ijk, double* xc) {
	for (int i = 0; i < 3; ++i) xc[i] = (double)ijk[i];
	xc[0] += (double)P.x0;  // a slab's cells at their global x
	#pragma unroll
	for (int i = 0; i < 3; ++i) if (i < P.nd) xc[i] += 0.5;
}
__device__ __forceinline__ int ncell(const Params& P, int d) { return d == 0 ? P.nx : (d == 1 ? P.ny : P.nz); }

// Grid::computeCellVolume, Grid.cpp:876-905.
__device__ __forceinline__ double cell_volume(const Params& P, double rc) {
	const double PI = 3.14159265359;
	double volume = 0, r1, r2;
	if (P.geometry == G_CART) {
		volume = 1.0;
		#pragma unroll
		for (int i = 0; i < 3; ++i) if (i < P.nd) volume *= P.dx[i];
	} else if (P.geometry == G_CYL) {
		r2 = rc * P.dx[0] + 0.5 * P.dx[0];
		r1 = rc * P.dx[0] - 0.5 * P.dx[0];
		volume = PI * (r2 - r1) * (r2 + r1);
		if (P.nd >= 2) volume *= P.dx[1];
	} else if (P.geometry == G_SPH) {
		r2 = rc * P.dx[0] + 0.5 * P.dx[0];
		r1 = rc * P.dx[0] - 0.5 * P.dx[0];
		volume = 4.0 * PI * (r2 - r1) * (r2 * r2 + r1 * r2 + r1 * r1) / 3.0;
	}
	return volume;
}

// Grid::computeJoinArea, Grid.cpp:846-874.
__device__ __forceinline__ double join_area(const Params& P, const double* xj, int dim) {
	const double PI = 3.14159265359;
	double area = 0, r1, r2;
	if (P.geometry == G_CART) {
		area = 1.0;
		#pragma unroll
		for (int i = 0; i < 3; ++i) if (i < P.nd)
			if (i != dim) area *= P.dx[i];
	} else if (P.geometry == G_CYL) {
		if (dim == 0) {
			r1 = xj[0] * P.dx[0];
			area = 2.0 * PI * r1;
			if (P.nd >= 2) area *= P.dx[1];
		} else if (dim == 1) {
			r1 = xj[0] * P.dx[0] - 0.5 * P.dx[0];
			r2 = xj[0] * P.dx[0] + 0.5 * P.dx[0];
			area = PI * (r2 - r1) * (r2 + r1);
		}
	} else if (P.geometry == G_SPH) {
		r1 = xj[0] * P.dx[0];
		area = 4.0 * PI * r1 * r1;
	}
	return area;
}

// Face on the left (side 0) or right (side 1) of a cell along dim; the join
// coordinate is the right-hand cell's centre minus half a cell (Grid.cpp:405-411).
__device__ __forceinline__ double face_area(const Params& P, const double* xc, int dim, int side) {
	double xj[3] = {xc[0], xc[1], xc[2]};
	xj[dim] += side ? 0.5 : -0.5;
	return join_area(P, xj, dim);
}

// Fluid::initialiseGrid wind test, Fluid.cpp:41-53.
__device__ __forceinline__ bool is_wind(const Params& P, long long id, const int* ijk, const double* xc) {
	double dist2 = 0;
	#pragma unroll
	for (int i = 0; i < 3; ++i) if (i < P.nd)
		dist2 += ((int)xc[i] - P.star_pos[i]) * (xc[i] - P.star_pos[i]);
	return dist2 <= (double)(P.wind_radius * P.wind_radius) || id == P.star_cell;
}

// ---------------------------------------------------------------- algebra
// GridCell.cpp:163-213.
__device__ __forceinline__ void UfromQ(double* u, const double* q, double gamma, int nd) {
	double ke = 0;
	u[DEN] = q[DEN];
	#pragma unroll
	for (int dim = 0; dim < 3; ++dim) if (dim < nd) {
		u[VEL + dim] = q[VEL + dim] * q[DEN];
		ke += 0.5 * q[DEN] * q[VEL + dim] * q[VEL + dim];
	}
	u[PRE] = q[PRE] / (gamma - 1.0) + ke;
	u[HII] = q[HII] * q[DEN];
	u[ADV] = q[ADV] * q[DEN];
}

__device__ __forceinline__ void QfromU(double* q, const double* u, double gamma, int nd) {
	q[DEN] = u[DEN];
	double ke = 0;
	#pragma unroll
	for (int dim = 0; dim < 3; ++dim) if (dim < nd) {
		q[VEL + dim] = u[VEL + dim] / u[DEN];
		ke += 0.5 * u[VEL + dim] * u[VEL + dim] / u[DEN];
	}
	q[PRE] = (u[PRE] - ke) * (gamma - 1.0);
	q[HII] = u[HII] / u[DEN];
	q[ADV] = u[ADV] / u[DEN];
}

__device__ __forceinline__ void FfromQ(double* f, const double* q, double gamma, int nd, int dim) {
	f[DEN] = q[DEN] * q[VEL + dim];
	double ke = 0;
	#pragma unroll
	for (int id = 0; id < 3; ++id) if (id < nd) {
		ke += q[VEL + id] * q[VEL + id];
		int c = (dim + id) % nd;
		f[VEL + c] = q[DEN] * q[VEL + c] * q[VEL + dim];
	}
	ke *= 0.5 * q[DEN];
	f[VEL + dim] += q[PRE];
	double g2 = gamma / (gamma - 1.0);
	f[PRE] = q[VEL + dim] * (g2 * q[PRE] + ke);
	f[HII] = q[DEN] * q[VEL + dim] * q[HII];
	f[ADV] = q[DEN] * q[VEL + dim] * q[ADV];
}

// Fluid::calcTemperature, Fluid.cpp:71-74.
__device__ __forceinline__ double calc_temperature(const Params& P, double hii, double pre, double den) {
	double mu_inv = P.X * (hii + 1.0) + (1.0 - P.X) * 0.25;
#ifdef TRG_FAST_MATH
	return pre / (den * mu_inv * P.specificGasConstant);  // one division instead of three
#else
	return (pre / den) * (1.0 / mu_inv) / P.specificGasConstant;
#endif
}

// Fluid::fixPrimitives for one cell, Fluid.cpp:138-150 (floor uses U[DEN]).
__device__ __forceinline__ void fix_primitives(const Params& P, double* q, double u_den) {
	q[HII] = smax(smin(q[HII], 1.0), 0.0);
	q[ADV] = smax(smin(q[ADV], 1.0), 0.0);
	q[DEN] = smax(q[DEN], P.dfloor);
	q[PRE] = smax(q[PRE], P.pfloor);
	double mu_inv = P.X * (q[HII] + 1.0) + (1.0 - P.X) * 0.25;
	double temperature = q[PRE] / (mu_inv * P.specificGasConstant * q[DEN]);
	if (temperature < P.tfloor)
		q[PRE] = mu_inv * P.specificGasConstant * u_den * P.tfloor;
}

// Fluid::fixSolution for one cell, Fluid.cpp:89-136.  Returns false on the
// conditions under which the reference throws.
__device__ __forceinline__ bool fix_solution(const Params& P, double* u) {
	if (!isfinite(u[DEN]) || !isfinite(u[PRE])) return false;
	double hii = smax(smin(u[HII] / u[DEN], 1.0), 0.0);
	double adv = smax(smin(u[ADV] / u[DEN], 1.0), 0.0);
	double v[3] = {0, 0, 0};
	double den = smax(u[DEN], P.dfloor);
	#pragma unroll
	for (int dim = 0; dim < 3; ++dim) if (dim < P.nd) v[dim] = u[VEL + dim] / u[DEN];
	double ke = 0.0;
	#pragma unroll
	for (int dim = 0; dim < 3; ++dim) if (dim < P.nd) ke += v[dim] * v[dim];
	ke *= 0.5 * u[DEN];
	double pre = (u[PRE] - ke) * (P.gamma - 1.0);
	ke *= den / u[DEN];
	if (pre < P.pfloor) pre = P.pfloor;
	double mu_inv = P.X * (hii + 1.0) + (1.0 - P.X) * 0.25;
	double temperature = pre / (mu_inv * P.specificGasConstant * den);
	if (temperature < P.tfloor) pre = mu_inv * P.specificGasConstant * den * P.tfloor;
	u[DEN] = den;
	u[PRE] = pre / (P.gamma - 1.0) + ke;
	u[HII] = hii * den;
	u[ADV] = adv * den;
	#pragma unroll
	for (int dim = 0; dim < 3; ++dim) if (dim < P.nd) u[VEL + dim] = den * v[dim];
	if (u[DEN] == 0 || u[PRE] == 0) return false;
	for (int f = 0; f < NU; ++f)
		if (u[f] != u[f] || isinf(u[f])) return false;
	return true;
}

// ---------------------------------------------------------------- splines
// SplineData::splint (SplineData.cpp:57-81) and the two interpolate() forms.
__device__ __forceinline__ double splint(const Spline& s, double x2) {
	int klo = 0, khi = s.n - 1, k;
	while (khi - klo > 1) {
		k = (khi + klo) >> 1;
		if (s.x[k] > x2) khi = k;
		else klo = k;
	}
	double h = s.x[khi] - s.x[klo];
#ifdef TRG_FAST_MATH
	const double ih = 1.0 / h;
	double a = (s.x[khi] - x2) * ih;
	double b = (x2 - s.x[klo]) * ih;
#else
	double a = (s.x[khi] - x2) / h;
	double b = (x2 - s.x[klo]) / h;
#endif
	return a * s.y[klo] + b * s.y[khi] + ((a * a * a - a) * s.y2[klo] + (b * b * b - b) * s.y2[khi]) * (h * h) / 6.0;
}

__device__ __forceinline__ double spline_eval(const Spline& s, double x) {
	int n = s.n;
	if (s.log_mode) {
		if (x > s.x[n - 1]) return s.y[n - 1] + s.max_slope * (x - s.x[n - 1]);
		else if (x < s.x[0]) return s.y[0] + s.min_slope * (x - s.x[0]);
		return splint(s, x);
	}
	if (x > s.x[n - 1]) return s.y[n - 1] * d_pow(x / s.x[n - 1], s.max_slope);
	else if (x < s.x[0]) return s.y[0] * d_pow(x / s.x[0], s.min_slope);
	return splint(s, x);
}

// Diagnostic counters: one atomic per warp (the lanes that reach the call
// together), so that enabling them costs little next to the solves they count.
__device__ __forceinline__ void stat_add(unsigned long long* st, int idx, unsigned v) {
	unsigned m = __activemask();
	unsigned s = __reduce_add_sync(m, v);
	if ((int)(threadIdx.x & 31) == __ffs(m) - 1 && s) atomicAdd(st + idx, (unsigned long long)s);
}
__device__ __forceinline__ void stat_max(unsigned long long* st, int idx, unsigned v) {
	unsigned m = __activemask();
	unsigned s = __reduce_max_sync(m, v);
	if ((int)(threadIdx.x & 31) == __ffs(m) - 1 && s) atomicMax(st + idx, (unsigned long long)s);
}
// Picard iteration histogram bin: 1, 2, 3-4, 5-8, 9-16, 17-64, 65-1024, >1024
__device__ __forceinline__ int iter_bin(unsigned it) {
	return it <= 1 ? 0 : it <= 2 ? 1 : it <= 4 ? 2 : it <= 8 ? 3 : it <= 16 ? 4 : it <= 64 ? 5 : it <= 1024 ? 6 : 7;
}
__device__ __forceinline__ void stat_picard(unsigned long long* st, unsigned iters) {
	stat_add(st, TRG_STAT_PICARD_CELLS, iters > 0);
	stat_add(st, TRG_STAT_PICARD_ITERS, iters);
	stat_max(st, TRG_STAT_PICARD_MAX, iters);
	int b = iter_bin(iters);
#pragma unroll
	for (int k = 0; k < 8; ++k) stat_add(st, TRG_STAT_PICARD_HIST + k, iters > 0 && b == k);
}

// ------------------------------------------------------- conservation sums
// Global FP64 mass and energy sums, sum(rho V) and sum(E V) over the cells.
// Each cell's product is formed exactly (a double-double, two_prod) and the
// sums are carried as double-double pairs combined in a fixed tree order, so
// the result is deterministic (independent of scheduling) and equals the
// exact sum of the products to within about 2^-100 relative before its final
// rounding.  Every operation is an explicit round-to-nearest intrinsic, so
// the exact and the fast build (FMA contraction) compute the same bits.
struct DD {
	double hi, lo;
};
__device__ __forceinline__ DD dd_two_sum(double a, double b) {
	const double s = __dadd_rn(a, b);
	const double bb = __dsub_rn(s, a);
	return {s, __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb))};
}
__device__ __forceinline__ DD dd_fast_two_sum(double a, double b) {  // |a| >= |b| or a == 0
	const double s = __dadd_rn(a, b);
	return {s, __dsub_rn(b, __dsub_rn(s, a))};
}
__device__ __forceinline__ DD dd_add(DD a, DD b) {
	const DD s = dd_two_sum(a.hi, b.hi), t = dd_two_sum(a.lo, b.lo);
	const DD u = dd_fast_two_sum(s.hi, __dadd_rn(s.lo, t.hi));
	return dd_fast_two_sum(u.hi, __dadd_rn(u.lo, t.lo));
}
__device__ __forceinline__ DD dd_prod(double a, double b) {
	const double p = __dmul_rn(a, b);
	return {p, __fma_rn(a, b, -p)};
}
// Grid::computeCellVolume (Grid.cpp:876-905) with every operation rounded
// separately (no contraction in either build), the value the sums weight by.
__device__ __forceinline__ double cell_volume_rn(const Params& P, double rc) {
	const double PI = 3.14159265359;
	if (P.geometry == G_CART) {
		double volume = 1.0;
#pragma unroll
		for (int i = 0; i < 3; ++i)
			if (i < P.nd) volume = __dmul_rn(volume, P.dx[i]);
		return volume;
	}
	const double r2 = __dadd_rn(__dmul_rn(rc, P.dx[0]), __dmul_rn(0.5, P.dx[0]));
	const double r1 = __dsub_rn(__dmul_rn(rc, P.dx[0]), __dmul_rn(0.5, P.dx[0]));
	if (P.geometry == G_CYL) {
		double volume = __dmul_rn(__dmul_rn(PI, __dsub_rn(r2, r1)), __dadd_rn(r2, r1));
		if (P.nd >= 2) volume = __dmul_rn(volume, P.dx[1]);
		return volume;
	}
	const double s = __dadd_rn(__dadd_rn(__dmul_rn(r2, r2), __dmul_rn(r1, r2)), __dmul_rn(r1, r1));
	return __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(4.0, PI), __dsub_rn(r2, r1)), s), 3.0);
}
// Sums (m, e) over a block of 256 threads in a fixed order; thread 0 writes
// the block's partial (m.hi, m.lo, e.hi, e.lo) to part[4 * slot].  Every
// thread of the block must call it.
__device__ __forceinline__ void block_cons_partial(DD m, DD e, double* part, long long slot) {
	__shared__ double red[8][4];
	for (int o = 16; o > 0; o >>= 1) {
		const DD mo = {__shfl_down_sync(0xffffffffu, m.hi, o), __shfl_down_sync(0xffffffffu, m.lo, o)};
		const DD eo = {__shfl_down_sync(0xffffffffu, e.hi, o), __shfl_down_sync(0xffffffffu, e.lo, o)};
		m = dd_add(m, mo);
		e = dd_add(e, eo);
	}
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	if (lane == 0) {
		red[wid][0] = m.hi;
		red[wid][1] = m.lo;
		red[wid][2] = e.hi;
		red[wid][3] = e.lo;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		DD ms = {red[0][0], red[0][1]}, es = {red[0][2], red[0][3]};
		const int nw = (blockDim.x + 31) >> 5;
		for (int w = 1; w < nw; ++w) {
			ms = dd_add(ms, DD{red[w][0], red[w][1]});
			es = dd_add(es, DD{red[w][2], red[w][3]});
		}
		part[4 * slot + 0] = ms.hi;
		part[4 * slot + 1] = ms.lo;
		part[4 * slot + 2] = es.hi;
		part[4 * slot + 3] = es.lo;
	}
}

// Grid of a batched launch whose (padded) range holds position `pos`:
// the last g with off[g] <= pos.
__device__ __forceinline__ int batch_slot(const long long* off, int G, long long pos) {
	int lo = 0, hi = G - 1;
	while (lo < hi) {
		int mid = (lo + hi + 1) >> 1;
		if (off[mid] <= pos) lo = mid;
		else hi = mid - 1;
	}
	return lo;
}

}  // namespace trg
