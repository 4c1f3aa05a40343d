// FP32 performance form of the hydro pass: one fused kernel per RK2 stage.
//
// Per stage and cell: Q = QfromU(U) (+ fixPrimitives in the predictor),
// albada-limited piecewise-linear reconstruction, rotated HLLC-HLL flux on
// every face, flux divergence with the geometric source terms and wind
// injection, the Euler update and fixSolution - the work of
// Hydrodynamics::integrate/updateSourceTerms + Fluid::advSolution/fixSolution
// (src/Integrators/Hydro.cpp:31-156, src/Fluid/Fluid.cpp:80-136) - in one pass
// over HBM: the predictor reads U0 and writes U*, the corrector reads U* and
// U0 and writes U1, and also reduces the next CFL time step (FP64, Hydro.cpp:77-89).
//
// Tiling: a CTA owns a 32 x 8 column of cells and marches along z, keeping the
// primitives of three consecutive z-planes in a shared-memory ring; x/y halos
// of two cells are loaded with each plane.  Every cell is read from HBM once
// per CTA (plus the 2-cell x/y halos, which other CTAs share through L2), and
// every face flux is evaluated once.  A thread owns one cell of the plane (a
// warp owns one row): it computes the cell's limited slope once per direction
// (a face takes the slopes of its two cells), its low x, low y and high z
// faces, and its update; the neighbours' slopes and fluxes pass through
// shared memory, while the z slope of the column and the flux through its
// lower z face stay in registers from one plane to the next.  The plane three
// ahead is staged while the current one is computed: by one tiled TMA copy
// (cp.async.bulk.tensor, the whole haloed box of all seven fields) in CTAs
// whose box lies inside the grid, by per-cell cp.async through the boundary
// rule in the others.
//
// The rotated solver is written in directional form: HLL with normal n1 and
// HLLC with normal n2 are the reference's rotate / 1-D solve / rotate-back
// sequences (Riemann.cpp:181-244) without the rotation matrices, since the HLL
// and HLLC fluxes are rotation invariant.
//
// Pressure from total energy uses a compensated subtraction: the kinetic
// energy is formed as a float pair with error-free products and sums, so that
// E - KE loses no more than E's own rounding.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "trg_device.cuh"
#include "trg_kernels.h"

namespace trg {
namespace f32 {

constexpr int BX = 32, BY = 8, HALO = 2;
constexpr int SX = BX + 2 * HALO, SY = BY + 2 * HALO;
constexpr int NPLANE = 3;

struct Prim {
	float d, p, x, a, v[3];
};

// Floors and constants in the FP32 form's scaled units (state / reference value).
struct Scaled {
	float dfloor, pfloor, tfloor, Rg, X, gamma;
	int nd;
	__device__ explicit Scaled(const Params& P)
		: dfloor((float)(P.dfloor / P.f32_rho0)), pfloor((float)(P.pfloor / P.f32_p0)), tfloor((float)P.tfloor),
		  Rg((float)(P.specificGasConstant * P.f32_rho0 / P.f32_p0)), X((float)P.X), gamma((float)P.gamma), nd(P.nd) {}
};

__device__ __forceinline__ float fminf_(float a, float b) { return (b < a) ? b : a; }
// Division and reciprocal of the FP32 form: the hardware approximation (one
// reciprocal and one multiply, within 2 ulp for divisors of magnitude in
// [2^-126, 2^126], which the scaled units keep every divisor of this file in).
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ float frcp(float b) { return __fdividef(1.0f, b); }
// ... and the correctly rounded ones, kept in the radiation-hydro form (FP64
// state, CR = true below) where the rounding noise of every hydro sub-step
// feeds the long-run error against the FP64 form most: the reciprocal density
// of the primitives, and the square roots, reciprocal and sound speeds of the
// Einfeldt wave-speed estimate.  (Measured on the 256^3 HII region after 1000
// steps: pressure L1 1.2e-4 with every operation approximate, 4.9e-5 with
// these five correctly rounded, for 8% more time in this kernel.)  The
// hydro-only form (FP32 state) keeps them all approximate.
__device__ __forceinline__ float pdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float prcp(float b) { return __frcp_rn(b); }
__device__ __forceinline__ float psqrt(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ float fmaxf_(float a, float b) { return (a < b) ? b : a; }

// Conserved-state storage of the FP32 kernels: float arrays hold the scaled
// units directly; double arrays (the operator split's FP64 state) hold code
// units and are scaled on load and unscaled on store.
struct StoreScale {
	double s[3], is[3];  // density-like, pressure / energy, momentum
	__host__ __device__ explicit StoreScale(const Params& P) {
		s[0] = P.f32_rho0;
		s[1] = P.f32_p0;
		s[2] = P.f32_rho0 * P.f32_v0;
		for (int i = 0; i < 3; ++i) is[i] = 1.0 / s[i];
	}
	__device__ __forceinline__ int cls(int f) const { return f == PRE ? 1 : (f >= VEL ? 2 : 0); }
};
__device__ __forceinline__ float load_u(const float* U, long long idx, const StoreScale&, int) { return __ldg(&U[idx]); }
__device__ __forceinline__ float load_u(const double* U, long long idx, const StoreScale& sc, int f) {
	return (float)(__ldg(&U[idx]) * sc.is[sc.cls(f)]);
}
__device__ __forceinline__ float scaled_u(float u, const StoreScale&, int) { return u; }
__device__ __forceinline__ float scaled_u(double u, const StoreScale& sc, int f) { return (float)(u * sc.is[sc.cls(f)]); }
__device__ __forceinline__ void store_u(float* U, long long idx, float v, const StoreScale&, int) { U[idx] = v; }
__device__ __forceinline__ void store_u(double* U, long long idx, float v, const StoreScale& sc, int f) {
	U[idx] = (double)v * sc.s[sc.cls(f)];
}

// error-free transformations
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
	s = a + b;
	float bb = s - a;
	e = (a - (s - bb)) + (b - bb);
}
__device__ __forceinline__ void two_prod(float a, float b, float& p, float& e) {
	p = a * b;
	e = fmaf(a, b, -p);
}

// Q from U with the compensated E - KE.  KE = 0.5 |m|^2 / rho as a float pair.
template <bool CR>
__device__ __forceinline__ Prim prim_from_cons(const float* u, float gamma, int nd) {
	Prim q;
	q.d = u[DEN];
	float inv = CR ? prcp(u[DEN]) : frcp(u[DEN]);
	float s = 0.f, se = 0.f;
#pragma unroll
	for (int k = 0; k < 3; ++k) {
		q.v[k] = k < nd ? u[VEL + k] * inv : 0.f;
		if (k < nd) {
			float p, pe, t, te;
			two_prod(u[VEL + k], u[VEL + k], p, pe);
			two_sum(s, p, t, te);
			s = t;
			se += pe + te;
		}
	}
	// ke = 0.5 (s + se) / rho as (kh, kl)
	float kh = s * inv;
	float r = fmaf(-kh, u[DEN], s);  // exact remainder of s / rho
	float kl = (r + se) * inv;
	kh *= 0.5f;
	kl *= 0.5f;
	float dh, dl;
	two_sum(u[PRE], -kh, dh, dl);
	q.p = (dh + (dl - kl)) * (gamma - 1.0f);
	q.x = u[HII] * inv;
	q.a = u[ADV] * inv;
	return q;
}

__device__ __forceinline__ void fix_prim(const Scaled& P, Prim& q, float u_den) {
	q.x = fmaxf_(fminf_(q.x, 1.f), 0.f);
	q.a = fmaxf_(fminf_(q.a, 1.f), 0.f);
	q.d = fmaxf_(q.d, P.dfloor);
	q.p = fmaxf_(q.p, P.pfloor);
	float mu_inv = P.X * (q.x + 1.f) + (1.f - P.X) * 0.25f;
	// temperature = p / (mu_inv Rg rho) below the floor
	if (q.p < P.tfloor * (mu_inv * P.Rg * q.d)) q.p = mu_inv * P.Rg * u_den * P.tfloor;
}

// Fluid::fixSolution in FP32 (compensated kinetic energy as in prim_from_cons).
__device__ __forceinline__ bool fix_cons(const Scaled& P, float* u) {
	if (!isfinite(u[DEN]) || !isfinite(u[PRE])) return false;
	float inv = frcp(u[DEN]);
	float hii = fmaxf_(fminf_(u[HII] * inv, 1.f), 0.f);
	float adv = fmaxf_(fminf_(u[ADV] * inv, 1.f), 0.f);
	float den = fmaxf_(u[DEN], P.dfloor);
	const int nd = P.nd;
	float v[3];
#pragma unroll
	for (int k = 0; k < 3; ++k) v[k] = k < nd ? u[VEL + k] * inv : 0.f;
	Prim q = prim_from_cons<false>(u, P.gamma, nd);
	float pre = q.p;
	float ke = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
	ke *= 0.5f * den;
	if (pre < P.pfloor) pre = P.pfloor;
	float mu_inv = P.X * (hii + 1.f) + (1.f - P.X) * 0.25f;
	if (pre < P.tfloor * (mu_inv * P.Rg * den)) pre = mu_inv * P.Rg * den * P.tfloor;
	u[DEN] = den;
	u[PRE] = fdiv(pre, P.gamma - 1.f) + ke;
	u[HII] = hii * den;
	u[ADV] = adv * den;
#pragma unroll
	for (int k = 0; k < 3; ++k)
		if (k < nd) u[VEL + k] = den * v[k];
	if (u[DEN] == 0.f || u[PRE] == 0.f) return false;
	bool ok = true;
#pragma unroll
	for (int f = 0; f < NU; ++f) ok &= isfinite(u[f]);
	return ok;
}

// `thr` is the reference's 1e-30 cut on a*b (code units) in the field's
// scaled units: 1e-30 / s^2 for a field stored divided by s.
// The slope arithmetic is written with explicit roundings (no contraction
// left to the compiler), so that every call site computes a cell's slope and
// face states identically: a face shared by two z chunks of the tiling gets
// the same flux from both.
__device__ __forceinline__ float albada(float a, float b, float thr) {
	float ab = __fmul_rn(a, b);
	return ab <= thr ? 0.f : fdiv(__fmul_rn(ab, __fadd_rn(a, b)), __fmaf_rn(a, a, __fmul_rn(b, b)));
}
__device__ __forceinline__ float minmod_(float a, float b) {
	return (a * b > 0) ? (fabsf(a) < fabsf(b) ? a : b) : 0.f;
}
__device__ __forceinline__ float maxmod_(float a, float b) {
	return (a * b > 0) ? (fabsf(a) > fabsf(b) ? a : b) : 0.f;
}
__device__ __forceinline__ float limiter32(int kind, float a, float b, float thr) {
	switch (kind) {
	case 0: return minmod_((a + b) * 0.5f, minmod_(2.f * a, 2.f * b));
	case 1: return maxmod_(minmod_(b, 2.f * a), minmod_(2.f * b, a));
	case 2: return minmod_(a, b);
	case 3: return maxmod_(a, b);
	case 4: {
		if (b == 0) return 0.f;
		float r = fabsf(fdiv(a, b));
		return fdiv(__fmaf_rn(b, r, a), __fadd_rn(1.f, r));
	}
	case 5: {
		const float ab = __fmul_rn(a, b), t = __fmaf_rn(a, a, ab);
		return (ab <= thr) ? 0.f : fdiv(__fmul_rn(__fmul_rn(1.5f, b), t), __fmaf_rn(b, b, t));
	}
	default: return albada(a, b, thr);
	}
}

// Limiter cut-offs of the scaled fields (density, pressure, fractions, velocity).
struct LimThr {
	float d, p, x, v;
};
// Limited slope of a cell c between its neighbours cm and cp along one
// direction, per field: limiter(c - cm, cp - c).  The reconstruction of
// Hydro.cpp:44-50 gives a face between cells c1 and c2 the states
// QR(c1) = c1 + slope(c1) / 2 and QL(c2) = c2 - slope(c2) / 2.
__device__ __forceinline__ Prim slope_of(int lim, const LimThr& th, const Prim& cm, const Prim& c, const Prim& cp) {
	Prim s;
#define SLOPE(field, thr) s.field = limiter32(lim, c.field - cm.field, cp.field - c.field, thr);
	SLOPE(d, th.d) SLOPE(p, th.p) SLOPE(x, th.x) SLOPE(a, th.x) SLOPE(v[0], th.v) SLOPE(v[1], th.v) SLOPE(v[2], th.v)
#undef SLOPE
	return s;
}
__device__ __forceinline__ Prim face_left(const Prim& c, const Prim& sl) {
	Prim r;
	r.d = __fmaf_rn(0.5f, sl.d, c.d);
	r.p = __fmaf_rn(0.5f, sl.p, c.p);
	r.x = __fmaf_rn(0.5f, sl.x, c.x);
	r.a = __fmaf_rn(0.5f, sl.a, c.a);
#pragma unroll
	for (int k = 0; k < 3; ++k) r.v[k] = __fmaf_rn(0.5f, sl.v[k], c.v[k]);
	return r;
}
__device__ __forceinline__ Prim face_right(const Prim& c, const Prim& sr) {
	Prim r;
	r.d = __fmaf_rn(-0.5f, sr.d, c.d);
	r.p = __fmaf_rn(-0.5f, sr.p, c.p);
	r.x = __fmaf_rn(-0.5f, sr.x, c.x);
	r.a = __fmaf_rn(-0.5f, sr.a, c.a);
#pragma unroll
	for (int k = 0; k < 3; ++k) r.v[k] = __fmaf_rn(-0.5f, sr.v[k], c.v[k]);
	return r;
}

struct Flux {
	float f[7];
};

// The normal-independent parts of a face's two states, computed once per
// face and shared by the HLL and HLLC solves of the rotated solver:
// conserved states and the normal-independent terms of the Einfeldt speeds
// (characteristicWaveSpeeds, Riemann.cpp:27-42).
struct FacePre {
	float UL[7], UR[7];
	float sl, sr, inv, c2, nu2;
};
__device__ __forceinline__ void cons_of(const Prim& q, float g1inv, float* U) {
	float ke = 0.5f * q.d * (q.v[0] * q.v[0] + q.v[1] * q.v[1] + q.v[2] * q.v[2]);
	U[DEN] = q.d;
	U[PRE] = q.p * g1inv + ke;
	U[HII] = q.d * q.x;
	U[ADV] = q.d * q.a;
	for (int k = 0; k < 3; ++k) U[VEL + k] = q.d * q.v[k];
}
template <bool CR>
__device__ __forceinline__ void face_pre(const Prim& L, const Prim& R, float gamma, float g1inv, FacePre& f) {
	cons_of(L, g1inv, f.UL);
	cons_of(R, g1inv, f.UR);
	f.sl = CR ? psqrt(L.d) : sqrtf(L.d);
	f.sr = CR ? psqrt(R.d) : sqrtf(R.d);
	f.inv = CR ? prcp(f.sl + f.sr) : frcp(f.sl + f.sr);
	f.nu2 = 0.5f * f.sr * f.sl * f.inv * f.inv;
	float aL2 = CR ? pdiv(gamma * L.p, L.d) : fdiv(gamma * L.p, L.d);
	float aR2 = CR ? pdiv(gamma * R.p, R.d) : fdiv(gamma * R.p, R.d);
	f.c2 = (f.sl * aL2 + f.sr * aR2) * f.inv;
}
// Physical flux of a state (conserved U) along unit normal n.
__device__ __forceinline__ void flux_n(const Prim& q, const float* U, const float* n, float& un, float* F) {
	un = q.v[0] * n[0] + q.v[1] * n[1] + q.v[2] * n[2];
	float mflux = q.d * un;
	F[DEN] = mflux;
	F[PRE] = (U[PRE] + q.p) * un;
	F[HII] = mflux * q.x;
	F[ADV] = mflux * q.a;
	for (int k = 0; k < 3; ++k) F[VEL + k] = mflux * q.v[k] + q.p * n[k];
}
template <bool CR>
__device__ __forceinline__ void speeds_n(const FacePre& f, float unL, float unR, float& SL, float& SR) {
	float ut = (f.sl * unL + f.sr * unR) * f.inv;
	float d2 = f.c2 + f.nu2 * (unR - unL) * (unR - unL);
	float dd = CR ? psqrt(d2) : sqrtf(d2);
	SL = ut - dd;
	SR = ut + dd;
}

template <bool CR>
__device__ __forceinline__ void hll_n(const Prim& L, const Prim& R, const FacePre& f, const float* n, float* F) {
	float FL[7], FR[7], unL, unR, SL, SR;
	flux_n(L, f.UL, n, unL, FL);
	flux_n(R, f.UR, n, unR, FR);
	speeds_n<CR>(f, unL, unR, SL, SR);
	if (SR <= 0) {
		for (int i = 0; i < 7; ++i) F[i] = FR[i];
	} else if (SL >= 0) {
		for (int i = 0; i < 7; ++i) F[i] = FL[i];
	} else {
		float inv = frcp(SR - SL);
		for (int i = 0; i < 7; ++i) F[i] = (SR * FL[i] - SL * FR[i] + SL * SR * (f.UR[i] - f.UL[i])) * inv;
	}
}

template <bool CR>
__device__ __forceinline__ void hllc_n(const Prim& L, const Prim& R, const FacePre& f, const float* n, float* F) {
	float FL[7], FR[7], unL, unR, SL, SR;
	flux_n(L, f.UL, n, unL, FL);
	flux_n(R, f.UR, n, unR, FR);
	speeds_n<CR>(f, unL, unR, SL, SR);
	if (SL >= 0) {
		for (int i = 0; i < 7; ++i) F[i] = FL[i];
	} else if (SR <= 0) {
		for (int i = 0; i < 7; ++i) F[i] = FR[i];
	} else {
		float mL = L.d * (SL - unL), mR = R.d * (SR - unR);
		float Sc = fdiv(R.p - L.p + mL * unL - mR * unR, mL - mR);
		bool left = Sc >= 0;
		const Prim& K = left ? L : R;
		const float* UK = left ? f.UL : f.UR;
		const float* FK = left ? FL : FR;
		float SK = left ? SL : SR, unK = left ? unL : unR;
		float mK = K.d * (SK - unK);
		float A = fdiv(mK, SK - Sc);
		float Us[7];
		Us[DEN] = A;
		Us[PRE] = A * (fdiv(UK[PRE], K.d) + (Sc - unK) * (Sc + fdiv(K.p, mK)));
		Us[HII] = A * K.x;
		Us[ADV] = A * K.a;
		for (int k = 0; k < 3; ++k) Us[VEL + k] = A * (K.v[k] + (Sc - unK) * n[k]);
		for (int i = 0; i < 7; ++i) F[i] = FK[i] + SK * (Us[i] - UK[i]);
	}
}

// Rotated HLLC-HLL flux through a face with normal e_dim (Riemann.cpp:181-244).
// The branch tests use the exact components of the velocity jump dv along
// and across the face normal (the reference tests n1 x d == 0 and
// n2 x d == 0 exactly), and n2 is built from them without cancellation:
//   n1 = sign(dv_par) dv / |dv|,  |n1 . d| = |dv_par| / |dv| = cos,
//   n2 = (d |dv|^2 - dv_par dv) / (|dv| |dv_perp|),  n2 . d = |dv_perp| / |dv| = sin.
// Every case is F = w1 HLL(n1) + w2 HLLC(n2): the rotated flux (w1 = cos,
// w2 = sin), pure HLLC across the face (|dv| < 1e-6 or dv normal to the face:
// w1 = 0, n2 = d) or pure HLL along it (dv parallel to the face normal:
// w2 = 0, n1 = d); a solve with weight 0 is skipped, so the exact flux of the
// pure cases is kept, and each solver is inlined once.
// No array is indexed with the run-time dim, so everything stays in registers.
template <bool CR>
__device__ __forceinline__ void riemann32(int kind, const Prim& L, const Prim& R, int dim, float gamma, float* F) {
	const float g1inv = 1.f / (gamma - 1.f);
	const float d[3] = {dim == 0 ? 1.f : 0.f, dim == 1 ? 1.f : 0.f, dim == 2 ? 1.f : 0.f};
	FacePre f;
	face_pre<CR>(L, R, gamma, g1inv, f);
	float n1[3] = {d[0], d[1], d[2]}, n2[3] = {d[0], d[1], d[2]};
	float w1 = kind == RS_HLL ? 1.f : 0.f, w2 = kind == RS_HLLC ? 1.f : 0.f;
	if (kind == RS_ROTATED) {
		const float dv[3] = {R.v[0] - L.v[0], R.v[1] - L.v[1], R.v[2] - L.v[2]};
		const float par = dv[0] * d[0] + dv[1] * d[1] + dv[2] * d[2];  // exact: one term is non-zero
		const float perp[3] = {dv[0] - par * d[0], dv[1] - par * d[1], dv[2] - par * d[2]};  // exact
		const float pp = perp[0] * perp[0] + perp[1] * perp[1] + perp[2] * perp[2];
		const float rr = par * par + pp;
		if (rr < 1.0e-12f || par == 0.f) {  // |dv| < 1e-6, or dv normal to d: HLLC
			w2 = 1.f;
		} else if (pp == 0.f) {  // dv parallel to d: HLL
			w1 = 1.f;
		} else {
			const float r = sqrtf(rr), s = sqrtf(pp);
			const float inv_r = frcp(r);
			const float sg = par < 0 ? -1.f : 1.f;
#pragma unroll
			for (int k = 0; k < 3; ++k) n1[k] = sg * dv[k] * inv_r;
			w1 = fabsf(par) * inv_r;
			w2 = s * inv_r;
			const float k2 = fdiv(par * inv_r, s);
#pragma unroll
			for (int k = 0; k < 3; ++k) n2[k] = w2 * d[k] - k2 * perp[k];
		}
	}
	float F1[7], F2[7];
#pragma unroll
	for (int i = 0; i < 7; ++i) F1[i] = F2[i] = 0.f;
	if (w1 != 0.f) hll_n<CR>(L, R, f, n1, F1);
	if (w2 != 0.f) hllc_n<CR>(L, R, f, n2, F2);
#pragma unroll
	for (int i = 0; i < 7; ++i) F[i] = w1 * F1[i] + w2 * F2[i];
}

// A Prim, or a flux, in shared memory as two 16-byte halves kept in two
// arrays of the same index (fields 0-3, then 4-6 and a pad): consecutive
// threads read and write them with conflict-free 16-byte accesses, two per
// cell instead of seven.
struct V8 {
	float4* a;
	float4* b;
	__device__ __forceinline__ Prim get(int k) const {
		const float4 u = a[k], w = b[k];
		Prim q;
		q.d = u.x;
		q.p = u.y;
		q.x = u.z;
		q.a = u.w;
		q.v[0] = w.x;
		q.v[1] = w.y;
		q.v[2] = w.z;
		return q;
	}
	__device__ __forceinline__ void put(int k, const Prim& q) const {
		a[k] = make_float4(q.d, q.p, q.x, q.a);
		b[k] = make_float4(q.v[0], q.v[1], q.v[2], 0.f);
	}
	__device__ __forceinline__ void get_f(int k, float* f) const {
		const float4 u = a[k], w = b[k];
		f[0] = u.x;
		f[1] = u.y;
		f[2] = u.z;
		f[3] = u.w;
		f[4] = w.x;
		f[5] = w.y;
		f[6] = w.z;
	}
	__device__ __forceinline__ void put_f(int k, const float* f) const {
		a[k] = make_float4(f[0], f[1], f[2], f[3]);
		b[k] = make_float4(f[4], f[5], f[6], 0.f);
	}
};
// V8 arrays of a CTA: the three-plane ring of primitives (the x/y box of each
// plane, index ly * SX + lx), face fluxes, slopes.
constexpr int N_FX = BY * (BX + 1), N_FY = (BY + 1) * BX, N_S = BY * BX, N_EX = 2 * BY, N_EY = 2 * BX;
struct SmemQ {
	float4 a[NPLANE][SY * SX];
	float4 b[NPLANE][SY * SX];
	__device__ __forceinline__ V8 ring(int slot) { return V8{a[slot], b[slot]}; }
};

// Source position (with the boundary rule) of coordinate c along dim.
__device__ __forceinline__ int bc_src(const Params& P, int dim, int c, int n, int& flip_cond, int& side) {
	flip_cond = -1;
	side = 0;
	if (c < 0) {
		int k = -c;
		flip_cond = P.lbc[dim];
		return flip_cond == BC_PERIODIC ? n - k : (flip_cond == BC_REFLECTING ? k : 0);
	}
	if (c >= n) {
		int k = c - n + 1;
		flip_cond = P.rbc[dim];
		side = 1;
		return flip_cond == BC_PERIODIC ? k - 1 : (flip_cond == BC_REFLECTING ? n - 1 - k : n - 1);
	}
	return c;
}

__device__ __forceinline__ void apply_flip(Prim& q, int dim, int cond, int side) {
	if (cond < 0) return;
	float v = q.v[dim];
	if (cond == BC_INFLOW) {
		if (side == 0 ? v < 0 : v > 0) q.v[dim] = -v;
	} else if (cond == BC_OUTFLOW) {
		if (side == 0 ? v > 0 : v < 0) q.v[dim] = -v;
	} else if (cond == BC_REFLECTING) {
		q.v[dim] = -v;
	}
}

// The staged cells of the CTA's x/y box (halo included, corners left out: no
// stencil reads them) and their sources under the boundary rule depend on
// the CTA's position only, not on the plane: a thread works out its (at most
// two) box positions once, before the z march.  Per position: the source
// offset xs + nx ys within a plane (-1: not staged - a corner, or beyond a
// ragged grid edge; below -1: a ghost layer of a slab face, from the halo)
// and the velocity flips the boundary rule applies there.
constexpr int STAGE_PER_THREAD = (SX * SY + BX * BY - 1) / (BX * BY);
struct StageMap {
	int off[STAGE_PER_THREAD];
	int flags[STAGE_PER_THREAD];  // x condition + 1 (3 bits), x side, y condition + 1 (3 bits), y side
};
__device__ __forceinline__ StageMap stage_map(const Params& P, int x0, int y0) {
	StageMap m;
#pragma unroll
	for (int j = 0; j < STAGE_PER_THREAD; ++j) {
		const int idx = threadIdx.x + j * BX * BY;
		m.off[j] = -1;
		m.flags[j] = 0;
		if (idx >= SX * SY) continue;
		const int ly = idx / SX, lx = idx - ly * SX;
		const bool xh = lx < HALO || lx >= HALO + BX, yh = ly < HALO || ly >= HALO + BY;
		if (xh && yh) continue;  // corners: never part of a stencil
		int xc, xside, yc = -1, yside = 0;
		const int gxp = x0 + lx - HALO;
		const int xs = bc_src(P, 0, gxp, P.nx, xc, xside);
		const int ys = P.nd > 1 ? bc_src(P, 1, y0 + ly - HALO, P.ny, yc, yside) : 0;
		if (P.nd <= 1) yc = -1;
		if (xc == BC_PARTITION) {
			// ghost layer of a slab face: from the neighbour's halo
			// ([side][layer][field][ny * nz]), coded as -2 - ((side 2 + layer) ny + ys).
			// Box positions further out than the HALO ghost layers (a tile that
			// overhangs a slab narrower than BX) are no stencil's cells and are
			// not staged: the halo holds HALO layers per side only.
			if (ys < 0 || ys >= P.ny) continue;
			const int layer = (xside ? gxp - P.nx + 1 : -gxp) - 1;
			if (layer >= HALO) continue;
			m.off[j] = -2 - ((xside * 2 + layer) * P.ny + ys);
			m.flags[j] = ((yc + 1) << 4) | (yside << 7);
			continue;
		}
		if (xs < 0 || xs >= P.nx || ys < 0 || ys >= P.ny) continue;  // tile beyond a ragged grid edge
		m.off[j] = xs + P.nx * ys;
		m.flags[j] = (xc + 1) | (xside << 3) | ((yc + 1) << 4) | (yside << 7);
	}
	return m;
}
__device__ __forceinline__ void apply_flips(const Params& P, Prim& q, int flags, int zc, int zside) {
	apply_flip(q, 0, (flags & 7) - 1, (flags >> 3) & 1);
	if (P.nd > 1) apply_flip(q, 1, ((flags >> 4) & 7) - 1, (flags >> 7) & 1);
	if (P.nd > 2) apply_flip(q, 2, zc, zside);
}
__device__ __forceinline__ void put_prim(SmemQ& s, int slot, int idx, const Prim& q) { s.ring(slot).put(idx, q); }
// Source plane of z under the boundary rule (2-D grids: plane 0).
__device__ __forceinline__ int plane_src(const Params& P, int z, int& zc, int& zside) {
	zc = -1;
	zside = 0;
	return P.nd > 2 ? bc_src(P, 2, z, P.nz, zc, zside) : 0;
}

// Source of field f of staged position j in source plane zs: the state, or
// for a ghost layer of a slab face the neighbour's halo.
template <typename TS>
__device__ __forceinline__ const TS* stage_src(const Params& P, const TS* Up, const void* halo, int off, int f,
                                               int zs) {
	if (off >= 0) return Up + (long long)f * P.N + off;
	const int code = -2 - off, sl = code / P.ny, ys = code - sl * P.ny;
	const long long nyz = (long long)P.ny * P.nz;
	return static_cast<const TS*>(halo) + (long long)(sl * NU + f) * nyz + ys + (long long)P.ny * zs;
}

// Loads plane z (global index, may be a ghost plane) of the CTA's x/y box into ring slot.
template <int STAGE, typename TS>
__device__ __forceinline__ void load_plane(const Params& P, const Scaled& SP, const StoreScale& SC,
                                           const TS* __restrict__ U, const void* halo, SmemQ& s, int slot,
                                           const StageMap& m, int z) {
	int zc, zside;
	const int zs = plane_src(P, z, zc, zside);
	const TS* Up = U + (long long)P.nx * P.ny * zs;
#pragma unroll
	for (int j = 0; j < STAGE_PER_THREAD; ++j) {
		if (m.off[j] == -1) continue;
		float u[7];
#pragma unroll
		for (int f = 0; f < 7; ++f) u[f] = load_u(stage_src(P, Up, halo, m.off[j], f, zs), 0, SC, f);
		Prim q = prim_from_cons<sizeof(TS) == sizeof(double)>(u, (float)P.gamma, P.nd);
		if (STAGE == 1) fix_prim(SP, q, u[DEN]);
		apply_flips(P, q, m.flags[j], zc, zside);
		put_prim(s, slot, threadIdx.x + j * BX * BY, q);
	}
}

// Asynchronous staging of a plane (cp.async): the raw conserved state of the
// plane's cells, with the boundary rule applied to the source index, is
// copied into a shared-memory buffer [7][SY * SX] while the CTA computes the
// current plane, and turned into primitives in the ring slot afterwards.
// The cells and the source rule are those of load_plane.
template <typename TS>
__device__ __forceinline__ void cp_async_elem(TS* dst, const TS* src) {
	const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
	if (sizeof(TS) == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
	else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Tiled TMA staging of a plane (FP64 state, CTAs whose haloed box lies inside
// the grid): one cp.async.bulk.tensor copy of the box x0 - 2 .. x0 + 33,
// y0 - 2 .. y0 + 9 of source plane zs, all seven fields, into the staging
// buffer in its [7][SY][SX] layout, completing on an mbarrier.  The x
// coordinate x0 - 2 with x0 a multiple of 32 is a multiple of 2 elements of
// 8 bytes, so the copy starts on a 16-byte boundary.
constexpr unsigned TMA_BYTES = 7u * SX * SY * 8u;
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void tma_bar_init(uint64_t* bar) {
	asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void tma_plane(const CUtensorMap* tmap, void* dst, uint64_t* bar, int x, int y, int z) {
	// generic-proxy reads of the buffer (the previous plane's conversion) are
	// ordered before the async-proxy writes of this copy
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(TMA_BYTES)
	             : "memory");
	asm volatile(
	    "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
	    "%5}], [%6];" ::"r"(smem_addr(dst)),
	    "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(z), "r"(0), "r"(smem_addr(bar))
	    : "memory");
}
// Bounded wait for the copy of the given phase: false if it did not complete
// within the limit (the caller reports it; the kernel never hangs).
__device__ __forceinline__ bool tma_wait(uint64_t* bar, uint32_t phase) {
	for (int i = 0; i < (1 << 22); ++i) {
		uint32_t ok;
		asm volatile(
		    "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
		    "selp.b32 %0, 1, 0, P1;\n\t}\n"
		    : "=r"(ok)
		    : "r"(smem_addr(bar)), "r"(phase)
		    : "memory");
		if (ok) return true;
	}
	return false;
}

template <typename TS>
__device__ __forceinline__ void plane_fetch(const Params& P, const TS* __restrict__ U, const void* halo, TS* raw,
                                            const StageMap& m, int z) {
	int zc, zside;
	const int zs = plane_src(P, z, zc, zside);
	const TS* Up = U + (long long)P.nx * P.ny * zs;
#pragma unroll
	for (int j = 0; j < STAGE_PER_THREAD; ++j) {
		if (m.off[j] == -1) continue;
		const int idx = threadIdx.x + j * BX * BY;
#pragma unroll
		for (int f = 0; f < 7; ++f) cp_async_elem(raw + f * (SX * SY) + idx, stage_src(P, Up, halo, m.off[j], f, zs));
	}
	cp_async_commit();
}
template <int STAGE, typename TS>
__device__ __forceinline__ void plane_convert(const Params& P, const Scaled& SP, const StoreScale& SC, const TS* raw,
                                              SmemQ& s, int slot, const StageMap& m, int z) {
	int zc, zside;
	plane_src(P, z, zc, zside);
#pragma unroll
	for (int j = 0; j < STAGE_PER_THREAD; ++j) {
		if (m.off[j] == -1) continue;
		const int idx = threadIdx.x + j * BX * BY;
		float u[7];
#pragma unroll
		for (int f = 0; f < 7; ++f) u[f] = scaled_u(raw[f * (SX * SY) + idx], SC, f);
		Prim q = prim_from_cons<sizeof(TS) == sizeof(double)>(u, (float)P.gamma, P.nd);
		if (STAGE == 1) fix_prim(SP, q, u[DEN]);
		apply_flips(P, q, m.flags[j], zc, zside);
		put_prim(s, slot, idx, q);
	}
}

__device__ __forceinline__ Prim get(SmemQ& s, int slot, int ly, int lx) { return s.ring(slot).get(ly * SX + lx); }

__device__ __forceinline__ double dmin_(double a, double b) { return (b < a) ? b : a; }

// Fluid::advSolution + fixSolution (Fluid.cpp:80-136) of one cell of the FP64
// state, in FP64: U_out = fix(U_base + inc), the increment inc = dt L(Q) formed
// in FP32 (scaled units) by the caller.  With `write_q` also the primitives
// that globalQfromU + fixPrimitives (Fluid.cpp:138-165) would form from the
// fixed state, taken from the fix itself (equal up to rounding: the fix has
// already applied the floors).  One reciprocal of the density replaces the
// reference's divisions, and the temperature floor is tested as
// pre < T_floor mu_inv R den.  Fields are formed one at a time, as they are
// needed, to keep the register footprint of the calling kernel small.
// Returns false where the reference throws.
__device__ __forceinline__ bool update_state64(const Params& P, const State& S, const StoreScale& SC,
                                               const double* __restrict__ Ub, double* __restrict__ Uo, long long id,
                                               float dtf, const float* udot, bool write_q) {
	const long long N = P.N;
	const int nd = P.nd;
	auto nu = [&](int f) { return __ldg(&Ub[f * N + id]) + (double)(dtf * udot[f]) * SC.s[SC.cls(f)]; };
	const double d = nu(DEN), e = nu(PRE);
	const double inv = 1.0 / d;
	const double hii = smax(smin(nu(HII) * inv, 1.0), 0.0);
	const double adv = smax(smin(nu(ADV) * inv, 1.0), 0.0);
	const double den = smax(d, P.dfloor);
	double v[3] = {0, 0, 0};
#pragma unroll
	for (int k = 0; k < 3; ++k)
		if (k < nd) v[k] = nu(VEL + k) * inv;
	double ke = ((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]) * (0.5 * d);
	double pre = (e - ke) * (P.gamma - 1.0);
	ke *= den * inv;
	if (pre < P.pfloor) pre = P.pfloor;
	const double mu_inv = P.X * (hii + 1.0) + (1.0 - P.X) * 0.25;
	const double pt = mu_inv * P.specificGasConstant * den * P.tfloor;
	if (pre < pt) pre = pt;
	const double E = pre / (P.gamma - 1.0) + ke;
	Uo[DEN * N + id] = den;
	Uo[PRE * N + id] = E;
	Uo[HII * N + id] = hii * den;
	Uo[ADV * N + id] = adv * den;
	bool ok = isfinite(d) && isfinite(e) && den != 0 && E != 0 && isfinite(E) && isfinite(hii * den) &&
	          isfinite(adv * den);
#pragma unroll
	for (int k = 0; k < 3; ++k)
		if (k < nd) {
			const double m = den * v[k];
			Uo[(VEL + k) * N + id] = m;
			ok &= isfinite(m);
		}
	if (write_q) {
		FLD(S.Q, DEN, id) = den;
		FLD(S.Q, PRE, id) = pre;
		FLD(S.Q, HII, id) = hii;
		FLD(S.Q, ADV, id) = adv;
#pragma unroll
		for (int k = 0; k < 3; ++k)
			if (k < nd) FLD(S.Q, VEL + k, id) = v[k];
	}
	return ok;
}

}  // namespace f32

using namespace f32;

// Byte offset of the plane staging buffer in the kernel's shared memory:
// after the ring and the flux and slope arrays.
__host__ __device__ constexpr size_t hydro_stage_raw_offset() {
	return (sizeof(f32::SmemQ) + 2 * sizeof(float4) * (f32::N_FX + f32::N_FY + 2 * f32::N_S + f32::N_EX + f32::N_EY) +
	        127) /
	       128 * 128;  // 128-byte aligned: the destination of the TMA plane copy
}

// Riemann solve for one face from its reconstructed states.
// CR: the correctly rounded operations of the radiation-hydro form (above).
template <int RS, bool CR>
__device__ __forceinline__ void face_flux(int rs_rt, const Prim& L, const Prim& R, int dim, float gamma, float* F) {
	riemann32<CR>(RS >= 0 ? RS : rs_rt, L, R, dim, gamma, F);
}

// One Euler stage U_out = fix(U_base + h dt L(Q(U_q))).
// STAGE 1: Q with floors (fixPrimitives) - the RK2 predictor (h = 1/2) and the
//          hydro sub-step of the operator split (h = 1/2 or 1);
// STAGE 2: Q(U*) without floors, plus the next step's CFL minimum - the RK2
//          corrector (h = 1).
// TS: storage type (float: scaled units; double: code units).
// LIM / RS: limiter and Riemann solver fixed at compile time (-1: chosen at run time).
// tmap / use_tma: the tensor map of the FP64 state Uq for the TMA plane
// staging (use_tma = 0: per-cell cp.async staging everywhere).
// The body runs the CTA's tile (bx, by, bz) of one grid (P, S): the kernel's
// own block index for a single grid, an entry of the tile table for a batch.
template <int STAGE, typename TS, int LIM, int RS>
__device__ __forceinline__ void hydro_stage_body(const Params& P, const State& S, const TS* __restrict__ Uq,
                                                 const TS* Ubase, TS* Uout, double hfac, int zchunk,
                                                 const CUtensorMap* tmap, int use_tma, int bx, int by, int bz) {
	extern __shared__ __align__(128) unsigned char smem_raw[];
	constexpr bool CR = sizeof(TS) == sizeof(double);  // the radiation-hydro form's correctly rounded operations
	SmemQ& s = *reinterpret_cast<SmemQ*>(smem_raw);
	float4* v8 = reinterpret_cast<float4*>(smem_raw + sizeof(SmemQ));
	const V8 Fx{v8, v8 + N_FX};                      // [BY][BX + 1] x-face fluxes
	v8 += 2 * N_FX;
	const V8 Fy{v8, v8 + N_FY};                      // [BY + 1][BX] y-face fluxes
	v8 += 2 * N_FY;
	const V8 Sx{v8, v8 + N_S};                       // [BY * BX] x slopes of the tile
	v8 += 2 * N_S;
	const V8 Sy{v8, v8 + N_S};                       // [BY * BX] y slopes of the tile
	v8 += 2 * N_S;
	const V8 Ex{v8, v8 + N_EX};                      // [2 * BY] x slopes of cells x0 - 1, x0 + BX
	v8 += 2 * N_EX;
	const V8 Ey{v8, v8 + N_EY};                      // [2 * BX] y slopes of cells y0 - 1, y0 + BY
	TS* raw = reinterpret_cast<TS*>(smem_raw + hydro_stage_raw_offset());  // [7][SY * SX] next plane, staged
	uint64_t* tbar = reinterpret_cast<uint64_t*>(smem_raw + hydro_stage_raw_offset() + sizeof(double) * 7 * SX * SY);
	const int tx = threadIdx.x % BX, ty = threadIdx.x / BX;
	const int lx = tx + HALO, ly = ty + HALO;
	const int x0 = bx * BX, y0 = by * BY;
	const int z0 = bz * zchunk;
	const int nd = P.nd;
	const int z1 = nd > 2 ? min(z0 + zchunk, P.nz) : 1;
	const float gamma = (float)P.gamma;
	const Scaled SP(P);
	// scaled time: t' = t v0 (lengths stay in code units)
	const StoreScale SC(P);
	const double dt = hfac * S.scal[0] * P.f32_v0;
	const float dtf = (float)dt;
	const float gscale = (float)(1.0 / P.f32_p0);
	const long long N = P.N;
	const int gx = x0 + tx, gy = y0 + ty;
	const bool active = gx < P.nx && gy < P.ny;
	const bool rec = P.order == 1;
	const int lim = LIM >= 0 ? LIM : P.limiter, rs_rt = P.riemann;
	const LimThr th{(float)(1.0e-30 / (P.f32_rho0 * P.f32_rho0)), (float)(1.0e-30 / (P.f32_p0 * P.f32_p0)), 1.0e-30f,
	                (float)(1.0e-30 / (P.f32_v0 * P.f32_v0))};
	// faces of this thread: x at gx - 1/2 and y at gy - 1/2 where they are
	// faces of the grid; the tile's last x face (x0 + BX - 1/2) of each row and
	// last y face (y0 + BY - 1/2) of each column are computed by warps 0-1
	const bool fx_ok = gx <= P.nx && gy < P.ny;
	const bool fy_ok = nd > 1 && gx < P.nx && gy <= P.ny;
	const int te = threadIdx.x;  // last faces: te < BX y face of column te; BX <= te < BX + BY x face of row te - BX
	const bool fe_ok = te < BX ? (nd > 1 && x0 + te < P.nx && y0 + BY <= P.ny)
	                           : (te < BX + BY && x0 + BX <= P.nx && y0 + te - BX < P.ny);
	// edge slopes (cells just outside the tile): the last 80 threads
	const int ts = (int)threadIdx.x - (BX * BY - 2 * (BX + BY));
	double tmin = 1.0e308;
	bool bad = false;

	// geometry of this thread's cell column: cartesian factors are uniform
	float axl = 0, axr = 0, ayl = 0, ayr = 0, azl = 0, azr = 0, rgeo = 0;
	int ijk[3] = {gx, gy, 0};
	double xc[3];
	cell_xc(P, ijk, xc);
	{
		double vol = cell_volume(P, xc[0]);
		axl = (float)(face_area(P, xc, 0, 0) / vol);
		axr = (float)(face_area(P, xc, 0, 1) / vol);
		if (nd > 1) { ayl = (float)(face_area(P, xc, 1, 0) / vol); ayr = (float)(face_area(P, xc, 1, 1) / vol); }
		if (nd > 2) { azl = (float)(face_area(P, xc, 2, 0) / vol); azr = (float)(face_area(P, xc, 2, 1) / vol); }
		if (P.geometry == G_CYL) rgeo = (float)(1.0 / (P.dx[0] * xc[0]));
		else if (P.geometry == G_SPH) rgeo = (float)((face_area(P, xc, 0, 1) - face_area(P, xc, 0, 0)) / vol);
	}

	const StageMap smap = stage_map(P, x0, y0);
	// TMA staging: FP64 state, 3-D, the CTA's haloed x/y box inside the grid
	const bool tma = sizeof(TS) == sizeof(double) && use_tma && nd > 2 && x0 >= HALO && x0 + BX + HALO <= P.nx &&
	                 y0 >= HALO && y0 + BY + HALO <= P.ny;
	uint32_t tphase = 0;
	bool tma_late = false;
	if (tma && threadIdx.x == 0) tma_bar_init(tbar);  // ordered before use by the first barrier below
	auto slot_of = [](int z) { return ((z % NPLANE) + NPLANE) % NPLANE; };
	int s_z = nd > 2 ? slot_of(z0 - 1) : 0;  // ring slot of the loop's plane z, advanced with z
	Prim zero;
	zero.d = zero.p = zero.x = zero.a = zero.v[0] = zero.v[1] = zero.v[2] = 0.f;
	Prim szc = zero;  // z slope of this column's cell in the current plane
	float fzlo[7];    // flux through the column's face z - 1/2
#pragma unroll
	for (int i = 0; i < 7; ++i) fzlo[i] = 0.f;
	// 3-D: the pass starts one plane early (z0 - 1), where it only forms the
	// flux through z0 - 1/2, so that every z face goes through the same code
	if (nd > 2) {
		for (int z = z0 - 2; z <= z0; ++z) load_plane<STAGE>(P, SP, SC, Uq, S.halo_recv, s, slot_of(z), smap, z);
		__syncthreads();
		if (rec)
			szc = slope_of(lim, th, get(s, slot_of(z0 - 2), ly, lx), get(s, slot_of(z0 - 1), ly, lx),
			               get(s, slot_of(z0), ly, lx));
		__syncthreads();  // plane z0 - 2 is read: its slot takes plane z0 + 1
		load_plane<STAGE>(P, SP, SC, Uq, S.halo_recv, s, slot_of(z0 + 1), smap, z0 + 1);
	} else {
		load_plane<STAGE>(P, SP, SC, Uq, S.halo_recv, s, 0, smap, 0);
	}

	// Plane z + 3 is staged (cp.async) while plane z is computed and turned into
	// primitives after its update, into the slot of plane z, which nothing
	// reads after the flux barrier.
	for (int z = nd > 2 ? z0 - 1 : z0; z < z1; ++z) {
		const int sc = s_z;  // planes z + 1 and z + 2 in the next slots; z + 3 comes into sc
		const int s_z1 = sc == NPLANE - 1 ? 0 : sc + 1, s_z2 = s_z1 == NPLANE - 1 ? 0 : s_z1 + 1;
		const bool plane = z >= z0;  // x/y faces and the update of this plane
		const bool stage_next = nd > 2 && z + 1 < z1;
		__syncthreads();  // planes z .. z + 2 are in the ring; the staging buffer is free
		if (stage_next) {
			if (tma) {
				if (threadIdx.x == 0) {
					int zc, zside;
					tma_plane(tmap, raw, tbar, x0 - HALO, y0 - HALO, plane_src(P, z + 3, zc, zside));
				}
			} else {
				plane_fetch(P, Uq, S.halo_recv, raw, smap, z + 3);
			}
		}
		// slopes: this cell in x, y and (of the next plane's cell) z; the cells
		// just outside the tile in x and y
		Prim szn = zero;
		if (rec) {
			const Prim qc = get(s, sc, ly, lx);
			if (nd > 2)
				szn = slope_of(lim, th, qc, get(s, s_z1, ly, lx), get(s, s_z2, ly, lx));
		}
		if (rec && plane) {
			const Prim qc = get(s, sc, ly, lx);
			Sx.put(threadIdx.x, slope_of(lim, th, get(s, sc, ly, lx - 1), qc, get(s, sc, ly, lx + 1)));
			if (nd > 1)
				Sy.put(threadIdx.x, slope_of(lim, th, get(s, sc, ly - 1, lx), qc, get(s, sc, ly + 1, lx)));
			if (ts >= 0 && ts < 2 * BY) {
				const int e = ts / BY, r = ts - e * BY, ex = e ? HALO + BX : HALO - 1;
				Ex.put(ts,
				     slope_of(lim, th, get(s, sc, r + HALO, ex - 1), get(s, sc, r + HALO, ex), get(s, sc, r + HALO, ex + 1)));
			} else if (ts >= 2 * BY && nd > 1) {
				const int u = ts - 2 * BY, e = u / BX, col = u - e * BX, ey = e ? HALO + BY : HALO - 1;
				Ey.put(u,
				     slope_of(lim, th, get(s, sc, ey - 1, col + HALO), get(s, sc, ey, col + HALO), get(s, sc, ey + 1, col + HALO)));
			}
		}
		__syncthreads();
		// faces: the x face below and the y face below this cell, then (warps
		// 0-1) the tile's last y and x faces, through one call of the solver;
		// then the z face above this cell through a second one, its flux kept
		// in registers (this thread's own update and, as the flux below, the
		// next plane's)
		const int nk = te < BX + BY ? 3 : 2;  // only threads 0 .. BX + BY - 1 take a last face
#pragma unroll 1
		for (int k = 0; k < nk; ++k) {
			Prim ql, qr, sl = zero, sr = zero;
			int dim;
			bool ok;
			V8 dst;
			int di;
			if (k == 0) {  // x face gx - 1/2, between cells lx - 1 and lx of row ly
				ok = fx_ok && plane;
				dim = 0;
				ql = get(s, sc, ly, lx - 1);
				qr = get(s, sc, ly, lx);
				if (rec && ok) {
					sl = tx > 0 ? Sx.get(threadIdx.x - 1) : Ex.get(ty);
					sr = Sx.get(threadIdx.x);
				}
				dst = Fx;
				di = ty * (BX + 1) + tx;
			} else if (k == 1) {  // y face gy - 1/2, between rows ly - 1 and ly of column lx
				ok = fy_ok && plane;
				dim = 1;
				ql = get(s, sc, ly - 1, lx);
				qr = get(s, sc, ly, lx);
				if (rec && ok) {
					sl = ty > 0 ? Sy.get(threadIdx.x - BX) : Ey.get(tx);
					sr = Sy.get(threadIdx.x);
				}
				dst = Fy;
				di = ty * BX + tx;
			} else if (te < BX) {  // y face y0 + BY - 1/2 of column te
				ok = fe_ok && plane;
				dim = 1;
				ql = get(s, sc, HALO + BY - 1, te + HALO);
				qr = get(s, sc, HALO + BY, te + HALO);
				if (rec && ok) {
					sl = Sy.get((BY - 1) * BX + te);
					sr = Ey.get(BX + te);
				}
				dst = Fy;
				di = BY * BX + te;
			} else {  // x face x0 + BX - 1/2 of row te - BX
				ok = fe_ok && plane;
				dim = 0;
				const int r = min(te - BX, BY - 1);
				ql = get(s, sc, r + HALO, HALO + BX - 1);
				qr = get(s, sc, r + HALO, HALO + BX);
				if (rec && ok) {
					sl = Sx.get(r * BX + BX - 1);
					sr = Ex.get(BY + r);
				}
				dst = Fx;
				di = r * (BX + 1) + BX;
			}
			if (!ok) continue;
			float f[7];
			face_flux<RS, CR>(rs_rt, rec ? face_left(ql, sl) : ql, rec ? face_right(qr, sr) : qr, dim, gamma, f);
			dst.put_f(di, f);
		}
		float fz[7];  // flux through this column's face z + 1/2
		if (nd > 2) {
			const Prim ql = get(s, sc, ly, lx), qr = get(s, s_z1, ly, lx);
			face_flux<RS, CR>(rs_rt, rec ? face_left(ql, szc) : ql, rec ? face_right(qr, szn) : qr, 2, gamma, fz);
		}
		// the cell itself for the source terms, read before the barrier: after
		// it, nothing of this plane is read, so the next plane's load may reuse
		// the slot without another barrier
		const Prim qc = get(s, sc, ly, lx);
		if (stage_next) {  // plane z + 3 has landed (this thread's copies, or the CTA's TMA copy)
			if (tma) {
				tma_late |= !tma_wait(tbar, tphase);
				tphase ^= 1u;
			} else {
				cp_async_wait_all();
			}
		}
		__syncthreads();
		if (active && plane) {
			const long long id = gx + (long long)P.nx * (gy + (long long)P.ny * z);
			float udot[7], fl[7], fr[7];
			Fx.get_f(ty * (BX + 1) + tx, fl);
			Fx.get_f(ty * (BX + 1) + tx + 1, fr);
#pragma unroll
			for (int i = 0; i < 7; ++i) udot[i] = axl * fl[i] - axr * fr[i];
			if (nd > 1) {
				Fy.get_f(ty * BX + tx, fl);
				Fy.get_f((ty + 1) * BX + tx, fr);
#pragma unroll
				for (int i = 0; i < 7; ++i) udot[i] += ayl * fl[i] - ayr * fr[i];
			}
			if (nd > 2) {
#pragma unroll
				for (int i = 0; i < 7; ++i) udot[i] += azl * fzlo[i] - azr * fz[i];
			}
			if (S.grav) {
				for (int k = 0; k < 3; ++k) {
					float g = (float)S.grav[(long long)k * N + id] * gscale;
					udot[VEL + k] += g;
					udot[PRE] += qc.v[k] * g;
				}
			}
			if (P.geometry == G_CYL) udot[VEL + 0] += qc.p * rgeo;
			else if (P.geometry == G_SPH) udot[VEL + 0] += qc.p * rgeo;
			if (P.star_on && P.mdot != 0) {
				int cijk[3] = {gx, gy, z};
				double cxc[3];
				cell_xc(P, cijk, cxc);
				if (is_wind(P, id, cijk, cxc)) {
					float mdot = (float)(P.mdot / (P.f32_rho0 * P.f32_v0));
					udot[DEN] += mdot;
					udot[PRE] += (float)(P.edot / (P.f32_p0 * P.f32_v0));
					udot[HII] += (load_u(Ubase, HII * N + id, SC, HII) / load_u(Ubase, DEN * N + id, SC, DEN)) * mdot;
					udot[ADV] += mdot;
				}
			}
			float u[7];
			if constexpr (sizeof(TS) == sizeof(double)) {
				// hydro sub-step of a radiation-hydro run on the FP64 state: the
				// FP32 increment dt L(Q) is added to the unrounded FP64 state and
				// fixSolution runs in FP64, so a cell keeps its FP64 digits where
				// the flux divergence is small (Fluid::advSolution, Fluid.cpp:80-87,
				// updates U in FP64).  The FP64 primitives of the fixed state are
				// written as well (what globalQfromU + fixPrimitives of the next
				// sub-step would compute), so that pass is skipped; cells of the
				// FP64 fallback keep their old Q for its update.
				bad |= !update_state64(P, S, SC, Ubase, Uout, id, dtf, udot, !(S.fb_flag && S.fb_flag[id]));
				if (STAGE == 2) {
#pragma unroll
					for (int i = 0; i < 7; ++i) u[i] = (float)(Uout[i * N + id] * SC.is[SC.cls(i)]);
				}
			} else {
#pragma unroll
				for (int i = 0; i < 7; ++i) u[i] = load_u(Ubase, i * N + id, SC, i) + dtf * udot[i];
				bad |= !fix_cons(SP, u);
#pragma unroll
				for (int i = 0; i < 7; ++i) store_u(Uout, i * N + id, u[i], SC, i);
			}
			if (STAGE == 2) {
				// the next step's CFL limit from Q(U1) with floors (Torch::fullStep:
				// globalQfromU + fixPrimitives, then Hydrodynamics::calculateTimeStep)
				Prim q = prim_from_cons<CR>(u, gamma, nd);
				fix_prim(SP, q, u[DEN]);
				// velocities are in units of v0: inv_t = (|v| + c) v0 / dx
				double ss = sqrt(P.gamma * (double)q.p / (double)q.d);
				double inv_t = 0;
#pragma unroll
				for (int k = 0; k < 3; ++k)
					if (k < nd) inv_t += (fabs((double)q.v[k]) + ss) * P.f32_v0 / P.dx[k];
				if (inv_t == 0) inv_t = 1.0 / P.dt_max;
				tmin = dmin_(tmin, 0.5 / inv_t);
			}
		}
		if (nd > 2) {
#pragma unroll
			for (int i = 0; i < 7; ++i) fzlo[i] = fz[i];
		}
		szc = szn;
		// no barrier before this: only the slot of plane z is written, and the
		// flux and slope arrays are rewritten after the next barrier
		if (stage_next) plane_convert<STAGE>(P, SP, SC, raw, s, sc, smap, z + 3);
		s_z = s_z1;
	}
	if (bad) atomicOr(S.err, ERRB_NAN);
	if (tma_late) atomicOr(S.err, ERRB_ASYNC);
	if (STAGE == 2) {
		for (int o = 16; o > 0; o >>= 1) tmin = dmin_(tmin, __shfl_down_sync(0xffffffffu, tmin, o));
		if ((threadIdx.x & 31) == 0) {
			unsigned long long* slots = reinterpret_cast<unsigned long long*>(S.scal + 2);
			atomicMin(&slots[0], (unsigned long long)__double_as_longlong(tmin));
		}
	}
}

template <int STAGE, typename TS, int LIM, int RS>
__global__ void __launch_bounds__(BX* BY, 2)
    k_hydro_stage_fp32(Params P, State S, const TS* __restrict__ Uq, const TS* Ubase, TS* Uout, double hfac,
                       int zchunk, const __grid_constant__ CUtensorMap tmap, int use_tma) {
	hydro_stage_body<STAGE, TS, LIM, RS>(P, S, Uq, Ubase, Uout, hfac, zchunk, &tmap, use_tma, blockIdx.x, blockIdx.y,
	                                     blockIdx.z);
}

// Hydro sub-step of the FP32 form on the FP64 states of a batch of 2-D grids:
// one CTA per entry (grid, tile x, tile y) of the batch's tile table; each
// grid's U into its U1.
template <int LIM, int RS>
__global__ void __launch_bounds__(BX* BY, 2) k_hydro_substep_fp32_batch(const BatchTable* __restrict__ B, double hfac) {
	const BatchTile t = B->tiles[blockIdx.x];
	const Params& P = B->P[t.g];
	const State& S = B->S[t.g];
	hydro_stage_body<1, double, LIM, RS>(P, S, S.U, S.U, S.U1, hfac, 1, nullptr, 0, t.tx, t.ty, 0);
}
// Every grid's U1 into its U (the batch keeps each grid's U where its own
// context has it).
__global__ void __launch_bounds__(256) k_batch_u1_to_u(Params Pv) {
	const BatchTable& B = *Pv.batch;
	const long long pos = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	const int g = batch_slot(B.cell_off, B.G, blockIdx.x * (long long)blockDim.x);
	const long long id = pos - B.cell_off[g];
	const Params& P = B.P[g];
	if (id >= P.N) return;
	const State& S = B.S[g];
#pragma unroll
	for (int f = 0; f < 7; ++f) S.U[f * P.N + id] = S.U1[f * P.N + id];
}

void launch_hydro_substep_fp32_batch(const Params& Pv, const BatchTable* B, int ntiles, double h, cudaStream_t stream) {
	const size_t smem = hydro_stage_fp32_smem();
	const bool fast = Pv.limiter == 6 && Pv.riemann == RS_ROTATED;
	if (fast) {
		cudaFuncSetAttribute(k_hydro_substep_fp32_batch<6, RS_ROTATED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
		                     (int)smem);
		k_hydro_substep_fp32_batch<6, RS_ROTATED><<<ntiles, BX * BY, smem, stream>>>(B, h);
	} else {
		cudaFuncSetAttribute(k_hydro_substep_fp32_batch<-1, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
		                     (int)smem);
		k_hydro_substep_fp32_batch<-1, -1><<<ntiles, BX * BY, smem, stream>>>(B, h);
	}
	k_batch_u1_to_u<<<(unsigned)((Pv.N + 255) / 256), 256, 0, stream>>>(Pv);
}

size_t hydro_stage_fp32_smem() {
	// the staging buffer is sized for the FP64 state of the radiation-hydro
	// form, followed by the TMA copy's mbarrier
	return hydro_stage_raw_offset() + sizeof(double) * 7 * SX * SY + 16;
}

// Tensor map of an FP64 state [7][nz][ny][nx] for the TMA plane staging: a
// 4-D tensor (x, y, z, field), box SX x SY x 1 x 7.  False where the driver
// entry point is unavailable or the strides are not multiples of 16 bytes
// (odd nx): the kernel then stages with cp.async.
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled_fn() {
	static EncodeTiledFn fn = nullptr;
	static std::once_flag once;
	std::call_once(once, [] {
		void* p = nullptr;
		cudaDriverEntryPointQueryResult q;
		if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
		    q == cudaDriverEntryPointSuccess)
			fn = reinterpret_cast<EncodeTiledFn>(p);
	});
	return fn;
}
static bool state_tensor_map(const Params& P, const double* U, CUtensorMap* m) {
	EncodeTiledFn enc = encode_tiled_fn();
	if (!enc || P.nd != 3 || (P.nx & 1) || P.nx < SX || P.ny < SY) return false;
	const cuuint64_t dims[4] = {(cuuint64_t)P.nx, (cuuint64_t)P.ny, (cuuint64_t)P.nz, 7};
	const cuuint64_t strides[3] = {(cuuint64_t)P.nx * 8, (cuuint64_t)P.nx * P.ny * 8, (cuuint64_t)P.N * 8};
	const cuuint32_t box[4] = {SX, SY, 1, 7};
	const cuuint32_t estr[4] = {1, 1, 1, 1};
	return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double*>(U), dims, strides, box, estr,
	           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
	           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int STAGE, typename TS, int LIM, int RS>
static void launch_one(const Params& P, const State& S, const TS* Uq, const TS* Ubase, TS* Uout, double hfac,
                       int zchunk, cudaStream_t stream) {
	size_t smem = hydro_stage_fp32_smem();
	int zc = P.nd > 2 ? zchunk : 1;
	dim3 grid((P.nx + BX - 1) / BX, (P.ny + BY - 1) / BY, P.nd > 2 ? (P.nz + zc - 1) / zc : 1);
	CUtensorMap tmap;
	memset(&tmap, 0, sizeof(tmap));
	int use_tma = 0;
	if (sizeof(TS) == sizeof(double) && P.hydro_tma)
		use_tma = state_tensor_map(P, reinterpret_cast<const double*>(Uq), &tmap) ? 1 : 0;
	cudaFuncSetAttribute(k_hydro_stage_fp32<STAGE, TS, LIM, RS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                     (int)smem);
	k_hydro_stage_fp32<STAGE, TS, LIM, RS><<<grid, BX * BY, smem, stream>>>(P, S, Uq, Ubase, Uout, hfac, zc, tmap,
	                                                                         use_tma);
}

// the reference's configured and default pair (albada, RotatedHLLC) is compiled
// with both fixed; any other pair takes the run-time switches
void launch_hydro_stage_fp32(int stage, const Params& P, const State& S, const float* Uq, const float* Ubase,
                             float* Uout, int zchunk, cudaStream_t stream) {
	bool fast = P.limiter == 6 && P.riemann == RS_ROTATED;
	if (stage == 1) {
		if (fast) launch_one<1, float, 6, RS_ROTATED>(P, S, Uq, Ubase, Uout, 0.5, zchunk, stream);
		else launch_one<1, float, -1, -1>(P, S, Uq, Ubase, Uout, 0.5, zchunk, stream);
	} else {
		if (fast) launch_one<2, float, 6, RS_ROTATED>(P, S, Uq, Ubase, Uout, 1.0, zchunk, stream);
		else launch_one<2, float, -1, -1>(P, S, Uq, Ubase, Uout, 1.0, zchunk, stream);
	}
}

// Hydro sub-step of the operator split in the FP32 form, on the FP64 state:
// Uout = fix(U + h dt L(fixPrimitives(Q(U)))).
void launch_hydro_substep_fp32(const Params& P, const State& S, const double* U, double* Uout, double h, int zchunk,
                               cudaStream_t stream) {
	bool fast = P.limiter == 6 && P.riemann == RS_ROTATED;
	if (fast) launch_one<1, double, 6, RS_ROTATED>(P, S, U, U, Uout, h, zchunk, stream);
	else launch_one<1, double, -1, -1>(P, S, U, U, Uout, h, zchunk, stream);
}

// x-slab decomposition: the two x layers next to each PARTITION face of a
// slab, packed [side][layer][field][ny * nz] (layer 0 next to the face) for
// the neighbour, from the state the next flux computation reads (primitives
// of the FP64 form, the hydro-only FP32 state): what the reference's
// applyBCs sends for its partition ghost cells (Grid.cpp:804-833).
template <typename T>
__global__ void __launch_bounds__(256) k_halo_pack(Params P, const T* __restrict__ src, T* __restrict__ dst) {
	const long long nyz = (long long)P.ny * P.nz;
	const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (i >= 4LL * NU * nyz) return;
	const long long yz = i % nyz;
	const int f = (int)((i / nyz) % NU);
	const int sl = (int)(i / (NU * nyz));  // side * 2 + layer
	const int side = sl >> 1, layer = sl & 1;
	if ((side ? P.rbc[0] : P.lbc[0]) != BC_PARTITION) return;
	const int x = side ? P.nx - 1 - layer : layer;
	dst[i] = src[(long long)f * P.N + x + (long long)P.nx * yz];
}
void launch_halo_pack(const Params& P, const void* src, void* dst, bool f32, cudaStream_t stream) {
	const long long n = 4LL * NU * P.ny * P.nz;
	const unsigned g = (unsigned)((n + 255) / 256);
	if (f32) k_halo_pack<float><<<g, 256, 0, stream>>>(P, static_cast<const float*>(src), static_cast<float*>(dst));
	else k_halo_pack<double><<<g, 256, 0, stream>>>(P, static_cast<const double*>(src), static_cast<double*>(dst));
}

// x-slab decomposition with a star: the slab's boundary x layer next to each
// partition face, packed [side][ny * nz][4] for the neighbour on the far side
// from the star after a causal sweep - the four optical depths of a cell (R
// quad) or its COL_DEN, DCOL_DEN (T pair) - as the reference sends them after
// Radiation::transferRadiation and Thermodynamics::rayTrace
// (Radiation.cpp:614-635, Thermodynamics.cpp:398-416).
__global__ void __launch_bounds__(256) k_sweep_pack(Params P, const double* __restrict__ src, int colden,
                                                    double* __restrict__ dst) {
	const long long nyz = (long long)P.ny * P.nz;
	const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (i >= 2 * nyz) return;
	const int side = (int)(i / nyz);
	const long long yz = i - side * nyz;
	if ((side ? P.rbc[0] : P.lbc[0]) != BC_PARTITION) return;
	const long long id = (side ? P.nx - 1 : 0) + (long long)P.nx * yz;
	double2* d = reinterpret_cast<double2*>(dst + i * 4);
	if (colden) {
		d[0] = reinterpret_cast<const double2*>(src + id * 2)[0];
	} else {
		const double2* q = reinterpret_cast<const double2*>(src + id * 4);
		d[0] = q[0];
		d[1] = q[1];
	}
}
void launch_sweep_pack(const Params& P, const double* src, bool colden, double* dst, cudaStream_t stream) {
	const long long n = 2LL * P.ny * P.nz;
	k_sweep_pack<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(P, src, colden ? 1 : 0, dst);
}

// FP64 <-> FP32 state conversion (entry to / exit from the FP32 form), with
// the per-field reference values of the scaled units.
__device__ __forceinline__ double field_scale(const Params& P, int f) {
	if (f == PRE) return P.f32_p0;
	if (f >= VEL) return P.f32_rho0 * P.f32_v0;
	return P.f32_rho0;
}
__global__ void k_f64_to_f32(Params P, const double* __restrict__ a, float* __restrict__ b) {
	long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (i < 7 * P.N) b[i] = (float)(a[i] / field_scale(P, (int)(i / P.N)));
}
__global__ void k_f32_to_f64(Params P, const float* __restrict__ a, double* __restrict__ b) {
	long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (i < 7 * P.N) b[i] = (double)a[i] * field_scale(P, (int)(i / P.N));
}

}  // namespace trg
