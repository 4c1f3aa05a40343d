// FP64 kernels of the operator-split step.
//
// This file is compiled twice.  The exact build (namespace trg::exact, the
// plain-FP64 form) uses --fmad=false: every kernel reproduces the reference's
// FP64 arithmetic in the reference's operation order, and exp/log/log10/pow
// come from trg_math.h (correctly rounded, IEEE operations only, so they
// return the host glibc's results wherever glibc rounds correctly), which the
// CPU oracle shares, so that the GPU and CPU runs agree to the last bit.  The fast build
// (trg::fast, -DTRG_FAST_MATH, FMA contraction on) serves the FP32 form, whose
// radiation, cooling and time-step kernels stay FP64 but need not round like
// the reference.
//
// Layout: SoA, field-major, interior cells only, flat index i + nx*(j + ny*k).
// Ghost cells are not stored: boundary conditions are applied while loading
// (Grid::applyBCs, Grid.cpp:649-836, restated by map_ghost below).
#include "trg_device.cuh"
#include "trg_kernels.h"
#include "tc_mlp.cuh"

#ifndef TRG_KNS
#define TRG_KNS exact
#endif
// Batch dispatch (a kernel over the cells or shells of many grids): in the
// exact build (FP64-form batches) and in a third build, fast arithmetic with
// the dispatch (trg::fastb, FP32-form batches); the fast build of single
// grids leaves it out, which keeps its kernels' instruction footprint small.
#if defined(TRG_FAST_MATH) && !defined(TRG_FAST_BATCHED)
#define TRG_BATCHED false
#else
#define TRG_BATCHED true
#endif
namespace trg {
namespace TRG_KNS {

// ------------------------------------------------------------------ limiters
__device__ __forceinline__ double minmod(double a, double b) { return (a * b > 0) ? (fabs(a) < fabs(b) ? a : b) : 0; }
__device__ __forceinline__ double maxmod(double a, double b) { return (a * b > 0) ? (fabs(a) > fabs(b) ? a : b) : 0; }

// SlopeLimiter::calculate variants, SlopeLimiter.cpp:5-54.
__device__ __forceinline__ double limiter(int kind, double a, double b) {
	switch (kind) {
	case 0: return minmod((a + b) / 2.0, minmod(2.0 * a, 2.0 * b));
	case 1: return maxmod(minmod(b, 2.0 * a), minmod(2.0 * b, a));
	case 2: return minmod(a, b);
	case 3: return maxmod(a, b);
	case 4: {
		if (b == 0) return 0;
		double r = fabs(a / b);
		return (a + b * r) / (1.0 + r);
	}
	case 5: return (a * b <= 1.0e-30) ? 0 : 1.5 * b * (a * a + a * b) / (a * a + a * b + b * b);
	default: return a * b <= 1.0e-30 ? 0 : a * b * (a + b) / (a * a + b * b);
	}
}

// ----------------------------------------------------------- Riemann solvers
// characteristicWaveSpeeds (Einfeldt), Riemann.cpp:27-42.
__device__ __forceinline__ void wave_speeds(double a_l2, double a_r2, const double* Ql, const double* Qr, int dim,
                                            double& Sl, double& Sr) {
	double sqrtrho_l = sqrt(Ql[DEN]);
	double sqrtrho_r = sqrt(Qr[DEN]);
	double u_tilde = (sqrtrho_l * Ql[VEL + dim] + sqrtrho_r * Qr[VEL + dim]) / (sqrtrho_l + sqrtrho_r);
	double nu2 = 0.5 * sqrtrho_r * sqrtrho_l / ((sqrtrho_l + sqrtrho_r) * (sqrtrho_l + sqrtrho_r));
	double dsqrd = (sqrtrho_l * a_l2 + sqrtrho_r * a_r2) / (sqrtrho_l + sqrtrho_r);
	dsqrd += nu2 * (Qr[VEL + dim] - Ql[VEL + dim]) * (Qr[VEL + dim] - Ql[VEL + dim]);
	double d = sqrt(dsqrd);
	Sl = u_tilde - d;
	Sr = u_tilde + d;
}

// HartenLaxLeerContactSolver::solve, Riemann.cpp:52-104.
__device__ void hllc(double* F, const double* Ql, const double* Qr, double a_l2, double a_r2, double gamma, int nd, int dim) {
	double S_l, S_r;
	wave_speeds(a_l2, a_r2, Ql, Qr, dim, S_l, S_r);
	if (S_l >= 0) {
		FfromQ(F, Ql, gamma, nd, dim);
	} else if (S_r <= 0) {
		FfromQ(F, Qr, gamma, nd, dim);
	} else {
		double S_c = Qr[PRE] - Ql[PRE];
		S_c += Ql[DEN] * Ql[VEL + dim] * (S_l - Ql[VEL + dim]);
		S_c -= Qr[DEN] * Qr[VEL + dim] * (S_r - Qr[VEL + dim]);
		S_c /= (Ql[DEN] * (S_l - Ql[VEL + dim]) - Qr[DEN] * (S_r - Qr[VEL + dim]));
		const double* Qlr = (S_c >= 0) ? Ql : Qr;
		double S_lr = (S_c >= 0) ? S_l : S_r;
		double U_lr[7] = {0, 0, 0, 0, 0, 0, 0}, F_lr[7] = {0, 0, 0, 0, 0, 0, 0}, U_c[7] = {0, 0, 0, 0, 0, 0, 0};
		UfromQ(U_lr, Qlr, gamma, nd);
		FfromQ(F_lr, Qlr, gamma, nd, dim);
		double A_lr = Qlr[DEN] * (S_lr - Qlr[VEL + dim]) / (S_lr - S_c);
		U_c[DEN] = A_lr;
		#pragma unroll
		for (int id = 0; id < 3; ++id) if (id < nd) U_c[VEL + id] = A_lr * Qlr[VEL + id];
		U_c[VEL + dim] = A_lr * S_c;
		U_c[PRE] = A_lr * ((U_lr[PRE] / Qlr[DEN]) +
		                   (S_c - Qlr[VEL + dim]) * (S_c + Qlr[PRE] / (Qlr[DEN] * (S_lr - Qlr[VEL + dim]))));
		U_c[HII] = A_lr * Qlr[HII];
		U_c[ADV] = A_lr * Qlr[ADV];
		for (int i = 0; i < NU; ++i) F[i] = F_lr[i] + S_lr * (U_c[i] - U_lr[i]);
		if (nd < 3) F[VEL + 2] = 0;
		if (nd < 2) F[VEL + 1] = 0;
	}
}

// HartenLaxLeerSolver::solve, Riemann.cpp:108-140.
__device__ void hll(double* F, const double* Ql, const double* Qr, double a_l2, double a_r2, double gamma, int nd, int dim) {
	double S_l, S_r;
	wave_speeds(a_l2, a_r2, Ql, Qr, dim, S_l, S_r);
	if (S_r <= 0) {
		FfromQ(F, Qr, gamma, nd, dim);
	} else if (S_l >= 0) {
		FfromQ(F, Ql, gamma, nd, dim);
	} else {
		double U_l[7] = {0, 0, 0, 0, 0, 0, 0}, U_r[7] = {0, 0, 0, 0, 0, 0, 0};
		double F_l[7] = {0, 0, 0, 0, 0, 0, 0}, F_r[7] = {0, 0, 0, 0, 0, 0, 0};
		UfromQ(U_l, Ql, gamma, nd);
		UfromQ(U_r, Qr, gamma, nd);
		FfromQ(F_l, Ql, gamma, nd, dim);
		FfromQ(F_r, Qr, gamma, nd, dim);
		for (int i = 0; i < NU; ++i)
			F[i] = (S_r * F_l[i] - S_l * F_r[i] + S_l * S_r * (U_r[i] - U_l[i])) / (S_r - S_l);
	}
}

// 3-vector helpers with the reduction order of the reference's vendored
// Eigen 3.2.1 (x + (y + z) for dot/norm; v /= s multiplies by 1/s; matrix
// coefficients accumulate (a + b) + c).
__device__ __forceinline__ void cross3(const double* a, const double* b, double* r) {
	r[0] = a[1] * b[2] - a[2] * b[1];
	r[1] = a[2] * b[0] - a[0] * b[2];
	r[2] = a[0] * b[1] - a[1] * b[0];
}
__device__ __forceinline__ double dot3(const double* a, const double* b) { return a[0] * b[0] + (a[1] * b[1] + a[2] * b[2]); }
__device__ __forceinline__ double norm3(const double* a) { return sqrt(dot3(a, a)); }
__device__ __forceinline__ void normalize3(double* a) {
	double r = 1.0 / norm3(a);
	a[0] *= r; a[1] *= r; a[2] *= r;
}

// getRotationFromA2B, Riemann.cpp:161-171 (Rodrigues: I + [v]x + (1-c)/s^2 [v]x^2).
__device__ __forceinline__ void rotation_a2b(const double* A, const double* B, double R[3][3]) {
	double v[3];
	cross3(A, B, v);
	double s = norm3(v);
	double cc = dot3(A, B);
	double vx[3][3] = {{0, -v[2], v[1]}, {v[2], 0, -v[0]}, {-v[1], v[0], 0}};
	double k = (1.0 - cc) / (s * s);
	double kvx[3][3];
#pragma unroll
	for (int i = 0; i < 3; ++i)
#pragma unroll
		for (int j = 0; j < 3; ++j) kvx[i][j] = k * vx[i][j];
#pragma unroll
	for (int i = 0; i < 3; ++i)
#pragma unroll
		for (int j = 0; j < 3; ++j) {
			double prod = kvx[i][0] * vx[0][j] + kvx[i][1] * vx[1][j] + kvx[i][2] * vx[2][j];
			R[i][j] = ((i == j ? 1.0 : 0.0) + vx[i][j]) + prod;
		}
}

// rotate, Riemann.cpp:154-159.
__device__ __forceinline__ void rotate(const double R[3][3], double* v) {
	double x = v[VEL + 0], y = v[VEL + 1], z = v[VEL + 2];
#pragma unroll
	for (int i = 0; i < 3; ++i) v[VEL + i] = R[i][0] * x + R[i][1] * y + R[i][2] * z;
}

// RotatedHartenLaxLeerSolver::solve (Nishikawa & Kitamura 2008), Riemann.cpp:181-244.
__device__ void rotated_hllc(double* F, const double* Ql, const double* Qr, double a_l2, double a_r2, double gamma, int nd,
                             int dim) {
	bool pureHLLC = false, pureHLL = false;
	double d[3] = {dim == 0 ? 1.0 : 0.0, dim == 1 ? 1.0 : 0.0, dim == 2 ? 1.0 : 0.0};
	double n1[3] = {Qr[VEL + 0] - Ql[VEL + 0], Qr[VEL + 1] - Ql[VEL + 1], Qr[VEL + 2] - Ql[VEL + 2]};
	double n2[3] = {0, 0, 0}, t[3];
	if (n1[dim] < 0)
		for (int i = 0; i < 3; ++i) n1[i] = -1.0 * n1[i];
	if (norm3(n1) < 1.0e-6)
		pureHLLC = true;
	else {
		normalize3(n1);
		cross3(n1, d, t);
		if (norm3(t) == 0)
			pureHLL = true;
		else {
			cross3(t, n1, n2);
			if (norm3(n2) == 0)
				pureHLL = true;
			else {
				if (n2[dim] < 0)
					for (int i = 0; i < 3; ++i) n2[i] = -1.0 * n2[i];
				normalize3(n2);
				cross3(n2, d, t);
				if (norm3(t) == 0) pureHLLC = true;
			}
		}
	}
	if (!pureHLLC && !pureHLL) {
		double F1[7] = {0, 0, 0, 0, 0, 0, 0}, F2[7] = {0, 0, 0, 0, 0, 0, 0};
		double QlR[7], QrR[7], Rm[3][3];
		for (int i = 0; i < NU; ++i) { QlR[i] = Ql[i]; QrR[i] = Qr[i]; }
		rotation_a2b(n1, d, Rm);
		rotate(Rm, QlR);
		rotate(Rm, QrR);
		hll(F1, QlR, QrR, a_l2, a_r2, gamma, nd, dim);
		rotation_a2b(d, n1, Rm);
		rotate(Rm, QlR);
		rotate(Rm, QrR);
		rotate(Rm, F1);
		rotation_a2b(n2, d, Rm);
		rotate(Rm, QlR);
		rotate(Rm, QrR);
		hllc(F2, QlR, QrR, a_l2, a_r2, gamma, nd, dim);
		rotation_a2b(d, n2, Rm);
		rotate(Rm, F2);
		double w1 = fabs(dot3(d, n1)), w2 = fabs(dot3(d, n2));
		for (int iu = 0; iu < NU; ++iu) F[iu] = w1 * F1[iu] + w2 * F2[iu];
	} else if (pureHLL)
		hll(F, Ql, Qr, a_l2, a_r2, gamma, nd, dim);
	else
		hllc(F, Ql, Qr, a_l2, a_r2, gamma, nd, dim);
}

// ------------------------------------------------------------- hydro faces
// Ghost position p (< 0 or >= n) along dim -> interior source index and the
// velocity rule of Grid::applyBCs (Grid.cpp:649-836).  Layer k = 1 is adjacent.
// A PARTITION face (x-slab decomposition) takes ghost layer k from the
// neighbour's halo, S.halo_recv [side][k - 1][field][ny * nz], as the
// reference's ghost cells take the neighbour's Q (Grid.cpp:804-833).
__device__ __forceinline__ void load_line(const Params& P, const double* __restrict__ Q, const void* halo,
                                          long long base, long long stride, int n, int dim, int pos, double* q) {
	int src = pos, cond = -1, side = 0;
	if (pos < 0) {
		int k = -pos;
		cond = P.lbc[dim];
		src = cond == BC_PERIODIC ? n - k : (cond == BC_REFLECTING ? k : 0);
	} else if (pos >= n) {
		int k = pos - n + 1;
		cond = P.rbc[dim];
		side = 1;
		src = cond == BC_PERIODIC ? k - 1 : (cond == BC_REFLECTING ? n - 1 - k : n - 1);
	}
	if (cond == BC_PARTITION) {  // x faces only: base = (j + ny k) nx
		const long long nyz = (long long)P.ny * P.nz, trans = base / P.nx;
		const int layer = (side ? pos - n + 1 : -pos) - 1;
		const double* h = static_cast<const double*>(halo) + (long long)(side * 2 + layer) * NU * nyz + trans;
#pragma unroll
		for (int f = 0; f < NU; ++f) q[f] = h[(long long)f * nyz];
		return;
	}
	long long id = base + (long long)src * stride;
#pragma unroll
	for (int f = 0; f < NU; ++f) q[f] = __ldg(&Q[(long long)f * P.N + id]);
	if (cond >= 0) {
		double v = q[VEL + dim];
		if (cond == BC_INFLOW) {
			if (side == 0 ? v < 0 : v > 0) q[VEL + dim] = -1.0 * v;
		} else if (cond == BC_OUTFLOW) {
			if (side == 0 ? v > 0 : v < 0) q[VEL + dim] = -1.0 * v;
		} else if (cond == BC_REFLECTING) {
			q[VEL + dim] = -v;
		}
	}
}

// Hydrodynamics::calcFluxes (Hydro.cpp:91-115) with the reconstruction of
// Hydro.cpp:44-67: one thread per face along dim; face f lies between line
// positions f-1 and f.
__device__ __forceinline__ void b_faces_fp64(const Params& P, const State& S, long long t, int dim);
__global__ void __launch_bounds__(128) k_faces_fp64(Params P, State S, int dim) {
	if (TRG_BATCHED && P.batch) {
		const BatchTable& B = *P.batch;
		const long long* off = B.face_off[dim];
		const int g = batch_slot(off, B.G, blockIdx.x * (long long)blockDim.x);
		const long long lt = blockIdx.x * (long long)blockDim.x + threadIdx.x - off[g];
		if (lt < B.S[g].nfaces[dim]) b_faces_fp64(B.P[g], B.S[g], lt, dim);
		return;
	}
	const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (t >= S.nfaces[dim]) return;
	b_faces_fp64(P, S, t, dim);
}
__device__ __forceinline__ void b_faces_fp64(const Params& P, const State& S, long long t, int dim) {
	int n = ncell(P, dim), f;
	long long base, stride;
	if (dim == 0) {
		f = (int)(t % (n + 1));
		long long rest = t / (n + 1);
		base = rest * P.nx;
		stride = 1;
	} else if (dim == 1) {
		int i = (int)(t % P.nx);
		long long rest = t / P.nx;
		f = (int)(rest % (n + 1));
		long long k = rest / (n + 1);
		base = i + (long long)P.nx * P.ny * k;
		stride = P.nx;
	} else {
		long long plane = (long long)P.nx * P.ny;
		f = (int)(t / plane);
		base = t % plane;
		stride = plane;
	}
	double Ls[7], Rs[7], Fv[7];
	if (P.order == 1) {
		double a[7], b[7], c[7], e[7];
		load_line(P, S.Q, S.halo_recv, base, stride, n, dim, f - 2, a);
		load_line(P, S.Q, S.halo_recv, base, stride, n, dim, f - 1, b);
		load_line(P, S.Q, S.halo_recv, base, stride, n, dim, f, c);
		load_line(P, S.Q, S.halo_recv, base, stride, n, dim, f + 1, e);
#pragma unroll
		for (int iq = 0; iq < NU; ++iq) {
			// QR of the cell at f-1 and QL of the cell at f (Hydro.cpp:44-50)
			double sl = limiter(P.limiter, b[iq] - a[iq], c[iq] - b[iq]);
			Ls[iq] = b[iq] + 0.5 * sl;
			double sr = limiter(P.limiter, c[iq] - b[iq], e[iq] - c[iq]);
			Rs[iq] = c[iq] - 0.5 * sr;
		}
	} else {
		load_line(P, S.Q, S.halo_recv, base, stride, n, dim, f - 1, Ls);
		load_line(P, S.Q, S.halo_recv, base, stride, n, dim, f, Rs);
	}
	double a_l2 = P.gamma * Ls[PRE] / Ls[DEN];
	double a_r2 = P.gamma * Rs[PRE] / Rs[DEN];
#pragma unroll
	for (int i = 0; i < NU; ++i) Fv[i] = 0;
	if (P.riemann == RS_HLLC) hllc(Fv, Ls, Rs, a_l2, a_r2, P.gamma, P.nd, dim);
	else if (P.riemann == RS_HLL) hll(Fv, Ls, Rs, a_l2, a_r2, P.gamma, P.nd, dim);
	else rotated_hllc(Fv, Ls, Rs, a_l2, a_r2, P.gamma, P.nd, dim);
	if (Fv[HII] != Fv[HII]) atomicOr(S.err, ERRB_FLUX);
	double* Fd = S.F[dim];
	long long nf = S.nfaces[dim];
#pragma unroll
	for (int i = 0; i < NU; ++i) Fd[(long long)i * nf + t] = Fv[i];
}

__device__ __forceinline__ void face_ids(const Params& P, const int* ijk, int dim, long long& l, long long& r) {
	if (dim == 0) {
		l = ijk[0] + (long long)(P.nx + 1) * (ijk[1] + (long long)P.ny * ijk[2]);
		r = l + 1;
	} else if (dim == 1) {
		l = ijk[0] + (long long)P.nx * (ijk[1] + (long long)(P.ny + 1) * ijk[2]);
		r = l + P.nx;
	} else {
		l = ijk[0] + (long long)P.nx * (ijk[1] + (long long)P.ny * ijk[2]);
		r = l + (long long)P.nx * P.ny;
	}
}

// Hydrodynamics::updateSourceTerms (Hydro.cpp:117-156) with
// Star::injectEnergyMomentum (Star.cpp:57-68) into udot[7].
__device__ __forceinline__ void hydro_udot(const Params& P, const State& S, long long id, const int* ijk, const double* xc,
                                           const double* Ubase, double* udot) {
	double vol = cell_volume(P, xc[0]);
#pragma unroll
	for (int i = 0; i < NU; ++i) udot[i] = 0;
	#pragma unroll
	for (int dim = 0; dim < 3; ++dim) if (dim < P.nd) {
		long long fl, fr;
		face_ids(P, ijk, dim, fl, fr);
		double al = face_area(P, xc, dim, 0), ar = face_area(P, xc, dim, 1);
		const double* Fd = S.F[dim];
		long long nf = S.nfaces[dim];
#pragma unroll
		for (int i = 0; i < NU; ++i) {
			udot[i] += (al / vol) * Fd[(long long)i * nf + fl];
			udot[i] -= (ar / vol) * Fd[(long long)i * nf + fr];
		}
	}
	for (int i = 0; i < 3; ++i) {
		double g = S.grav ? S.grav[(long long)i * P.N + id] : 0.0;
		udot[VEL + i] += g;
		udot[PRE] += FLD(S.Q, VEL + i, id) * g;
	}
	if (P.geometry == G_CYL) {
		double r = P.dx[0] * xc[0];
		udot[VEL + 0] += FLD(S.Q, PRE, id) / r;
	} else if (P.geometry == G_SPH) {
		double area1 = face_area(P, xc, 0, 1), area2 = face_area(P, xc, 0, 0);
		double r = vol / (area1 - area2);
		udot[VEL + 0] += FLD(S.Q, PRE, id) / r;
	}
	if (P.star_on && P.mdot != 0 && is_wind(P, id, ijk, xc)) {
		udot[DEN] += P.mdot;
		udot[PRE] += P.edot;
		udot[HII] += (FLD(Ubase, HII, id) / FLD(Ubase, DEN, id)) * P.mdot;
		udot[ADV] += P.mdot;
	}
}

// globalQfromU + fixPrimitives + checkValues of a cell whose new conserved
// state u the caller has in registers (the FP32 form's updates finish with
// it, so that the next sub-step's Q pass is skipped).  Q fields of velocity
// components beyond nd are left as they are, as QfromU leaves them.
__device__ __forceinline__ void store_fixed_q(const Params& P, const State& S, long long id, const double* u) {
	double q[7] = {0, 0, 0, 0, 0, 0, 0};
	QfromU(q, u, P.gamma, P.nd);
	fix_primitives(P, q, u[DEN]);
	bool bad = q[DEN] == 0 || q[PRE] == 0;
#pragma unroll
	for (int i = 0; i < NU; ++i) bad |= (u[i] != u[i]) || isinf(u[i]);
	FLD(S.Q, DEN, id) = q[DEN];
	FLD(S.Q, PRE, id) = q[PRE];
	FLD(S.Q, HII, id) = q[HII];
	FLD(S.Q, ADV, id) = q[ADV];
#pragma unroll
	for (int k = 0; k < 3; ++k)
		if (k < P.nd) FLD(S.Q, VEL + k, id) = q[VEL + k];
	if (bad) atomicOr(S.err, ERRB_NAN);
}

// Hydro update: UDOT from the face fluxes, then Fluid::advSolution (Fluid.cpp:80-87)
// from Ubase and Fluid::fixSolution, written to Uout (may alias Ubase); the
// selectors pick S.U (0) or S.U1 (1).
// mode 1 accumulates UDOT into S.UDOT instead (component-phase interface).
__device__ __forceinline__ void b_hydro_update_fp64(const Params& P, const State& S, long long id, double h, int sel_base,
                                                    int sel_out, int mode) {
	const double* Ubase = sel_base ? S.U1 : S.U;
	double* Uout = sel_out ? S.U1 : S.U;
	int ijk[3];
	double xc[3], udot[7];
	cell_ijk(P, id, ijk);
	cell_xc(P, ijk, xc);
	hydro_udot(P, S, id, ijk, xc, Ubase, udot);
	if (mode == 1) {
		for (int i = 0; i < NU; ++i) FLD(S.UDOT, i, id) += udot[i];
		return;
	}
	double dt = h * S.scal[0];
	double u[7];
#pragma unroll
	for (int i = 0; i < NU; ++i) u[i] = FLD(Ubase, i, id) + dt * udot[i];
	if (!fix_solution(P, u)) atomicOr(S.err, ERRB_NAN);
#pragma unroll
	for (int i = 0; i < NU; ++i) FLD(Uout, i, id) = u[i];
	if (mode == 2) store_fixed_q(P, S, id, u);
}
__global__ void __launch_bounds__(256) k_hydro_update_fp64(Params P, State S, double h, int sel_base, int sel_out,
                                                          int mode) {
	if (TRG_BATCHED && P.batch) {
		const BatchTable& B = *P.batch;
		const int g = batch_slot(B.cell_off, B.G, blockIdx.x * (long long)blockDim.x);
		const long long lid = blockIdx.x * (long long)blockDim.x + threadIdx.x - B.cell_off[g];
		if (lid < B.P[g].N) b_hydro_update_fp64(B.P[g], B.S[g], lid, h, sel_base, sel_out, mode);
		return;
	}
	const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (id >= P.N) return;
	b_hydro_update_fp64(P, S, id, h, sel_base, sel_out, mode);
}

// Fluid::globalQfromU (+ fixPrimitives), Fluid.cpp:138-165, with the Q half of
// Torch::checkValues (Torch.cpp:420-443).
__device__ __forceinline__ void b_q_from_u_fp64(const Params& P, const State& S, long long id, int sel_src, int fix) {
	const double* Usrc = sel_src ? S.U1 : S.U;
	double u[7], q[7];
#pragma unroll
	for (int i = 0; i < NU; ++i) { u[i] = FLD(Usrc, i, id); q[i] = FLD(S.Q, i, id); }
	QfromU(q, u, P.gamma, P.nd);
	bool bad = false;
	if (fix) {
		// Torch::checkValues runs where Q was just rebuilt with floors; the
		// RK2 predictor's Q(U*) (fix == 0) is not checked by the reference.
		fix_primitives(P, q, u[DEN]);
		bad = q[DEN] == 0 || q[PRE] == 0;
#pragma unroll
		for (int i = 0; i < NU; ++i) bad |= (u[i] != u[i]) || isinf(u[i]);
	}
#pragma unroll
	for (int i = 0; i < NU; ++i) FLD(S.Q, i, id) = q[i];
	if (bad) atomicOr(S.err, ERRB_NAN);
}
__global__ void __launch_bounds__(256) k_q_from_u_fp64(Params P, State S, int sel_src, int fix) {
	if (TRG_BATCHED && P.batch) {
		const BatchTable& B = *P.batch;
		const int g = batch_slot(B.cell_off, B.G, blockIdx.x * (long long)blockDim.x);
		const long long lid = blockIdx.x * (long long)blockDim.x + threadIdx.x - B.cell_off[g];
		if (lid < B.P[g].N) b_q_from_u_fp64(B.P[g], B.S[g], lid, sel_src, fix);
		return;
	}
	const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (id >= P.N) return;
	b_q_from_u_fp64(P, S, id, sel_src, fix);
}

// advSolution(dt) + fixSolution over the UDOT array (component-phase interface).
__device__ __forceinline__ void b_advance_fp64(const Params& P, const State& S, long long id, double dt) {

	double u[7];
	for (int i = 0; i < NU; ++i) {
		u[i] = FLD(S.U, i, id) + dt * FLD(S.UDOT, i, id);
		FLD(S.UDOT, i, id) = 0;
	}
	if (!fix_solution(P, u)) atomicOr(S.err, ERRB_NAN);
	for (int i = 0; i < NU; ++i) FLD(S.U, i, id) = u[i];
}
__global__ void __launch_bounds__(256) k_advance_fp64(Params P, State S, double dt) {
	if (TRG_BATCHED && P.batch) {
		const BatchTable& B = *P.batch;
		const int g = batch_slot(B.cell_off, B.G, blockIdx.x * (long long)blockDim.x);
		const long long lid = blockIdx.x * (long long)blockDim.x + threadIdx.x - B.cell_off[g];
		if (lid < B.P[g].N) b_advance_fp64(B.P[g], B.S[g], lid, dt);
		return;
	}
	const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (id >= P.N) return;
	b_advance_fp64(P, S, id, dt);
}

// ------------------------------------------------------------------ radiation
// Radiation.cpp:243-251.
// emT = exp(-T), passed in where T is fixed across calls.  Beyond the
// ionisation front exp(-T) underflows to 0 (T >= 750 in both builds' exp),
// and then the rate is exactly +0 whatever delT: the second exponential is
// skipped (a NaN delT still propagates).
__device__ __forceinline__ double photoionisation_rate_e(double nHI, double emT, double delT, double shellVol,
                                                         double photonRate) {
	if (nHI == 0 || shellVol == 0) return 0.0;
	if (emT == 0 && delT == delT) return 0.0;
	double emdT = d_exp(-delT);
	return photonRate * emT * (1.0 - emdT) / (nHI * shellVol);
}
__device__ __forceinline__ double photoionisation_rate(double nHI, double T, double delT, double shellVol, double photonRate) {
	if (nHI == 0 || shellVol == 0) return 0.0;
	if (T >= 750.0 && delT == delT) return 0.0;
	return photoionisation_rate_e(nHI, d_exp(-T), delT, shellVol, photonRate);
}

// Voronov (1997) fit, Radiation.cpp:231-237.
__device__ __forceinline__ double collisional_ionisation_rate(const Params& P, double T) {
	if (!P.collisions_on || T < 5.0e3) return 0.0;
	double U = P.voronov_DE / T;
	return P.voronov_A * (1. + P.voronov_P * sqrt(U)) * d_exp(P.voronov_K * d_log(U) - U) / (P.voronov_X + U);
}

// Radiation::doric, Radiation.cpp:140-179.
__device__ __forceinline__ void doric(double dt, double& HII_avg, double& HII, double Api, double nHII_aB, double nHII_Aci) {
	double xeq, inv_ti, epsilon = 1.0e-8;
	double HII_old = HII;
	inv_ti = Api + nHII_Aci + nHII_aB;
#ifdef TRG_FAST_MATH
	// one division, 1 / (dt / t_i), for xeq and the time average (when
	// dt / t_i < 1e-8 neither is used)
	const double ti_dt = 1.0 / (dt * inv_ti);
	if (nHII_aB == 0.0) xeq = 1.0;
	else xeq = (Api + nHII_Aci) * (ti_dt * dt);
#else
	if (nHII_aB == 0.0) xeq = 1.0;
	else xeq = (Api + nHII_Aci) / (Api + nHII_Aci + nHII_aB);
#endif
	if (dt * inv_ti < 1.0e-8) {
		HII = HII_old;
		HII = smax(smin(HII, 1.0), 0.0);
		if (1.0 - HII < epsilon) HII = 1.0 - epsilon;
		HII_avg = HII;
	} else {
		double e = d_exp(-dt * inv_ti);
		HII = xeq + (HII_old - xeq) * e;
		HII = smax(smin(HII, 1.0), 0.0);
		if (1.0 - HII < epsilon) HII = 1.0 - epsilon;
#ifdef TRG_FAST_MATH
		HII_avg = xeq + (HII_old - xeq) * (1.0 - e) * ti_dt;
#else
		HII_avg = xeq + (HII_old - xeq) * (1.0 - e) / (dt * inv_ti);
#endif
		HII_avg = smax(smin(HII_avg, 1.0), 0.0);
		if (1.0 - HII_avg < epsilon) HII_avg = 1.0 - epsilon;
	}
}

__device__ __forceinline__ double pick3(double a0, double a1, double a2, int k) { return k == 0 ? a0 : (k == 1 ? a1 : a2); }

// C2-Ray upwind neighbours and weights (Grid::calculateNearestNeighbours,
// Grid.cpp:922-952) computed on the fly.  A neighbour outside the interior
// (a ghost cell or none in the reference) contributes zero optical depth and
// is returned as -1.  In an x slab, a neighbour one layer beyond a partition
// face is the reference's partition ghost cell (reached through the grid
// joins, Grid.cpp:936-943), which holds the star-side neighbour's boundary
// layer as received before the sweep (Radiation.cpp:578-588,
// Thermodynamics.cpp:372-380): it is returned as -2 - (side ny nz + j + ny k),
// its index into S.sweep_recv.
// The rotated frame (irot) is resolved with selects rather than indexed
// arrays, so that everything stays in registers.
__device__ __forceinline__ void neighbours(const Params& P, const int* ijk, const double* xc, long long* nb, double* w) {
	int plane = 0;
	double dmax = 0;
#pragma unroll
	for (int i = 0; i < 3; ++i)
		if (i < P.nd) {
			double dd = fabs(xc[i] - P.sxc[i]);
			if (dd > dmax) { dmax = dd; plane = i; }
		}
	// irot = {(plane + 1) % 3, (plane + 2) % 3, plane}
	const int r0 = plane == 2 ? 0 : plane + 1, r1 = plane == 0 ? 2 : plane - 1, r2 = plane;
	const double x0 = pick3(xc[0], xc[1], xc[2], r0), x1 = pick3(xc[0], xc[1], xc[2], r1);
	const double d0 = x0 - pick3(P.sxc[0], P.sxc[1], P.sxc[2], r0);
	const double d1 = x1 - pick3(P.sxc[0], P.sxc[1], P.sxc[2], r1);
	const double d2 = pick3(xc[0], xc[1], xc[2], r2) - pick3(P.sxc[0], P.sxc[1], P.sxc[2], r2);
	const int s0 = d0 < -1.0 / 10.0 ? -1 : 1, s1 = d1 < -1.0 / 10.0 ? -1 : 1, s2 = d2 < -1.0 / 10.0 ? -1 : 1;
	const int L0 = fabs(d0) < 1.0 / 10.0 ? 0 : s0, L1 = fabs(d1) < 1.0 / 10.0 ? 0 : s1, L2 = fabs(d2) < 1.0 / 10.0 ? 0 : s2;
	// offsets in the rotated frame: n = 0: (0, 0, -L2), 1: (0, -L1, -L2), 2: (-L0, 0, -L2), 3: (-L0, -L1, -L2)
	const bool slab = P.lbc[0] == BC_PARTITION || P.rbc[0] == BC_PARTITION;  // the same for every thread
#pragma unroll
	for (int n = 0; n < 4; ++n) {
		const int o0 = (n & 2) ? -L0 : 0, o1 = (n & 1) ? -L1 : 0, o2 = -L2;
		const int ti = ijk[0] + (r0 == 0 ? o0 : 0) + (r1 == 0 ? o1 : 0) + (r2 == 0 ? o2 : 0);
		const int tj = ijk[1] + (r0 == 1 ? o0 : 0) + (r1 == 1 ? o1 : 0) + (r2 == 1 ? o2 : 0);
		const int tk = ijk[2] + (r0 == 2 ? o0 : 0) + (r1 == 2 ? o1 : 0) + (r2 == 2 ? o2 : 0);
		const bool yz = tj >= 0 && tj < P.ny && tk >= 0 && tk < P.nz;
		const bool in = ti >= 0 && ti < P.nx && yz;
		nb[n] = in ? flat_id(P, ti, tj, tk) : -1;
		if (slab && !in && yz &&
		    ((ti == -1 && P.lbc[0] == BC_PARTITION) || (ti == P.nx && P.rbc[0] == BC_PARTITION)))
			nb[n] = -2 - ((ti < 0 ? 0 : (long long)P.ny * P.nz) + tj + (long long)P.ny * tk);
	}
	double ic0 = (int)x0 - 0.5 * (s2 * d0 / d2);
	double ic1 = (int)x1 - 0.5 * (s2 * d1 / d2);
	double delta0 = fabs(2.0 * ic0 - 2.0 * (int)x0 + s0);
	double delta1 = fabs(2.0 * ic1 - 2.0 * (int)x1 + s1);
	w[0] = (fabs(d2) > 0.9) ? delta0 * delta1 : 0;
	w[1] = ((fabs(d1) > 0.9) && (fabs(d2) > 0.9)) ? delta0 * (1.0 - delta1) : 0;
	w[2] = ((fabs(d0) > 0.9) && (fabs(d2) > 0.9)) ? (1.0 - delta0) * delta1 : 0;
	w[3] = ((fabs(d0) > 0.9) && (fabs(d1) > 0.9) && (fabs(d2) > 0.9)) ? (1.0 - delta0) * (1.0 - delta1) : 0;
}

__device__ __forceinline__ double dist2_cells(const Params& P, const double* xc) {
	double d2 = 0;
	#pragma unroll
	for (int i = 0; i < 3; ++i) if (i < P.nd) d2 += (xc[i] - P.sxc[i]) * (xc[i] - P.sxc[i]);
	return d2;
}

// Programmatic dependent launch.  The shells of a sweep after the first are
// launched with programmatic stream serialisation, so that a shell's CTAs can
// start while the previous shell still runs.  What a shell kernel does before
// sweep_wait() reads only fields of its own cells that no shell of the sweep
// writes (density, pressure, fractions, path lengths, volumes) and the rate
// tables; sweep_wait() returns once the previous shell has completed and its
// writes are visible (at once when the launch had no such dependency).  Each
// shell lets the next one launch only after its own wait, so at most two
// shells are resident at a time.
__device__ __forceinline__ void sweep_wait() {
	asm volatile("griddepcontrol.wait;" ::: "memory");
	asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Radiation::updateTauSC, Radiation.cpp:353-373: the weighted interpolation of
// the inner neighbours' optical depths tau[i] (zero where not read).
__device__ __forceinline__ double tau_interp(const Params& P, const double* tau, const double* w0) {
#ifdef TRG_FAST_MATH
	// sum(w0 tau / m) / sum(w0 / m), m = max(tau0, tau), with numerator and
	// denominator multiplied by the product of the four m: one division (the
	// weights w0 of an inner cell sum to 1, so the denominator is positive).
	// Optical depths large enough for the product to overflow take the
	// per-neighbour divisions.
	double m[4];
	for (int i = 0; i < 4; ++i) m[i] = smax(P.tau0, tau[i]);
	const double m01 = m[0] * m[1], m23 = m[2] * m[3];
	if (m01 * m23 < 1.0e300) {
		const double p0 = m[1] * m23, p1 = m[0] * m23, p2 = m[3] * m01, p3 = m[2] * m01;
		const double num = w0[0] * p0 * tau[0] + w0[1] * p1 * tau[1] + w0[2] * p2 * tau[2] + w0[3] * p3 * tau[3];
		const double den = w0[0] * p0 + w0[1] * p1 + w0[2] * p2 + w0[3] * p3;
		return num / den;
	}
#endif
	double w[4];
	for (int i = 0; i < 4; ++i) w[i] = w0[i] / smax(P.tau0, tau[i]);
	double sum_w = w[0] + w[1] + w[2] + w[3];
#ifdef TRG_FAST_MATH
	double num = 0.0;
	for (int i = 0; i < 4; ++i) num += w[i] * tau[i];
	return num / sum_w;
#else
	double newtau = 0.0;
	for (int i = 0; i < 4; ++i) {
		w[i] = w[i] / sum_w;
		newtau += w[i] * tau[i];
	}
	return newtau;
#endif
}
// Where the inner neighbours' optical depths (R quads, STRIDE 4) or column
// densities (T pairs, STRIDE 2) are read, resolved before the sweep's wait so
// that no address arithmetic sits between the wait and the loads: null where
// a neighbour is not read (outside the grid, or of zero weight: it
// contributes 0 * tau = 0 whatever its tau, and may belong to the shell being
// swept); across a slab's partition face, its entry of the received boundary
// layer (4 doubles per cell).  A slab whose layer was never exchanged (a
// sweep outside the exchange, which the host does not launch) reports
// ERRB_SLAB and reads nothing.  Neighbour values written by the previous
// shell are read past L1, one 16-byte pair at a time.
template <int STRIDE>
__device__ __forceinline__ void nb_sources(const State& S, const double* base, const long long* nb, const double* w0,
                                           const double2** src) {
#pragma unroll
	for (int i = 0; i < 4; ++i) {
		src[i] = nullptr;
		if (w0[i] == 0 || nb[i] == -1) continue;
		if (nb[i] >= 0) src[i] = reinterpret_cast<const double2*>(base + nb[i] * STRIDE);
		else if (S.sweep_recv) src[i] = reinterpret_cast<const double2*>(S.sweep_recv + (-2 - nb[i]) * 4);
		else atomicOr(S.err, ERRB_SLAB);
	}
}
// TAU (from TAU + DTAU of the neighbours)
__device__ __forceinline__ double tau_sc(const Params& P, const double2* const* src, const double* w0) {
	double tau[4] = {0, 0, 0, 0};
	for (int i = 0; i < 4; ++i)
		if (src[i]) {
			const double2 a = __ldcg(src[i]);
			tau[i] = a.x + a.y;
		}
	return tau_interp(P, tau, w0);
}
// TAU and TAU_A together (each neighbour's four optical depths share a sector)
__device__ __forceinline__ void tau_sc2(const Params& P, const double2* const* src, const double* w0,
                                        double& tau_out, double& tau_a_out) {
	double tau[4] = {0, 0, 0, 0}, tau_a[4] = {0, 0, 0, 0};
	for (int i = 0; i < 4; ++i)
		if (src[i]) {
			const double2 a = __ldcg(src[i]), b = __ldcg(src[i] + 1);
			tau[i] = a.x + a.y;
			tau_a[i] = b.x + b.y;
		}
	tau_out = tau_interp(P, tau, w0);
	tau_a_out = tau_interp(P, tau_a, w0);
}
// All four optical depths of a cell in one store.
__device__ __forceinline__ void store_taus(const State& S, long long id, double tau, double dtau, double tau_a,
                                           double dtau_a) {
	double2* q = reinterpret_cast<double2*>(S.R + id * 4);
	q[0] = make_double2(tau, dtau);
	q[1] = make_double2(tau_a, dtau_a);
}

// Wind cells of Radiation::transferRadiation, Radiation.cpp:590-598.
__device__ __forceinline__ void b_rad_wind_reset(const Params& P, const State& S, long long id) {
	store_taus(S, id, 0, 0, 0, 0);
	FLD(S.Q, HII, id) = 1;
	RFLD(S.R, R_HII_A, id) = 1;
}
__global__ void k_rad_wind_reset(Params P, State S, const int* __restrict__ cells, int count) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= count) return;
	if (TRG_BATCHED && P.batch) {
		const int e = cells[t];
		b_rad_wind_reset(P.batch->P[e >> BATCH_CELL_BITS], P.batch->S[e >> BATCH_CELL_BITS], e & BATCH_CELL_MASK);
		return;
	}
	b_rad_wind_reset(P, S, cells[t]);
}

// Radiation::preTimeStepCalculations for one non-wind cell (Radiation.cpp:257-296):
// the heating rate from the current fractions and optical depths.
__device__ __forceinline__ void rad_heating_cell(const Params& P, const State& S, long long id, double q_hii,
                                                 double q_pre, double q_den) {
	double Tmin = S.Tmin[id];
	double n_H = (P.X * q_den / P.hydrogenMass);
	double excessEnergy = P.photonEnergy - P.rydbergEnergy;
	double T = calc_temperature(P, q_hii, q_pre, q_den);
	double nHI = (1.0 - q_hii) * n_H;
	double A_pi = photoionisation_rate(nHI, RFLD(S.R, R_TAU, id), RFLD(S.R, R_DTAU, id), S.shellVol[id], P.photonRate);
	double photoion = n_H * (1.0 - q_hii) * A_pi * excessEnergy;
	double rate_rc = spline_eval(S.tables->rad_cool, T);
	double recombination = q_hii * q_hii * n_H * n_H * P.boltzmannConst * T * rate_rc;
	double collisions = q_hii * (1.0 - q_hii) * n_H * n_H * collisional_ionisation_rate(P, T);
	double rate = photoion - recombination - collisions;
	double softrate = rate;
	if (T < Tmin + 200 && rate < 0.0) softrate = smin(0.0, softrate * (T - Tmin) / 200.0);
	softrate *= P.heating_amp;
	RFLD(S.R, R_HEAT, id) = softrate;
	if (S.H) {
		// Radiation.cpp:278-279 (0/0 when rate is 0, as in the reference)
		FLD(S.H, H_EUVH, id) = photoion * (softrate / rate);
		FLD(S.H, H_RHII, id) = -recombination * (softrate / rate);
	}
	if (rate != rate) atomicOr(S.err, ERRB_NAN);
}

// Learned starting iterate: cells whose solve may take more than one Picard
// iteration (the ionisation front: optically thin enough to be reached,
// not yet ionised) are the ones the network serves and the plain solver
// records for its training set.
__device__ __forceinline__ bool front_cell(double tau_avg, double q_hii) { return tau_avg < 20.0 && q_hii < 0.99; }

// Network inputs of a cell (before its solve): log10 n_H, log10 T, x_HII,
// log10 of the optically thin photoionisation rate photonRate e^-tau sigma
// ds / shellVol, and log10 dt.
__device__ __forceinline__ void learned_features(const Params& P, double n_H, double T, double q_hii, double tau_avg,
                                                 double ds, double shellVol, double dt, float* f) {
	f[0] = (float)log10(n_H);
	f[1] = (float)log10(T);
	f[2] = (float)q_hii;
	f[3] = shellVol > 0 ? (float)(log10(P.photonRate * P.photoIonXsec * ds / shellVol) - 0.4342944819032518 * tau_avg)
	                    : -30.0f;
	f[4] = (float)log10(dt);
}

// log10(p / (1 - p)) with p clipped to [1e-9, 1 - 1e-9], and its inverse.
__device__ __forceinline__ float logit10(double p) {
	double q = fmin(fmax(p, 1e-9), 1.0 - 1e-9);
	return (float)log10(q / (1.0 - q));
}
__device__ __forceinline__ double inv_logit10(float l) {
	double v = fmin(fmax((double)l, -9.0), 9.0);
	return 1.0 / (1.0 + exp10(-v));
}

// One shell of the causal sweep of Radiation::transferRadiation
// (Radiation.cpp:600-612): tau interpolation, the implicit HII update
// (update_HIIfrac, :375-478) and the new optical depths.  Every cell of a
// shell reads only cells of inner shells, so a shell is fully parallel.
//
// Learned start (S.lstart set, LS or DIAG builds): a front cell whose entry of
// S.lstart holds a prediction (written by k_learned_infer before the sweep)
// runs one Picard iteration from it beside the plain first iteration from
// x_HII.  The prediction is accepted when its iteration meets the solver's own
// convergence test (its residual is below the solver tolerance) and the plain
// one does not; otherwise the plain iteration goes on as without it, so a
// rejected prediction leaves the plain result and iteration count unchanged.
// DIAG: the counters and the training-set recording are compiled in (a
// lean build without them keeps the sweep's instruction footprint small).
// SW: the cell's own inputs come from the sweep-ordered arrays (S.sw_rad,
// `sw` pointing at this cell's column, stride `swn`), formed by
// k_rad_sweep_prep with this function's own arithmetic.
template <bool DIAG, bool SW = false, bool LS = false>
__device__ __forceinline__ void rad_shell(const Params& P, const State& S, const long long id, double h,
                                          double* sw = nullptr, long long swn = 0) {
	const double dt = h * S.scal[0];
	bool star = false, front = false, inner = false;
	double q_den = 0, q_pre = 0, q_hii = 0, ds = 0, n_H = 0, T = 1, alphaB = 0, A_ci = 0, tau_avg = 0, shellVol = 0;
	double nH_cell = 0;
	long long nb[4] = {-1, -1, -1, -1};
	double w[4] = {0, 0, 0, 0};
	// everything that does not depend on the inner shells
	int ijk[3];
	double xc[3];
	cell_ijk(P, id, ijk);
	cell_xc(P, ijk, xc);
	inner = dist2_cells(P, xc) > 0.95;
	if (inner) neighbours(P, ijk, xc, nb, w);
	// Radiation::isStar (Radiation.cpp:682-684): z compares an int with a double.
	star = (int)xc[0] == (int)P.sxc[0] && (int)xc[1] == (int)P.sxc[1] && (double)(int)xc[2] == P.sxc[2];
	if (SW) {
		nH_cell = sw[0];
		q_hii = sw[3 * swn];
		ds = sw[4 * swn];
		if (!star) {
			n_H = nH_cell;
			alphaB = sw[swn];
			A_ci = sw[2 * swn];
			shellVol = sw[5 * swn];
		}
	} else {
		q_den = FLD(S.Q, DEN, id);
		q_pre = FLD(S.Q, PRE, id);
		q_hii = FLD(S.Q, HII, id);
		ds = S.ds[id];
#ifdef TRG_FAST_MATH
		nH_cell = P.X * q_den / P.hydrogenMass;
#endif
		if (!star) {
#ifdef TRG_FAST_MATH
			n_H = nH_cell;
#else
			n_H = P.X * q_den / P.hydrogenMass;
#endif
			T = calc_temperature(P, q_hii, q_pre, q_den);
			alphaB = spline_eval(S.tables->rad_recomb, T);
			A_ci = collisional_ionisation_rate(P, T);
			shellVol = S.shellVol[id];
		}
	}
	const double2* src[4];
	nb_sources<4>(S, S.R, nb, w, src);
	sweep_wait();
	double tau = 0, tau_a = 0;
	if (inner) tau_sc2(P, src, w, tau, tau_a);
	if (!star) {
		tau_avg = tau_a;
		front = front_cell(tau_avg, q_hii);
	}
	double start = q_hii;
	bool learned = false, used_learned = false;
	if ((LS || DIAG) && front && S.lstart) {
		// a candidate of this sweep (at the front by the previous sweep's optical
		// depth, not yet overwritten) holds the network's output in its slot -
		// in sweep order (single grids) or per cell (batches) - unless the
		// candidate list overflowed and the network did not run
		const double tau_prev = SW ? sw[SW_TAU_A * swn] : RFLD(S.R, R_TAU_A, id);
		if (front_cell(tau_prev, q_hii) && *S.lcand_n <= (unsigned)LCAND_MAX) {
			const double st = SW ? sw[SW_LSTART * swn] : S.lstart[id];
			if (st == st) {
				start = st;
				learned = used_learned = true;
			}
		}
	}
	if (SW) sw[SW_TAU_A * swn] = tau_a;  // the next sweep's learned-start candidates are chosen from it
	unsigned iters = 0;
	double hii_new = 1, hii_a_new = 1;
	if (star) {
		RFLD(S.R, R_HEAT, id) = 0;
		FLD(S.Q, HII, id) = 1;
		RFLD(S.R, R_HII_A, id) = 1;
	} else {
		double A_pi = 0;
		double x_new = q_hii;
		double HII_avg = q_hii;
		double HII_avg_old;
		int niter = 0, miter = 0;
		bool converged = false;
		const double em_tau = d_exp(-tau_avg);  // the same in every iteration
		while (!converged) {
			niter++;
			HII_avg_old = HII_avg;
			x_new = q_hii;
			double dtau_avg = (1.0 - HII_avg) * n_H * P.photoIonXsec * ds;
			double nHI = (1.0 - HII_avg) * n_H;
			A_pi = photoionisation_rate_e(nHI, em_tau, dtau_avg, shellVol, P.photonRate);
			double nHII_aB = HII_avg * n_H * alphaB;
			double nHII_Aci = HII_avg * n_H * A_ci;
			doric(dt, HII_avg, x_new, A_pi, nHII_aB, nHII_Aci);
#ifdef TRG_FAST_MATH
			// the same test without its division
			const bool small_step = fabs(HII_avg - HII_avg_old) < 1.0e-3 * fabs(HII_avg);
#else
			const bool small_step = fabs((HII_avg - HII_avg_old) / HII_avg) < 1.0e-3;
#endif
			if ((small_step || (HII_avg < 1.0e-5) || A_pi == 0)) converged = true;
			if (learned) {
				// beside the plain first iteration (from x_HII), one iteration
				// from the prediction: its residual test is the solver's own
				// convergence test.  It is taken when the plain first iteration
				// has not converged and the prediction's has; otherwise it is
				// dropped and the plain iteration goes on untouched, so the
				// prediction never costs an iteration.
				learned = false;
				double hp = start, xp = q_hii;
				const double dtau_p = (1.0 - hp) * n_H * P.photoIonXsec * ds;
				const double A_p = photoionisation_rate_e((1.0 - hp) * n_H, em_tau, dtau_p, shellVol, P.photonRate);
				doric(dt, hp, xp, A_p, hp * n_H * alphaB, hp * n_H * A_ci);
#ifdef TRG_FAST_MATH
				const bool small_p = fabs(hp - start) < 1.0e-3 * fabs(hp);
#else
				const bool small_p = fabs((hp - start) / hp) < 1.0e-3;
#endif
				const bool take = !converged && (small_p || hp < 1.0e-5 || A_p == 0);
				if (DIAG && P.stats_on) {
					stat_add(S.stats, TRG_STAT_LEARNED_CELLS, 1u);
					stat_add(S.stats, TRG_STAT_LEARNED_ACCEPTED, take ? 1u : 0u);
				}
				if (take) {
					HII_avg = hp;
					x_new = xp;
					A_pi = A_p;
					break;
				}
			}
			if (niter > 10005) {
				miter++;
				niter = 0;
				HII_avg = 0.5 * (HII_avg + HII_avg_old);
			}
			if (miter > 5 || x_new != x_new) {
				atomicOr(S.err, ERRB_PICARD);
				break;
			}
		}
		RFLD(S.R, R_HII_A, id) = HII_avg;
		FLD(S.Q, HII, id) = x_new;
		hii_a_new = HII_avg;
		hii_new = x_new;
		if (x_new > 0.001) FLD(S.Q, ADV, id) = 1;
		iters += (unsigned)miter * 10006u + (unsigned)niter;
		if (DIAG && P.stats_on && used_learned) stat_add(S.stats, TRG_STAT_LEARNED_ITERS, iters);
		if (DIAG && front && S.harvest && !used_learned) {
			// training record: 5 inputs, then the converged <x>, x and the iteration count
			unsigned long long slot = atomicAdd(S.harvest_n, 1ull);
			if (slot < (unsigned long long)S.harvest_cap) {
				float* r = S.harvest + slot * 8;
				if (SW) T = calc_temperature(P, q_hii, FLD(S.Q, PRE, id), FLD(S.Q, DEN, id));
				learned_features(P, n_H, T, q_hii, tau_avg, ds, shellVol, dt, r);
				r[5] = logit10(HII_avg) - logit10(q_hii);
				r[6] = logit10(x_new) - logit10(q_hii);
				r[7] = log2f((float)iters);
			}
		}
	}
#ifdef TRG_FAST_MATH
	const double nH = nH_cell;
#else
	const double nH = SW ? nH_cell : P.X * q_den / P.hydrogenMass;
#endif
	store_taus(S, id, tau, (1.0 - hii_new) * nH * P.photoIonXsec * ds, tau_a, (1.0 - hii_a_new) * nH * P.photoIonXsec * ds);
	if (DIAG && P.stats_on) {
		stat_picard(S.stats, iters);
		stat_add(S.stats, TRG_STAT_FRONT_CELLS, front ? 1u : 0u);
		stat_add(S.stats, TRG_STAT_FRONT_ITERS, front ? iters : 0u);
	}
}

// The fast build fits 7 CTAs per SM (28 warps, one spilled register pair) for
// the latency-bound large shells; the exact build keeps the plain bound (a
// minimum-blocks argument of 1 alone made its code 8% slower).
#ifdef TRG_FAST_MATH
#define TRG_RAD_SHELL_BOUNDS __launch_bounds__(128, 7)
#else
#define TRG_RAD_SHELL_BOUNDS __launch_bounds__(128)
#endif
__global__ void TRG_RAD_SHELL_BOUNDS k_rad_shell_fp64(Params P, State S, const int* __restrict__ cells, int count,
                                                       double h) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= count) return;
	if (TRG_BATCHED && P.batch) {
		const int e = cells[t];
		const int g = e >> BATCH_CELL_BITS;
		rad_shell<false>(P.batch->P[g], P.batch->S[g], e & BATCH_CELL_MASK, h);
		return;
	}
	rad_shell<false>(P, S, cells[t], h);
}
// The same with the solver counters and training-set recording compiled in.
__global__ void __launch_bounds__(128) k_rad_shell_diag(Params P, State S, const int* __restrict__ cells, int count,
                                                       double h) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= count) return;
	rad_shell<true>(P, S, cells[t], h);
}

// ----------------------------------------------- learned starting iterate
// Before each radiation sweep with a network loaded, k_rad_sweep_prep lists
// the candidate front cells (by the previous sweep's TAU_A and x_HII, the
// front criterion) as sweep positions; this kernel runs the network over
// the candidates and writes each candidate's slot (a prediction, or NaN),
// in tcgen05 tiles of 128: a persistent grid of INFER_CTAS CTAs, each loading
// the model image and allocating its tensor memory once and looping over the
// tiles (CTAs beyond the list return at once):
// inputs log n_H, log T, x_HII, log of the optically thin photoionisation
// rate at that TAU_A, log dt; cells predicted to need more than two plain
// iterations get the predicted time-averaged fraction as their starting
// iterate.  More than LCAND_MAX candidates (the first sweep of a run, before
// any optical depth exists, lists every neutral cell) means no predictions
// for that sweep.
__global__ void __launch_bounds__(128) k_learned_infer(Params P, State S, const int* __restrict__ cells, double h) {
	extern __shared__ __align__(128) unsigned char sm_mlp[];
	const unsigned n = *S.lcand_n;
	if (n > (unsigned)LCAND_MAX || blockIdx.x * 128u >= n) return;  // uniform over the CTA
	const double dt = h * S.scal[0];
	const long long sn = S.sw_rad_n;
	const uint32_t tm = mlp::infer_begin(sm_mlp, reinterpret_cast<const uint4*>(S.mlp_img));
	uint32_t phase = 0;
	bool ok = true;
	for (unsigned base = blockIdx.x * 128u; base < n; base += gridDim.x * 128u) {
		const unsigned t = base + threadIdx.x;
		const bool valid = t < n;
		const int pos = valid ? S.lcand[t] : 0;
		float f[5] = {0, 0, 0, 0, 0}, y[3];
		double q_hii = 0;
		if (valid) {
			const long long id = cells[pos];
			const double* sw = S.sw_rad + pos;
			const double q_den = FLD(S.Q, DEN, id), q_pre = FLD(S.Q, PRE, id);
			q_hii = sw[3 * sn];
			const double T = calc_temperature(P, q_hii, q_pre, q_den);
			learned_features(P, sw[0], T, q_hii, sw[SW_TAU_A * sn], sw[4 * sn], sw[5 * sn], dt, f);
		}
		ok = mlp::infer_step(sm_mlp, tm, phase, f, y);
		if (!ok) break;
		if (valid)
			S.sw_rad[SW_LSTART * sn + pos] =
			    y[2] > 1.0f ? inv_logit10(logit10(q_hii) + y[0]) : __longlong_as_double(0x7ff8000000000000LL);
	}
	mlp::infer_end(tm);
	if (!ok && threadIdx.x == 0) atomicOr(S.err, ERRB_TC);
}

// The network over a batch's candidates (packed (grid, cell) entries): the
// same inputs as k_learned_infer, each grid's cells read in place (n_H with
// the radiation sweep's own arithmetic), the prediction into the cell's slot.
__global__ void __launch_bounds__(128) k_batch_learned_infer(Params Pv, State Sv, double h) {
#if TRG_BATCHED
	extern __shared__ __align__(128) unsigned char sm_mlp[];
	const unsigned n = *Sv.lcand_n;
	if (n > (unsigned)LCAND_MAX || blockIdx.x * 128u >= n) return;  // uniform over the CTA
	const BatchTable& B = *Pv.batch;
	const uint32_t tm = mlp::infer_begin(sm_mlp, reinterpret_cast<const uint4*>(Sv.mlp_img));
	uint32_t phase = 0;
	bool ok = true;
	for (unsigned base = blockIdx.x * 128u; base < n; base += gridDim.x * 128u) {
		const unsigned t = base + threadIdx.x;
		const bool valid = t < n;
		const int e = valid ? Sv.lcand[t] : 0;
		const int g = e >> BATCH_CELL_BITS;
		const long long id = e & BATCH_CELL_MASK;
		float f[5] = {0, 0, 0, 0, 0}, y[3];
		double q_hii = 0;
		if (valid) {
			const Params& P = B.P[g];
			const State& S = B.S[g];
			const double q_den = FLD(S.Q, DEN, id), q_pre = FLD(S.Q, PRE, id);
			q_hii = FLD(S.Q, HII, id);
			const double n_H = P.X * q_den / P.hydrogenMass;
			const double T = calc_temperature(P, q_hii, q_pre, q_den);
			learned_features(P, n_H, T, q_hii, RFLD(S.R, R_TAU_A, id), S.ds[id], S.shellVol[id], h * S.scal[0], f);
		}
		ok = mlp::infer_step(sm_mlp, tm, phase, f, y);
		if (!ok) break;
		if (valid)
			B.S[g].lstart[id] =
			    y[2] > 1.0f ? inv_logit10(logit10(q_hii) + y[0]) : __longlong_as_double(0x7ff8000000000000LL);
	}
	mlp::infer_end(tm);
	if (!ok && threadIdx.x == 0) atomicOr(Sv.err, ERRB_TC);
#endif
}

// The cell's own inputs of the radiation sweep in sweep order (S.sw_rad):
// what rad_shell computes from the cell's density, pressure and fraction
// before waiting for the inner shells, with its arithmetic: n_H, the case-B
// recombination rate and the collisional ionisation rate at the cell's
// temperature, and x_HII; with `init` also the fixed path length and shell
// volume.  One parallel pass before each sweep (single grids only).
__global__ void __launch_bounds__(256) k_rad_sweep_prep(Params P, State S, const int* __restrict__ cells, int n,
                                                         int init) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n) return;
	const long long id = cells[t];
	const long long sn = S.sw_rad_n;
	double* sw = S.sw_rad + t;
	const double q_den = FLD(S.Q, DEN, id), q_pre = FLD(S.Q, PRE, id), q_hii = FLD(S.Q, HII, id);
	const double n_H = P.X * q_den / P.hydrogenMass;
	const double T = calc_temperature(P, q_hii, q_pre, q_den);
	sw[0] = n_H;
	sw[sn] = spline_eval(S.tables->rad_recomb, T);
	sw[2 * sn] = collisional_ionisation_rate(P, T);
	sw[3 * sn] = q_hii;
	if (init) {
		sw[4 * sn] = S.ds[id];
		sw[5 * sn] = S.shellVol[id];
		sw[SW_TAU_A * sn] = RFLD(S.R, R_TAU_A, id);
	}
	if (S.lstart) {
		// learned start: a cell at the front by the previous sweep's optical
		// depth becomes a candidate (its sweep position); the network writes
		// every candidate's slot, and no other slot is read
		const bool cand = front_cell(sw[SW_TAU_A * sn], q_hii);
		const unsigned ballot = __ballot_sync(__activemask(), cand);
		if (cand) {
			const int lane = threadIdx.x & 31, leader = __ffs(ballot) - 1;
			unsigned base = 0;
			if (lane == leader) base = atomicAdd(S.lcand_n, (unsigned)__popc(ballot));
			base = __shfl_sync(ballot, base, leader);
			S.lcand[base + __popc(ballot & ((1u << lane) - 1))] = t;
		}
	}
}
// A radiation shell reading its cells' own inputs from S.sw_rad; `off` is the
// shell's offset in the non-wind sweep list.
__global__ void TRG_RAD_SHELL_BOUNDS k_rad_shell_sw(Params P, State S, const int* __restrict__ cells, int count,
                                                     double h, long long off) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= count) return;
	rad_shell<false, true>(P, S, cells[t], h, S.sw_rad + off + t, S.sw_rad_n);
}
// The same with the solver counters and training-set recording compiled in.
__global__ void __launch_bounds__(128) k_rad_shell_sw_diag(Params P, State S, const int* __restrict__ cells,
                                                           int count, double h, long long off) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= count) return;
	rad_shell<true, true>(P, S, cells[t], h, S.sw_rad + off + t, S.sw_rad_n);
}
// The same, front cells starting from the learned prediction (S.lstart).
__global__ void TRG_RAD_SHELL_BOUNDS k_rad_shell_sw_ls(Params P, State S, const int* __restrict__ cells, int count,
                                                        double h, long long off) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= count) return;
	rad_shell<false, true, true>(P, S, cells[t], h, S.sw_rad + off + t, S.sw_rad_n);
}

// Learned start in batches (exact build, cells read in place): a front cell
// of any grid whose per-cell slot S.lstart[id] holds a prediction (written by
// k_batch_learned_infer before the sweep) tries it beside its plain first
// iteration, as in single grids.
__global__ void TRG_RAD_SHELL_BOUNDS k_rad_shell_fp64_ls(Params P, State S, const int* __restrict__ cells, int count,
                                                         double h) {
#if TRG_BATCHED
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= count || !P.batch) return;
	const int e = cells[t];
	const int g = e >> BATCH_CELL_BITS;
	rad_shell<false, false, true>(P.batch->P[g], P.batch->S[g], e & BATCH_CELL_MASK, h);
#endif
}
// Before each radiation sweep of a batch with a network loaded: the cells at
// the front by the previous sweep's optical depth (TAU_A, kept in R) and x_HII
// become candidates, listed as packed (grid, cell) entries; the network writes
// every candidate's slot.  One thread per cell of the padded ranges (a
// 256-thread block never straddles two grids).
__global__ void __launch_bounds__(256) k_batch_learned_prep(Params Pv, State Sv) {
#if TRG_BATCHED
	const BatchTable& B = *Pv.batch;
	const long long pos = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	const int g = batch_slot(B.cell_off, B.G, blockIdx.x * (long long)blockDim.x);
	const long long id = pos - B.cell_off[g];
	const Params& P = B.P[g];
	const State& S = B.S[g];
	const bool cand = id < P.N && front_cell(RFLD(S.R, R_TAU_A, id), FLD(S.Q, HII, id));
	const unsigned ballot = __ballot_sync(0xffffffffu, cand);
	if (cand) {
		const int lane = threadIdx.x & 31, leader = __ffs(ballot) - 1;
		unsigned base = 0;
		if (lane == leader) base = atomicAdd(Sv.lcand_n, (unsigned)__popc(ballot));
		base = __shfl_sync(ballot, base, leader);
		Sv.lcand[base + __popc(ballot & ((1u << lane) - 1))] = (g << BATCH_CELL_BITS) | (int)id;
	}
#endif
}

// Radiation::transferRadiation2 (Radiation.cpp:508-567) for the implicit2 and
// explicit schemes.  Its rayTrace (:480-506) is a causal sweep that only
// interpolates TAU and sets DTAU / DTAU_A from the current fractions (one
// shell per launch); the fractions are then updated by one launch over all
// non-wind cells, which are independent of each other in these schemes.
__device__ __forceinline__ void b_rad_tau_shell(const Params& P, const State& S, long long id) {
	int ijk[3];
	double xc[3];
	cell_ijk(P, id, ijk);
	cell_xc(P, ijk, xc);
	const bool inner = dist2_cells(P, xc) > 0.95;
	long long nb[4];
	double w[4];
	if (inner) neighbours(P, ijk, xc, nb, w);
	const double nH = P.X * FLD(S.Q, DEN, id) / P.hydrogenMass;
	const double dtau = (1.0 - FLD(S.Q, HII, id)) * nH * P.photoIonXsec * S.ds[id];
	const double dtau_a = (1.0 - RFLD(S.R, R_HII_A, id)) * nH * P.photoIonXsec * S.ds[id];
	const double2* src[4] = {nullptr, nullptr, nullptr, nullptr};
	if (inner) nb_sources<4>(S, S.R, nb, w, src);
	sweep_wait();
	RFLD(S.R, R_TAU, id) = inner ? tau_sc(P, src, w) : 0.0;
	RFLD(S.R, R_DTAU, id) = dtau;
	RFLD(S.R, R_DTAU_A, id) = dtau_a;
}
__global__ void __launch_bounds__(128) k_rad_tau_shell(Params P, State S, const int* __restrict__ cells, int count) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= count) return;
	if (TRG_BATCHED && P.batch) {
		const int e = cells[t];
		b_rad_tau_shell(P.batch->P[e >> BATCH_CELL_BITS], P.batch->S[e >> BATCH_CELL_BITS], e & BATCH_CELL_MASK);
		return;
	}
	b_rad_tau_shell(P, S, cells[t]);
}

// Radiation::update_HIIfrac (Radiation.cpp:375-478) for implicit2 (Picard
// iteration with tau_avg = TAU) and explicit (one doric step whose
// time-averaged result becomes Q[HII]; HII_A is not written).
__device__ __forceinline__ void b_rad_solve2(const Params& P, const State& S, long long id, double h) {
	int ijk[3];
	double xc[3];
	cell_ijk(P, id, ijk);
	cell_xc(P, ijk, xc);
	const double dt = h * S.scal[0];
	if ((int)xc[0] == (int)P.sxc[0] && (int)xc[1] == (int)P.sxc[1] && (double)(int)xc[2] == P.sxc[2]) {
		RFLD(S.R, R_HEAT, id) = 0;
		FLD(S.Q, HII, id) = 1;
		RFLD(S.R, R_HII_A, id) = 1;
		return;
	}
	const double q_den = FLD(S.Q, DEN, id), q_pre = FLD(S.Q, PRE, id), q_hii = FLD(S.Q, HII, id);
	const double n_H = P.X * q_den / P.hydrogenMass;
	const double T = calc_temperature(P, q_hii, q_pre, q_den);
	const double alphaB = spline_eval(S.tables->rad_recomb, T);
	const double A_ci = collisional_ionisation_rate(P, T);
	const double ds = S.ds[id], shellVol = S.shellVol[id];
	double x = q_hii;
	if (P.rt_scheme == 1) {
		double x_avg = x, x_avg_old, A_pi;
		const double tau_avg = RFLD(S.R, R_TAU, id);
		int niter = 0, miter = 0;
		bool converged = false;
		while (!converged) {
			niter++;
			x_avg_old = x_avg;
			x = q_hii;
			double dtau_avg = (1.0 - x_avg) * n_H * P.photoIonXsec * ds;
			double nHI = (1.0 - x_avg) * n_H;
			A_pi = photoionisation_rate(nHI, tau_avg, dtau_avg, shellVol, P.photonRate);
			double nHII_aB = x_avg * n_H * alphaB;
			double nHII_Aci = x_avg * n_H * A_ci;
			doric(dt, x_avg, x, A_pi, nHII_aB, nHII_Aci);
			if ((fabs((x_avg - x_avg_old) / x_avg) < 1.0e-3 || (x_avg < 1.0e-5) || A_pi == 0)) converged = true;
			if (niter > 10005) {
				miter++;
				niter = 0;
				x_avg = 0.5 * (x_avg + x_avg_old);
			}
			if (miter > 5 || x != x) {
				atomicOr(S.err, ERRB_PICARD);
				break;
			}
		}
		RFLD(S.R, R_HII_A, id) = x_avg;
	} else {
		const double x_avg = x;
		const double nHI = (1.0 - x) * (P.X * q_den / P.hydrogenMass);
		const double A_pi = photoionisation_rate(nHI, RFLD(S.R, R_TAU, id), RFLD(S.R, R_DTAU, id), shellVol, P.photonRate);
		const double nHII_aB = x_avg * n_H * alphaB;
		const double nHII_Aci = x_avg * n_H * A_ci;
		double x_dummy = x;
		doric(dt, x, x_dummy, A_pi, nHII_aB, nHII_Aci);
	}
	FLD(S.Q, HII, id) = x;
	if (x > 0.001) FLD(S.Q, ADV, id) = 1;
}
__global__ void __launch_bounds__(128) k_rad_solve2(Params P, State S, const int* __restrict__ cells, int count,
                                                    double h) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= count) return;
	if (TRG_BATCHED && P.batch) {
		const int e = cells[t];
		b_rad_solve2(P.batch->P[e >> BATCH_CELL_BITS], P.batch->S[e >> BATCH_CELL_BITS], e & BATCH_CELL_MASK, h);
		return;
	}
	b_rad_solve2(P, S, cells[t], h);
}

// Star off: Radiation::transferRadiation else-branch (Radiation.cpp:638-650), interior cells.
__device__ __forceinline__ void b_rad_no_star_fp64(const Params& P, const State& S, long long id, double h) {

	const double dt = h * S.scal[0];
	double x_new = FLD(S.Q, HII, id), x_dummy = x_new;
	double n_H = P.X * FLD(S.Q, DEN, id) / P.hydrogenMass;
	double T = calc_temperature(P, FLD(S.Q, HII, id), FLD(S.Q, PRE, id), FLD(S.Q, DEN, id));
	double nHII_aB = x_new * n_H * spline_eval(S.tables->rad_recomb, T);
	double nHII_Aci = x_new * n_H * collisional_ionisation_rate(P, T);
	doric(dt, x_new, x_dummy, 0, nHII_aB, nHII_Aci);
	FLD(S.Q, HII, id) = x_new;
}
__global__ void k_rad_no_star_fp64(Params P, State S, double h) {
	if (TRG_BATCHED && P.batch) {
		const BatchTable& B = *P.batch;
		const int g = batch_slot(B.cell_off, B.G, blockIdx.x * (long long)blockDim.x);
		const long long lid = blockIdx.x * (long long)blockDim.x + threadIdx.x - B.cell_off[g];
		if (lid < B.P[g].N) b_rad_no_star_fp64(B.P[g], B.S[g], lid, h);
		return;
	}
	const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (id >= P.N) return;
	b_rad_no_star_fp64(P, S, id, h);
}

// Radiation::preTimeStepCalculations (photoheating), Radiation.cpp:257-296, non-wind cells.
__device__ __forceinline__ void b_rad_heating_fp64(const Params& P, const State& S, long long id) {
	int ijk[3];
	double xc[3];
	cell_ijk(P, id, ijk);
	cell_xc(P, ijk, xc);
	if (is_wind(P, id, ijk, xc)) return;
	rad_heating_cell(P, S, id, FLD(S.Q, HII, id), FLD(S.Q, PRE, id), FLD(S.Q, DEN, id));
}
__global__ void __launch_bounds__(256) k_rad_heating_fp64(Params P, State S) {
	if (TRG_BATCHED && P.batch) {
		const BatchTable& B = *P.batch;
		const int g = batch_slot(B.cell_off, B.G, blockIdx.x * (long long)blockDim.x);
		const long long lid = blockIdx.x * (long long)blockDim.x + threadIdx.x - B.cell_off[g];
		if (lid < B.P[g].N) b_rad_heating_fp64(B.P[g], B.S[g], lid);
		return;
	}
	const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (id >= P.N) return;
	b_rad_heating_fp64(P, S, id);
}

// Radiation::updateSourceTerms (Radiation.cpp:653-680) then advSolution + fixSolution.
__device__ __forceinline__ void b_rad_update_fp64(const Params& P, const State& S, long long id, double h, int mode) {

	const double dt = h * S.scal[0];
	double u[7], udot[7] = {0, 0, 0, 0, 0, 0, 0};
#pragma unroll
	for (int i = 0; i < NU; ++i) u[i] = FLD(S.U, i, id);
	if (P.star_on) {
		double q_hii = FLD(S.Q, HII, id), q_den = FLD(S.Q, DEN, id), q_adv = FLD(S.Q, ADV, id);
		if (P.coupling == CP_TTI) {
			double mu_inv_new = P.X * (q_hii + 1.0) + (1.0 - P.X) * 0.25;
			double T_new = P.THI + (P.THII - P.THI) * q_hii;
			double pre_new = P.specificGasConstant * mu_inv_new * q_den * T_new;
			double ke = 0.0;
			#pragma unroll
			for (int dim = 0; dim < 3; ++dim) if (dim < P.nd) ke += 0.5 * u[VEL + dim] * u[VEL + dim] / u[DEN];
			double E_new = pre_new / (P.gamma - 1.0) + ke;
			udot[PRE] += (E_new - u[PRE]) / dt;
		} else if (P.coupling == CP_NEQ) {
			udot[PRE] += RFLD(S.R, R_HEAT, id);
		}
		udot[HII] += (q_hii * q_den - u[HII]) / dt;
		udot[ADV] += (q_adv * q_den - u[ADV]) / dt;
	}
	if (mode == 1) {
		for (int i = 0; i < NU; ++i) FLD(S.UDOT, i, id) += udot[i];
		return;
	}
#pragma unroll
	for (int i = 0; i < NU; ++i) u[i] = u[i] + dt * udot[i];
	if (!fix_solution(P, u)) atomicOr(S.err, ERRB_NAN);
#pragma unroll
	for (int i = 0; i < NU; ++i) FLD(S.U, i, id) = u[i];
	if (mode == 2) store_fixed_q(P, S, id, u);
}
__global__ void __launch_bounds__(256) k_rad_update_fp64(Params P, State S, double h, int mode) {
	if (TRG_BATCHED && P.batch) {
		const BatchTable& B = *P.batch;
		const int g = batch_slot(B.cell_off, B.G, blockIdx.x * (long long)blockDim.x);
		const long long lid = blockIdx.x * (long long)blockDim.x + threadIdx.x - B.cell_off[g];
		if (lid < B.P[g].N) b_rad_update_fp64(B.P[g], B.S[g], lid, h, mode);
		return;
	}
	const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (id >= P.N) return;
	b_rad_update_fp64(P, S, id, h, mode);
}

// ----------------------------------------------------------- thermodynamics
// Henney et al. (2009) heating and cooling, Thermodynamics.cpp:113-211.
__device__ __forceinline__ double th_imlc(const Params& P, double ne, double T) {
	return P.imlc * P.z0 * ne * ne * d_exp(-P.T1 / T - (P.T2 / T) * (P.T2 / T));
}
__device__ __forceinline__ double th_nmlc(const Params& P, double ne, double nn, double T) {
	return P.nmlc * P.z0 * ne * nn * d_exp(-P.T3 / T - (P.T4 / T) * (P.T4 / T));
}
__device__ __forceinline__ double th_ciec(const Params& P, double ne, double T) {
	if (T > P.ciec_minT) {
		double cie_rate = P.ciec * ne * ne * P.z0 * d_exp(-0.63 * d_log(T)) * (1.0 - d_exp(-d_pow(1.0e-5 * T, 1.63)));
		double smoothing = smin(1.0, (T - 5.0e4) / (2.0e4));
		return cie_rate * smoothing;
	}
	return 0;
}
__device__ __forceinline__ double th_nmc(const Params& P, double nH, double x, double T) {
	double T0 = 70.0 + 220.0 * d_pow(nH / P.n0, 0.2);
	return P.nmc * (1.0 - x) * (1.0 - x) * d_pow(nH, 1.6) * sqrt(T) * d_exp(-T0 / T);
}
__device__ __forceinline__ double th_cxhi(const Params& P, const State& S, double nH, double x, double T) {
	double rate = spline_eval(S.tables->th_cxhi, d_log10(T));
	return x * (1.0 - x) * nH * nH * d_exp((2.302585093 * rate) - ((T / P.cxhi_damp) * (T / P.cxhi_damp)));
}
__device__ __forceinline__ double th_fuvh(const Params& P, double nH, double Av, double F) {
	return P.fuvh_a * nH * F * d_exp(-1.9 * Av) / (P.fuvh_b + P.fuvh_c * F * d_exp(-1.9 * Av) / nH);
}
__device__ __forceinline__ double th_irh(const Params& P, double nH, double Av, double F) {
	return P.irh_a * nH * F * d_exp(-0.05 * Av) * d_exp(-2.0 * d_log(1.0 + P.irh_b / nH));
}
__device__ __forceinline__ double soft_landing(double rate, double T, double T_min) {
	double result = rate;
	if (rate < 0.0) {
		if (T <= T_min) result = 0;
		else if (T <= T_min + 200) result = rate * (T - T_min) / 200;
	}
	return result;
}
__device__ __forceinline__ double th_cooling(const Params& P, const State& S, double heat, double ne, double nn, double nH,
                                             double x, double T) {
	double r = heat;
	r -= th_imlc(P, ne, T);
	r -= th_nmlc(P, ne, nn, T);
	r -= th_cxhi(P, S, nH, x, T);
	r -= th_ciec(P, ne, T);
	r -= th_nmc(P, nH, x, T);
	return r;
}

// One shell of Thermodynamics::rayTrace / updateColDen (Thermodynamics.cpp:339-417).
// `own`: the cell's ds rho / m_H in the sweep-ordered array, or null.
__device__ __forceinline__ void b_colden_shell_fp64(const Params& P, const State& S, long long id,
                                                    const double* own = nullptr) {
	int ijk[3];
	double xc[3];
	cell_ijk(P, id, ijk);
	cell_xc(P, ijk, xc);
	const bool inner = dist2_cells(P, xc) > 0.95 * 0.95;
	long long nb[4];
	double w0[4];
	if (inner) neighbours(P, ijk, xc, nb, w0);
	const double dcolden = own ? *own : (FLD(S.Q, DEN, id) / P.hydrogenMass) * S.ds[id];
	const double2* src[4] = {nullptr, nullptr, nullptr, nullptr};
	if (inner) nb_sources<2>(S, S.T, nb, w0, src);
	sweep_wait();
	double newcolden = 0.0;
	if (inner) {
		double colden[4] = {0, 0, 0, 0}, w[4];
#ifdef TRG_FAST_MATH
		for (int i = 0; i < 4; ++i)
			if (src[i]) {
				const double2 c = __ldcg(src[i]);  // COL_DEN, DCOL_DEN
				colden[i] = c.x + c.y;
			}
		// The interpolation is the weighted harmonic mean sum(w0) / sum(w0 / c)
		// over the non-zero c; numerator and denominator scaled by the product
		// of those c take one division (per-neighbour divisions where that
		// product would overflow).
		double m[4];
		for (int i = 0; i < 4; ++i) m[i] = colden[i] == 0 ? 1.0 : colden[i];
		const double m01 = m[0] * m[1], m23 = m[2] * m[3], prod = m01 * m23;
		if (prod < 1.0e300) {
			const double p[4] = {m[1] * m23, m[0] * m23, m[3] * m01, m[2] * m01};
			double num = 0, den = 0;
			for (int i = 0; i < 4; ++i)
				if (colden[i] != 0) {
					num += w0[i];
					den += w0[i] * p[i];
				}
			newcolden = den != 0 ? num * prod / den : 0.0;
		} else {
			for (int i = 0; i < 4; ++i) w[i] = colden[i] == 0 ? 0 : w0[i] / colden[i];
			double sum_w = w[0] + w[1] + w[2] + w[3];
			for (int i = 0; i < 4 && sum_w != 0; ++i) {
				w[i] = w[i] / sum_w;
				newcolden += w[i] * colden[i];
			}
		}
#else
		for (int i = 0; i < 4; ++i) {
			if (src[i]) {
				const double2 c = __ldcg(src[i]);  // COL_DEN, DCOL_DEN
				colden[i] = c.x + c.y;
			}
			w[i] = colden[i] == 0 ? 0 : w0[i] / colden[i];
		}
		double sum_w = w[0] + w[1] + w[2] + w[3];
		for (int i = 0; i < 4 && sum_w != 0; ++i) {
			w[i] = w[i] / sum_w;
			newcolden += w[i] * colden[i];
		}
#endif
	}
	reinterpret_cast<double2*>(S.T + id * 2)[0] = make_double2(newcolden, dcolden);
}
// The cell's own column density of the sweep in sweep order (S.sw_col):
// ds rho / m_H, as b_colden_shell_fp64 forms it; with `init` also the fixed
// path lengths.  One parallel pass before each column-density sweep.
__global__ void __launch_bounds__(256) k_colden_sweep_prep(Params P, State S, const int* __restrict__ cells, int n,
                                                            int init) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n) return;
	const long long id = cells[t];
	if (init) S.sw_col[S.sw_col_n + t] = S.ds[id];
	S.sw_col[t] = (FLD(S.Q, DEN, id) / P.hydrogenMass) * S.sw_col[S.sw_col_n + t];
}
__global__ void __launch_bounds__(128) k_colden_shell_sw(Params P, State S, const int* __restrict__ cells, int count,
                                                          long long off) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= count) return;
	b_colden_shell_fp64(P, S, cells[t], S.sw_col + off + t);
}
__global__ void __launch_bounds__(128) k_colden_shell_fp64(Params P, State S, const int* __restrict__ cells, int count) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= count) return;
	if (TRG_BATCHED && P.batch) {
		const int e = cells[t];
		b_colden_shell_fp64(P.batch->P[e >> BATCH_CELL_BITS], P.batch->S[e >> BATCH_CELL_BITS], e & BATCH_CELL_MASK);
		return;
	}
	b_colden_shell_fp64(P, S, cells[t]);
}

// Thermodynamics::preTimeStepCalculations rates, Thermodynamics.cpp:224-263, non-wind cells.
__device__ __forceinline__ void b_thermo_rates_fp64(const Params& P, const State& S, long long id) {

	int ijk[3];
	double xc[3];
	cell_ijk(P, id, ijk);
	cell_xc(P, ijk, xc);
	if (is_wind(P, id, ijk, xc)) return;
	if (FLD(S.Q, ADV, id) < P.thermo_hii_switch) {
		TFLD(S.T, T_RATE, id) = 0;
		return;
	}
	double q_den = FLD(S.Q, DEN, id), x = FLD(S.Q, HII, id), q_pre = FLD(S.Q, PRE, id);
	double nH = P.X * q_den / P.hydrogenMass;
	double ne = nH * (x);
	double nn = nH * (1.0 - x);
	double T = calc_temperature(P, x, q_pre, q_den);
	double rsqrd = 0, F_FUV = 0;
	if (P.star_on) {
		#pragma unroll
		for (int i = 0; i < 3; ++i) if (i < P.nd) rsqrd += (xc[i] - P.sxc[i]) * (xc[i] - P.sxc[i]) * P.dx[i] * P.dx[i];
		double Q_FUV = 0.5 * P.photonRate;
		F_FUV = rsqrd != 0 ? Q_FUV / (1.2e7 * 4 * P.pi * rsqrd) : 0;
	}
	double Av_FUV = 1.086 * P.dustXsec * TFLD(S.T, T_COL_DEN, id);
	double rate = 0;
	rate += th_fuvh(P, nH, Av_FUV, F_FUV);
	rate += th_irh(P, nH, Av_FUV, F_FUV);
	rate += P.crh * nH;
	TFLD(S.T, T_HEAT, id) = rate;
	rate = th_cooling(P, S, rate, ne, nn, nH, x, T);
	rate = soft_landing(rate, T, S.Tmin[id]);
	TFLD(S.T, T_RATE, id) = P.heating_amp * rate;
}
__global__ void __launch_bounds__(256) k_thermo_rates_fp64(Params P, State S) {
	if (TRG_BATCHED && P.batch) {
		const BatchTable& B = *P.batch;
		const int g = batch_slot(B.cell_off, B.G, blockIdx.x * (long long)blockDim.x);
		const long long lid = blockIdx.x * (long long)blockDim.x + threadIdx.x - B.cell_off[g];
		if (lid < B.P[g].N) b_thermo_rates_fp64(B.P[g], B.S[g], lid);
		return;
	}
	const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (id >= P.N) return;
	b_thermo_rates_fp64(P, S, id);
}

// Thermodynamics::integrate (pressure subcycling), Thermodynamics.cpp:266-337, non-wind cells.
// Thermodynamics::integrate (pressure subcycling), Thermodynamics.cpp:266-337,
// for one cell, split in three: the set-up (the first explicit step and the
// closed-form sub-cycle count, :285-310), the sub-cycles (:312-331) and the
// result (:334-335).  The work queue below runs the same three pieces.
struct ThermoCell {
	double qpre, ne, nn, nH, x, Tmin, heat, pre2temp, temp2pre, rate2dpre, dpre2rate, pressure, subT;
	int nsteps;  // sub-cycles still to run (0: none)
};
// false: a wind cell or one below the HII switch (nothing, or T_RATE = 0, to write)
// `count`: update the sub-cycle counters (the drain, which repeats the set-up
// of a queued cell, does not count it again)
__device__ __forceinline__ bool thermo_setup(const Params& P, const State& S, long long id, double h, ThermoCell& c,
                                             bool count = true) {
	int ijk[3];
	double xc[3];
	cell_ijk(P, id, ijk);
	cell_xc(P, ijk, xc);
	if (is_wind(P, id, ijk, xc)) return false;
	if (FLD(S.Q, ADV, id) < P.thermo_hii_switch) {
		if (S.H)
			for (int i = 0; i < NH; ++i) FLD(S.H, i, id) = 0;
		TFLD(S.T, T_RATE, id) = 0;
		return false;
	}
	const double dt = h * S.scal[0];
	double qden = FLD(S.Q, DEN, id), qpre = FLD(S.Q, PRE, id), x = FLD(S.Q, HII, id);
	c.qpre = qpre;
	c.x = x;
	c.Tmin = S.Tmin[id];
	double rate0 = TFLD(S.T, T_RATE, id);
	c.heat = TFLD(S.T, T_HEAT, id);
	c.nH = P.X * qden / P.hydrogenMass;
	c.ne = c.nH * (x);
	c.nn = c.nH * (1.0 - x);
	double dti = fabs(0.10 * FLD(S.U, PRE, id) / rate0);
	double mu_inv = P.X * (x + 1.0) + (1.0 - P.X) * 0.25;
	c.pre2temp = 1.0 / (mu_inv * P.specificGasConstant * qden);
	c.temp2pre = (mu_inv * P.specificGasConstant * qden);
	c.rate2dpre = smin(dt, dti) * (P.gamma - 1.0);
	c.dpre2rate = 1.0 / c.rate2dpre;
	c.pressure = qpre + rate0 * c.rate2dpre;
	c.subT = c.pressure * c.pre2temp;
	if (c.pressure < P.pfloor || c.subT < c.Tmin) {
		double pfl = smax(c.Tmin * c.temp2pre, P.pfloor);
		c.subT = pfl * c.pre2temp;
		c.pressure = pfl;
	}
	c.nsteps = 0;
	if (dt > dti) {
		double dtdti = dt / dti;
		int nsteps = dtdti - (int)dtdti > 0 ? (int)(dtdti + 1.0) : (int)(dtdti + 0.5);
		c.nsteps = nsteps - 1;
		if (count && P.stats_on) {
			stat_add(S.stats, TRG_STAT_THERMO_CELLS, 1u);
			stat_add(S.stats, TRG_STAT_THERMO_SUBCYCLES, (unsigned)c.nsteps);
			stat_max(S.stats, TRG_STAT_THERMO_MAX, (unsigned)c.nsteps);
		}
	}
	return true;
}
__device__ __forceinline__ void thermo_subcycles(const Params& P, const State& S, ThermoCell& c) {
	for (int i = 0; i < c.nsteps; ++i) {
		double r = th_cooling(P, S, c.heat, c.ne, c.nn, c.nH, c.x, c.subT);
		r = P.heating_amp * soft_landing(r, c.subT, c.Tmin);
		c.pressure += r * c.rate2dpre;
		c.subT = c.pressure * c.pre2temp;
		if (c.pressure < P.pfloor || c.subT < c.Tmin) {
			double pfl = smax(c.Tmin * c.temp2pre, P.pfloor);
			c.subT = pfl * c.pre2temp;
			c.pressure = pfl;
		}
	}
}
__device__ __forceinline__ void thermo_finish(const Params& P, const State& S, long long id, const ThermoCell& c) {
	TFLD(S.T, T_RATE, id) = (c.pressure - c.qpre) * c.dpre2rate;
	if (S.H) FLD(S.H, H_TOT, id) = TFLD(S.T, T_RATE, id);  // Thermodynamics.cpp:335
}

// Work queue of the uneven sub-cycles (single grids, when S.thq is set): a
// cell with at least S.thq_min sub-cycles is not run in place but appended
// to the queue with the bit length of its count (its bin); the bins are then
// laid out heaviest first, and a persistent kernel drains them, each warp
// taking 32 consecutive entries, so that the lanes of a warp run sub-cycle
// loops of similar length and the longest loops start first.
__device__ __forceinline__ int thq_bin(int nsteps) { return min(31 - __clz(nsteps), THQ_BINS - 1); }
__device__ __forceinline__ void thq_push(const State& S, long long id, int nsteps) {
	const unsigned slot = atomicAdd(&S.thq_ctl[THQ_COUNT], 1u);
	const int b = thq_bin(nsteps);
	S.thq[slot] = (int)id;
	S.thq_binof[slot] = (unsigned char)b;
	atomicAdd(&S.thq_ctl[THQ_BIN + b], 1u);
}

__device__ __forceinline__ void b_thermo_integrate_fp64(const Params& P, const State& S, long long id, double h,
                                                        bool queue) {
	if (!P.thermo_subcycling) return;
	ThermoCell c;
	if (!thermo_setup(P, S, id, h, c)) return;
	if (queue && c.nsteps >= S.thq_min) {
		thq_push(S, id, c.nsteps);
		return;
	}
	thermo_subcycles(P, S, c);
	thermo_finish(P, S, id, c);
}
__global__ void __launch_bounds__(256) k_thermo_integrate_fp64(Params P, State S, double h) {
	if (TRG_BATCHED && P.batch) {
		const BatchTable& B = *P.batch;
		const int g = batch_slot(B.cell_off, B.G, blockIdx.x * (long long)blockDim.x);
		const long long lid = blockIdx.x * (long long)blockDim.x + threadIdx.x - B.cell_off[g];
		if (lid < B.P[g].N) b_thermo_integrate_fp64(B.P[g], B.S[g], lid, h, false);
		return;
	}
	const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (id >= P.N) return;
	b_thermo_integrate_fp64(P, S, id, h, S.thq != nullptr);
}

// Bin offsets of the queue, heaviest bin first, and the drain head.
__global__ void k_thq_layout(State S) {
	if (threadIdx.x != 0) return;
	unsigned pos = 0;
	for (int b = THQ_BINS - 1; b >= 0; --b) {
		S.thq_ctl[THQ_CURSOR + b] = pos;
		pos += S.thq_ctl[THQ_BIN + b];
	}
	S.thq_ctl[THQ_HEAD] = 0;
}
// Entries into their bins' ranges (the order within a bin does not matter:
// the cells are independent).
__global__ void __launch_bounds__(256) k_thq_scatter(State S) {
	const unsigned n = S.thq_ctl[THQ_COUNT];
	for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
		const unsigned pos = atomicAdd(&S.thq_ctl[THQ_CURSOR + S.thq_binof[t]], 1u);
		S.thq_sorted[pos] = S.thq[t];
	}
}
// Persistent drain: warps take 32 entries at a time until the queue is empty.
// A cell whose count exceeds THQ_MAX_SUBCYCLES is not run: the error word
// reports it (the loop of every cell is bounded).
__global__ void __launch_bounds__(128) k_thq_drain(Params P, State S, double h) {
	const unsigned n = S.thq_ctl[THQ_COUNT];
	const int lane = threadIdx.x & 31;
	for (;;) {
		unsigned base = 0;
		if (lane == 0) base = atomicAdd(&S.thq_ctl[THQ_HEAD], 32u);
		base = __shfl_sync(0xffffffffu, base, 0);
		if (base >= n) return;
		const unsigned t = base + lane;
		if (t < n) {
			const long long id = S.thq_sorted[t];
			ThermoCell c;
			if (thermo_setup(P, S, id, h, c, false)) {
				if (c.nsteps > THQ_MAX_SUBCYCLES) {
					atomicOr(S.err, ERRB_SUBCYCLE);
				} else {
					thermo_subcycles(P, S, c);
					thermo_finish(P, S, id, c);
				}
			}
		}
	}
}

// Thermodynamics::updateSourceTerms (Thermodynamics.cpp:478-485) then advSolution + fixSolution.
__device__ __forceinline__ void b_thermo_update_fp64(const Params& P, const State& S, long long id, double h, int mode) {
	// every load is issued before the first store, so that they overlap
	double u[7];
#pragma unroll
	for (int i = 0; i < NU; ++i) u[i] = FLD(S.U, i, id);
	const double rate = TFLD(S.T, T_RATE, id);
	int ijk[3];
	double xc[3];
	cell_ijk(P, id, ijk);
	cell_xc(P, ijk, xc);
	double udot_pre = 0;
	if (!is_wind(P, id, ijk, xc)) {
		udot_pre += rate;
		TFLD(S.T, T_RATE, id) = 0;
		TFLD(S.T, T_HEAT, id) = 0;
	}
	if (mode == 1) {
		FLD(S.UDOT, PRE, id) += udot_pre;
		return;
	}
	const double dt = h * S.scal[0];
#pragma unroll
	for (int i = 0; i < NU; ++i) u[i] = u[i] + dt * (i == PRE ? udot_pre : 0.0);
	if (!fix_solution(P, u)) atomicOr(S.err, ERRB_NAN);
#pragma unroll
	for (int i = 0; i < NU; ++i) FLD(S.U, i, id) = u[i];
	if (mode == 2) store_fixed_q(P, S, id, u);
}
__global__ void __launch_bounds__(256) k_thermo_update_fp64(Params P, State S, double h, int mode) {
	if (TRG_BATCHED && P.batch) {
		const BatchTable& B = *P.batch;
		const int g = batch_slot(B.cell_off, B.G, blockIdx.x * (long long)blockDim.x);
		const long long lid = blockIdx.x * (long long)blockDim.x + threadIdx.x - B.cell_off[g];
		if (lid < B.P[g].N) b_thermo_update_fp64(B.P[g], B.S[g], lid, h, mode);
		return;
	}
	const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (id >= P.N) return;
	b_thermo_update_fp64(P, S, id, h, mode);
}

// Thermodynamics::fillHeatingArrays (Thermodynamics.cpp:419-461) after its
// rayTrace (the column-density sweep, launched before), non-wind cells.
// Single grids only.
__global__ void __launch_bounds__(256) k_heating_arrays_fp64(Params P, State S) {
	const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (id >= P.N) return;
	int ijk[3];
	double xc[3];
	cell_ijk(P, id, ijk);
	cell_xc(P, ijk, xc);
	if (is_wind(P, id, ijk, xc)) return;
	if (FLD(S.Q, ADV, id) < P.thermo_hii_switch) {
		for (int i = 0; i < NH; ++i) FLD(S.H, i, id) = 0;
		return;
	}
	double nH = P.X * FLD(S.Q, DEN, id) / P.hydrogenMass;
	double x = FLD(S.Q, HII, id);
	double ne = x * nH;
	double nn = (1.0 - x) * nH;
	double T = calc_temperature(P, x, FLD(S.Q, PRE, id), FLD(S.Q, DEN, id));
	double rsqrd = 0, F_FUV = 0;
	if (P.star_on) {
#pragma unroll
		for (int i = 0; i < 3; ++i)
			if (i < P.nd) rsqrd += (xc[i] - P.sxc[i]) * (xc[i] - P.sxc[i]) * P.dx[i] * P.dx[i];
		double Q_FUV = 0.5 * P.photonRate;
		F_FUV = rsqrd != 0 ? Q_FUV / (1.2e7 * 4 * P.pi * rsqrd) : 0;
	}
	double Av_FUV = 1.086 * P.dustXsec * TFLD(S.T, T_COL_DEN, id);
	FLD(S.H, H_FUVH, id) = th_fuvh(P, nH, Av_FUV, F_FUV);
	FLD(S.H, H_IRH, id) = th_irh(P, nH, Av_FUV, F_FUV);
	FLD(S.H, H_CRH, id) = P.crh * nH;
	FLD(S.H, H_IMLC, id) = -th_imlc(P, ne, T);
	FLD(S.H, H_NMLC, id) = -th_nmlc(P, ne, nn, T);
	FLD(S.H, H_CEHI, id) = -th_cxhi(P, S, nH, x, T);
	FLD(S.H, H_CIEC, id) = -th_ciec(P, ne, T);
	FLD(S.H, H_NMC, id) = -th_nmc(P, nH, x, T);
	FLD(S.H, H_TOT, id) += FLD(S.H, H_RHII, id) + FLD(S.H, H_EUVH, id);
}

// ----------------------------------------------------------------- time step
__device__ __forceinline__ unsigned long long dbits(double v) { return (unsigned long long)__double_as_longlong(v); }

__device__ __forceinline__ double block_min(double v) {
	__shared__ double red[32];
	for (int o = 16; o > 0; o >>= 1) v = smin(v, __shfl_down_sync(0xffffffffu, v, o));
	int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	if (lane == 0) red[wid] = v;
	__syncthreads();
	if (wid == 0) {
		int nw = (blockDim.x + 31) >> 5;
		v = lane < nw ? red[lane] : 1.0e308;
		for (int o = 16; o > 0; o >>= 1) v = smin(v, __shfl_down_sync(0xffffffffu, v, o));
	}
	return v;
}

// Hydrodynamics::calculateTimeStep (Hydro.cpp:77-89), Radiation::calculateTimeStep
// (Radiation.cpp:298-351) and Thermodynamics::calculateTimeStep
// (Thermodynamics.cpp:463-476) as one pass.  Minima of positive doubles are
// exact and order independent; they are combined with atomicMin on the bit
// pattern.  first_cell: the first non-wind cell in causal order on the first
// radiation call (the reference's static `once`), else -1.
//
// With cons_part set (single grids only) the pass also forms the block's
// partial of the global FP64 mass and energy sums of the state (U), the
// conservation check of the step.
__device__ __forceinline__ void b_dt_reduce_fp64(const Params& P, const State& S, long long id, long long first_cell,
                                                 double* cons_part);
__global__ void __launch_bounds__(256) k_dt_reduce_fp64(Params P, State S, long long first_cell) {
	if (TRG_BATCHED && P.batch) {
		// grid ranges are padded to whole blocks: the block reduction stays within one grid
		const BatchTable& B = *P.batch;
		const int g = batch_slot(B.cell_off, B.G, blockIdx.x * (long long)blockDim.x);
		const long long lid = blockIdx.x * (long long)blockDim.x + threadIdx.x - B.cell_off[g];
		b_dt_reduce_fp64(B.P[g], B.S[g], lid, first_cell >= 0 ? B.first_cell[g] : -1, nullptr);
		return;
	}
	b_dt_reduce_fp64(P, S, blockIdx.x * (long long)blockDim.x + threadIdx.x, first_cell, S.cons_part);
}
__device__ __forceinline__ void b_dt_reduce_fp64(const Params& P, const State& S, long long id, long long first_cell,
                                                 double* cons_part) {
	double th = 1.0e308, tr = 1.0e308, tt = 1.0e308;
	DD cm = {0.0, 0.0}, ce = {0.0, 0.0};
	if (cons_part && id < P.N) {
		int ijk[3];
		double xc[3];
		cell_ijk(P, id, ijk);
		cell_xc(P, ijk, xc);
		const double vol = cell_volume_rn(P, xc[0]);
		cm = dd_prod(FLD(S.U, DEN, id), vol);
		ce = dd_prod(FLD(S.U, PRE, id), vol);
	}
	if (id < P.N) {
		double q_den = FLD(S.Q, DEN, id), q_pre = FLD(S.Q, PRE, id), q_hii = FLD(S.Q, HII, id);
		double inv_t = 0;
		double ss = sqrt(P.gamma * q_pre / q_den);
		#pragma unroll
#ifdef TRG_FAST_MATH
		for (int dim = 0; dim < 3; ++dim) if (dim < P.nd) inv_t += (fabs(FLD(S.Q, VEL + dim, id)) + ss) * (1.0 / P.dx[dim]);
#else
		for (int dim = 0; dim < 3; ++dim) if (dim < P.nd) inv_t += (fabs(FLD(S.Q, VEL + dim, id)) + ss) / P.dx[dim];
#endif
		if (inv_t == 0) inv_t = 1.0 / P.dt_max;
		th = 0.5 / inv_t;
		int ijk[3];
		double xc[3];
		cell_ijk(P, id, ijk);
		cell_xc(P, ijk, xc);
		if (P.radiation_on && P.star_on && !is_wind(P, id, ijk, xc)) {
			double dt_max = P.dt_max;
			double dtc = dt_max, dt1 = dt_max, dt2 = dt_max, dt3 = dt_max, dt4 = dt_max;
			if (P.coupling == CP_NEQ) {
				double heat = RFLD(S.R, R_HEAT, id);
				if (heat != 0) dtc = fabs(FLD(S.U, PRE, id) / heat);
			}
			if (P.K1 != 0.0) {
				double T = calc_temperature(P, q_hii, q_pre, q_den);
				if (id == first_cell)
					dt1 = P.K1 * P.hydrogenMass / (P.X * q_den * spline_eval(S.tables->rad_recomb, T));
				else if (q_hii != 0)
					dt1 = P.K1 * P.hydrogenMass / (P.X * q_den * q_hii * spline_eval(S.tables->rad_recomb, T));
			}
			if (P.K3 != 0.0 || P.K4 != 0.0) {
				double nH = P.X * q_den / P.hydrogenMass;
				double nHI = (1.0 - q_hii) * nH;
				double A_pi = photoionisation_rate(nHI, RFLD(S.R, R_TAU, id), RFLD(S.R, R_DTAU, id), S.shellVol[id], P.photonRate);
				double Tq = calc_temperature(P, q_hii, q_pre, q_den);
				double A_ci = collisional_ionisation_rate(P, Tq);
				double A_rr = spline_eval(S.tables->rad_recomb, Tq);
				double fracRate = (1.0 - q_hii) * (A_pi + q_hii * nH * A_ci) - q_hii * q_hii * nH * A_rr;
				if (P.K3 != 0.0 && fracRate != 0.0) dt3 = P.K3 * smax(0.05, 1.0 - q_hii) / fabs(fracRate);
				if (P.K4 != 0.0 && fracRate != 0.0) dt4 = P.K4 * 1.0 / fabs(fracRate);
			}
			tr = smin(dt_max, smin(dtc, smin(dt1, smin(dt2, smin(dt3, dt4)))));
			if (tr == 0.0 || tr != tr || isinf(tr)) atomicOr(S.err, ERRB_DT);
		}
		if (P.cooling_on) {
			double rate = TFLD(S.T, T_RATE, id);
			if (rate != 0) {
				double frac = P.thermo_subcycling ? 1.0 : 0.1;
				tt = fabs(frac * FLD(S.U, PRE, id) / rate);
			}
		}
	}
	if (cons_part) block_cons_partial(cm, ce, cons_part, blockIdx.x);
	th = block_min(th);
	__syncthreads();
	tr = block_min(tr);
	__syncthreads();
	tt = block_min(tt);
	if (threadIdx.x == 0) {
		unsigned long long* slots = reinterpret_cast<unsigned long long*>(S.scal + 2);
		atomicMin(&slots[0], dbits(th));
		atomicMin(&slots[1], dbits(tr));
		atomicMin(&slots[2], dbits(tt));
	}
}

// Torch::calculateTimeStep + the dt of Torch::fullStep (Torch.cpp:304-339, :394).
__device__ __forceinline__ void b_dt_finalize(const Params& P, const State& S, double dt_next, int first_time, int step);
__global__ void k_dt_finalize(Params P, State S, double dt_next, int first_time, int step) {
	if (TRG_BATCHED && P.batch) {
		const int g = blockIdx.x * blockDim.x + threadIdx.x;
		if (g < P.batch->G) b_dt_finalize(P.batch->P[g], P.batch->S[g], dt_next, first_time, step);
		return;
	}
	b_dt_finalize(P, S, dt_next, first_time, step);
}
__device__ __forceinline__ void b_dt_finalize(const Params& P, const State& S, double dt_next, int first_time, int step) {
	double dt;
	if (first_time) {
		dt = P.dt_max * 1.0e-20;
	} else {
		double dt_hydro = smin(S.scal[2], P.dt_max);
		double dt_rad = dt_hydro, dt_thermo = dt_hydro;
		if (P.radiation_on) dt_rad = P.star_on ? smin(P.dt_max, S.scal[3]) : P.dt_max;
		if (P.cooling_on) dt_thermo = smin(P.dt_max, S.scal[4]);
		dt = smin(smin(dt_hydro, dt_rad), dt_thermo);
	}
	dt = smin(dt_next, dt);
	S.scal[0] = dt;
	if (S.dt_hist && step >= 0) S.dt_hist[step] = dt;
}

__global__ void k_time_advance(Params P, State S) {
	if (TRG_BATCHED && P.batch) {
		const int g = blockIdx.x * blockDim.x + threadIdx.x;
		if (g < P.batch->G) P.batch->S[g].scal[1] += P.batch->S[g].scal[0];
		return;
	}
	S.scal[1] += S.scal[0];
}

__device__ __forceinline__ void b_dt_reset(const Params& P, const State& S) {
	unsigned long long big = (unsigned long long)__double_as_longlong(P.dt_max);
	unsigned long long* slots = reinterpret_cast<unsigned long long*>(S.scal + 2);
	slots[0] = big;
	slots[1] = big;
	slots[2] = big;
}
__global__ void k_dt_reset(Params P, State S) {
	if (TRG_BATCHED && P.batch) {
		const int g = blockIdx.x * blockDim.x + threadIdx.x;
		if (g < P.batch->G) b_dt_reset(P.batch->P[g], P.batch->S[g]);
		return;
	}
	b_dt_reset(P, S);
}

// ------------------------------------------- FP64 fallback of the FP32 form
// A hydro sub-step of the FP32 form keeps FP64 arithmetic for the cells whose
// stencil (two cells either side along each axis) spans a pressure ratio
// above `contrast`: across such a jump (the blast wave the star drives into
// the neutral gas) the FP32 flux differences keep too few digits.  The flag
// pass lists those cells; their faces are computed in FP64 from the
// sub-step's primitives before the FP32 pass overwrites Q, and their update
// (FP64, with Q of the result) follows the FP32 pass, overwriting its values.
__device__ __forceinline__ long long clamp_nb(const Params& P, const int* ijk, int dim, int off) {
	int t[3] = {ijk[0], ijk[1], ijk[2]};
	const int n = ncell(P, dim);
	int v = (dim == 0 ? t[0] : dim == 1 ? t[1] : t[2]) + off;
	v = v < 0 ? 0 : (v >= n ? n - 1 : v);
	if (dim == 0) t[0] = v;
	else if (dim == 1) t[1] = v;
	else t[2] = v;
	return flat_id(P, t[0], t[1], t[2]);
}
// The flag of a cell: its pressure and those of its neighbours up to 2 cells
// away along each axis (indices clamped to the grid) span a ratio above
// `contrast`.  A CTA owns a 32 x 8 tile of columns and marches along z through
// FB_ZCHUNK planes: each plane's pressures, with two clamped cells of halo in x
// and y, are staged in shared memory once; the z neighbours come from a window
// of the column's pressures kept in registers.
__global__ void __launch_bounds__(256) k_fb_flags(Params P, State S, double contrast) {
	__shared__ double tile[8 + 4][32 + 4];
	const int lane = threadIdx.x & 31, row = threadIdx.x >> 5;
	const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 8;
	const int x = x0 + lane, y = y0 + row;
	const int nx = P.nx, ny = P.ny, nz = P.nz, nd = P.nd;
	const int xc = min(x, nx - 1), yc = min(y, ny - 1);
	const bool in = x < nx && y < ny;
	const int z0 = blockIdx.z * FB_ZCHUNK, z1 = min(z0 + FB_ZCHUNK, nz);
	const double* pre = S.Q + (long long)PRE * P.N;
	auto at = [&](int i, int j, int k) {
		i = i < 0 ? 0 : (i >= nx ? nx - 1 : i);
		j = j < 0 ? 0 : (j >= ny ? ny - 1 : j);
		k = k < 0 ? 0 : (k >= nz ? nz - 1 : k);
		return pre[i + (long long)nx * (j + (long long)ny * k)];
	};
	// the column's pressures at z - 2 .. z + 2 (clamped)
	double w0 = 0, w1 = 0, w2 = 0, w3 = 0;
	if (nd > 2) {
		w0 = at(xc, yc, z0 - 2);
		w1 = at(xc, yc, z0 - 1);
		w2 = at(xc, yc, z0);
		w3 = at(xc, yc, z0 + 1);
	}
	for (int z = z0; z < z1; ++z) {
		for (int k = threadIdx.x; k < 12 * 36; k += 256) {
			const int ly = k / 36, lx = k - ly * 36;
			tile[ly][lx] = at(x0 + lx - 2, nd > 1 ? y0 + ly - 2 : 0, z);
		}
		const double w4 = nd > 2 ? at(xc, yc, z + 2) : 0.0;
		__syncthreads();
		const int lx = lane + 2, ly = row + 2;
		const double pc = tile[ly][lx];
		double pmin = pc, pmax = pc;
		pmin = smin(smin(smin(pmin, tile[ly][lx - 1]), smin(tile[ly][lx - 2], tile[ly][lx + 1])), tile[ly][lx + 2]);
		pmax = smax(smax(smax(pmax, tile[ly][lx - 1]), smax(tile[ly][lx - 2], tile[ly][lx + 1])), tile[ly][lx + 2]);
		if (nd > 1) {
			pmin = smin(smin(smin(pmin, tile[ly - 1][lx]), smin(tile[ly - 2][lx], tile[ly + 1][lx])), tile[ly + 2][lx]);
			pmax = smax(smax(smax(pmax, tile[ly - 1][lx]), smax(tile[ly - 2][lx], tile[ly + 1][lx])), tile[ly + 2][lx]);
		}
		if (nd > 2) {
			pmin = smin(smin(smin(pmin, w0), smin(w1, w3)), w4);
			pmax = smax(smax(smax(pmax, w0), smax(w1, w3)), w4);
			w0 = w1;
			w1 = w2;
			w2 = w3;
			w3 = w4;
		}
		__syncthreads();  // the tile is read: the next plane may overwrite it
		const bool f = in && pmax > contrast * pmin;
		const long long id = xc + (long long)nx * (yc + (long long)ny * z);
		if (in) S.fb_flag[id] = f ? 1 : 0;
		const unsigned ballot = __ballot_sync(0xffffffffu, f);
		if (!ballot) continue;
		const int leader = __ffs(ballot) - 1;
		unsigned base = 0;
		if (lane == leader) base = atomicAdd(S.fb_count, (unsigned)__popc(ballot));
		base = __shfl_sync(0xffffffffu, base, leader);
		if (f) S.fb_list[base + __popc(ballot & ((1u << lane) - 1))] = (int)id;
		if (P.stats_on && lane == leader) atomicAdd(S.stats + TRG_STAT_FP64_CELLS, (unsigned long long)__popc(ballot));
	}
}
// FP64 face fluxes (into S.F) of every listed cell's faces.
__global__ void __launch_bounds__(128) k_fb_faces(Params P, State S) {
	const unsigned n = *S.fb_count;
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * 2 * P.nd;
	     t += (long long)gridDim.x * blockDim.x) {
		const long long id = S.fb_list[t / (2 * P.nd)];
		const int k = (int)(t % (2 * P.nd)), dim = k >> 1;
		int ijk[3];
		cell_ijk(P, id, ijk);
		long long fl, fr;
		face_ids(P, ijk, dim, fl, fr);
		b_faces_fp64(P, S, (k & 1) ? fr : fl, dim);
	}
}
// FP64 update of every listed cell, U -> U1, with Q of the result.
__global__ void __launch_bounds__(256) k_fb_update(Params P, State S, double h) {
	const unsigned n = *S.fb_count;
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
		b_hydro_update_fp64(P, S, S.fb_list[t], h, 0, 1, 2);
}

}  // namespace TRG_KNS
}  // namespace trg
