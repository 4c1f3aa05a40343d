/*
 * CPU oracle for the TORCH operator-split timestep.  TEST INFRASTRUCTURE ONLY
 * (see torch_oracle.h): a sequential plain-C restatement of the reference,
 * written so that every floating-point operation happens in the reference's
 * order.  Each function cites the reference file:line it restates.  Build with
 * -ffp-contract=off (oracle/Makefile) so that no multiply-add is fused.
 */
#include "torch_oracle.h"

#include <math.h>
#include <stdarg.h>

/* Transcendentals of the step.  Default: the host libm (as the reference).
 * With ORACLE_PORTABLE_MATH: the IEEE-only implementations of
 * torch_b200/csrc/trg_math.h, which the FP64 GPU kernels use too - that build
 * is the GPU's bit-exact CPU twin.  Set-up code (tables, unit conversion)
 * always uses the host libm, like both the reference and the GPU library. */
#ifdef ORACLE_PORTABLE_MATH
#include "../torch_b200/csrc/trg_math.h"
#define m_exp trg_exp
#define m_log trg_log
#define m_log10 trg_log10
#define m_pow trg_pow
void orc_set_libm_noise(double fraction) { (void)fraction; }
#else
/* Host libm, with an optional test hook (orc_set_libm_noise): a fixed,
 * input-determined fraction of the results moved by one ulp, to show how the
 * step amplifies single-ulp differences between math libraries. */
#include <stdint.h>
#include <string.h>
static double g_libm_noise = 0.0;
void orc_set_libm_noise(double fraction) { g_libm_noise = fraction; }
static double libm_noise(double x, double salt, double r) {
	if (g_libm_noise <= 0.0 || !isfinite(r) || r == 0.0) return r;
	uint64_t b;
	double k = x + salt;
	memcpy(&b, &k, sizeof b);
	b *= 0xff51afd7ed558ccdULL; /* 64-bit mixing (multiply, xor-shift) */
	b ^= b >> 33;
	b *= 0xc4ceb9fe1a85ec53ULL;
	b ^= b >> 33;
	if ((double)(b >> 11) * 0x1p-53 >= g_libm_noise) return r;
	return nextafter(r, (b & 1) ? INFINITY : -INFINITY);
}
static double m_exp(double x) { return libm_noise(x, 0.0, exp(x)); }
static double m_log(double x) { return libm_noise(x, 1.0, log(x)); }
static double m_log10(double x) { return libm_noise(x, 2.0, log10(x)); }
static double m_pow(double x, double y) { return libm_noise(x * 1.000001 + y, 3.0, pow(x, y)); }
#endif
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

enum { DEN = 0, PRE = 1, HII = 2, ADV = 3, VEL = 4, NU = 7 };
enum { R_HII_A = 0, R_TAU, R_TAU_A, R_DTAU, R_DTAU_A, R_HEAT, NR };
enum { T_COL_DEN = 0, T_DCOL_DEN, T_HEAT, T_RATE, NT };
enum { G_CART = 0, G_CYL = 1, G_SPH = 2 };
enum { BC_FREE = 0, BC_REFLECTING = 1, BC_OUTFLOW = 2, BC_INFLOW = 3, BC_PERIODIC = 4 };
enum { CP_TTI = 0, CP_NEQ = 1, CP_OFF = 2 };
enum { RS_HLLC = 0, RS_ROTATED = 1, RS_HLL = 2 };
enum { COMP_HYDRO = 0, COMP_RAD = 1, COMP_THERMO = 2 };

#define ORC_ERR_NAN 1
#define ORC_ERR_PICARD 2
#define ORC_ERR_DT 3
#define ORC_ERR_FLUX 4
#define ORC_ERR_PARAM 5

/* IEEE comparisons exactly as std::min/std::max (libstdc++): min(a,b) = b<a?b:a. */
static inline double smin(double a, double b) { return (b < a) ? b : a; }
static inline double smax(double a, double b) { return (a < b) ? b : a; }

/* ---------------------------------------------------------------- units --- */
/* Converter, src/Torch/Converter.cpp:7-63. */
typedef struct { double M, L, T; } conv_t;

static void conv_init(conv_t* c) {
	c->M = 1.0 * 2.0e33;          /* MO_2_G(1.0)   Converter.cpp:89-91 */
	c->L = 14.6 * 3.09e18;        /* PC_2_CM(14.6) Converter.cpp:81-83 */
	c->T = 10000.0 * 3.15569e7;   /* YR_2_S(1e4)   Converter.cpp:73-75 */
}

static void conv_set_dpt(conv_t* c, double rho, double pressure, double time) {
	/* Converter::set_rho_pressure_time, Converter.cpp:17-26 */
	double rho_0 = (rho > 0) ? rho : c->M / (c->L * c->L * c->L);
	double pressure_0 = (pressure > 0) ? pressure : rho_0 * c->L * c->L / (c->T * c->T);
	double time_0 = (time > 0) ? time : c->T;
	c->T = time_0;
	c->M = sqrt((pressure_0 / rho_0) * pressure_0 * pressure_0) * c->T * c->T * c->T;
	c->L = sqrt(pressure_0 / rho_0) * c->T;
}

static double conv_units(const conv_t* c, double val, double mi, double li, double ti, int to_code) {
	/* Converter::convertCodeUnits, Converter.cpp:36-63 */
	double MM = mi >= 0 ? c->M : 1.0 / c->M;
	MM = to_code ? 1.0 / MM : MM;
	double LL = li >= 0 ? c->L : 1.0 / c->L;
	LL = to_code ? 1.0 / LL : LL;
	double TT = ti >= 0 ? c->T : 1.0 / c->T;
	TT = to_code ? 1.0 / TT : TT;
	int im = (int)fabs(mi), il = (int)fabs(li), it = (int)fabs(ti);
	double result = val;
	while (im >= 1 || il >= 1 || it >= 1) {
		if (im-- >= 1) result *= MM;
		if (il-- >= 1) result *= LL;
		if (it-- >= 1) result *= TT;
	}
	double left = fabs(mi) - (int)fabs(mi);
	if (left != 0) result *= pow(MM, left);
	left = fabs(li) - (int)fabs(li);
	if (left != 0) result *= pow(LL, left);
	left = fabs(ti) - (int)fabs(ti);
	if (left != 0) result *= pow(TT, left);
	return result;
}
#define TO_CODE(c, v, m, l, t) conv_units((c), (v), (m), (l), (t), 1)

/* -------------------------------------------------------------- splines --- */
/* SplineData, src/Integrators/SplineData.cpp:15-151. */
typedef struct {
	int n, log_mode;
	double x[32], y[32], y2[32];
	double min_slope, max_slope;
} spline_t;

static void spline_second_derivs(spline_t* s) {
	/* SplineData::spline with natural ends (yp1 = ypn = 1e99), SplineData.cpp:15-55 */
	int n = s->n, i, k;
	double u[32], p, qn, sig, un;
	const double* x = s->x;
	const double* f = s->y;
	double* y2 = s->y2;
	for (i = 0; i < n; ++i) y2[i] = 0.0;
	for (i = 0; i < n - 1; ++i) u[i] = 0.0;
	y2[0] = 0.0;
	u[0] = 0.0;
	for (i = 1; i < n - 1; i++) {
		sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1]);
		p = sig * y2[i - 1] + 2.0;
		y2[i] = (sig - 1.0) / p;
		u[i] = (f[i + 1] - f[i]) / (x[i + 1] - x[i]) - (f[i] - f[i - 1]) / (x[i] - x[i - 1]);
		u[i] = (6.0 * u[i] / (x[i + 1] - x[i - 1]) - sig * u[i - 1]) / p;
	}
	qn = 0.0;
	un = 0.0;
	y2[n - 1] = (un - qn * u[n - 2]) / (qn * y2[n - 2] + 1.0);
	for (k = n - 2; k >= 0; k--)
		y2[k] = y2[k] * y2[k + 1] + u[k];
}

static void spline_init(spline_t* s, const double* x, const double* y, int n, int log_mode) {
	/* LinearSplineData / LogSplineData constructors, SplineData.cpp:83-101, :121-140 */
	s->n = n;
	s->log_mode = log_mode;
	for (int i = 0; i < n; ++i) { s->x[i] = x[i]; s->y[i] = y[i]; }
	spline_second_derivs(s);
	if (log_mode) {
		s->min_slope = (s->y[1] - s->y[0]) / (s->x[1] - s->x[0]);
		s->max_slope = (s->y[n - 1] - s->y[n - 2]) / (s->x[n - 1] - s->x[n - 2]);
	} else {
		s->min_slope = (log10(s->y[1]) - log10(s->y[0])) / (log10(s->x[1]) - log10(s->x[0]));
		s->max_slope = (log10(s->y[n - 1]) - log10(s->y[n - 2])) / (log10(s->x[n - 1]) - log10(s->x[n - 2]));
	}
}

static double splint(const spline_t* s, double x2) {
	/* SplineData::splint, SplineData.cpp:57-81 */
	int klo = 0, khi = s->n - 1, k;
	while (khi - klo > 1) {
		k = (khi + klo) >> 1;
		if (s->x[k] > x2) khi = k;
		else klo = k;
	}
	double h = s->x[khi] - s->x[klo];
	double a = (s->x[khi] - x2) / h;
	double b = (x2 - s->x[klo]) / h;
	return a * s->y[klo] + b * s->y[khi] + ((a * a * a - a) * s->y2[klo] + (b * b * b - b) * s->y2[khi]) * (h * h) / 6.0;
}

static double spline_eval(const spline_t* s, double x) {
	/* LinearSplineData::interpolate :108-119, LogSplineData::interpolate :142-151 */
	int n = s->n;
	if (s->log_mode) {
		if (x > s->x[n - 1]) return s->y[n - 1] + s->max_slope * (x - s->x[n - 1]);
		else if (x < s->x[0]) return s->y[0] + s->min_slope * (x - s->x[0]);
		return splint(s, x);
	}
	if (x > s->x[n - 1]) return s->y[n - 1] * m_pow(x / s->x[n - 1], s->max_slope);
	else if (x < s->x[0]) return s->y[0] * m_pow(x / s->x[0], s->min_slope);
	return splint(s, x);
}

/* ---------------------------------------------------------------- state --- */
struct orc_ctx {
	orc_params p;
	conv_t cv;
	/* Constants in code units (Constants.cpp:27-40) */
	double hydrogenMass, specificGasConstant, boltzmannConst, rydbergEnergy, dustXsec, pi;
	double voronov_A, voronov_X, voronov_K, voronov_P, voronov_DE;
	/* TorchParameters after initialise (Parameters.cpp:9-27) */
	double tmax, dt_max, side, dfloor, pfloor, tfloor;
	double photoIonXsec, alphaB, photonEnergy, photonRate, massLossRate, windVelocity;
	int nd, nx, ny, nz, geometry, order, ng;
	int lbc[3], rbc[3];
	long N;
	double dx[3];
	double gamma, X;
	/* star (Star.cpp:13-40, :42-51) */
	double sxc[3];
	double mdot, edot;
	/* cells */
	double* U;     /* [7][N] */
	double* Q;     /* [7][N] */
	double* W;     /* [7][N] */
	double* UDOT;  /* [7][N] */
	double* R;     /* [6][N] */
	double* T;     /* [4][N] */
	double* Tmin;  /* [N]   */
	double* grav;  /* [3][N] */
	double* vol;   /* [N]   */
	double* ds;    /* [N]   */
	double* shellVol;
	int* nbr;      /* [4][N] interior index or -1 */
	double* nbw;   /* [4][N] */
	/* reconstructed states per cell per dim: [3][7][N] */
	double* QL;
	double* QR;
	/* face fluxes per dim: F[dim][7][faces] with faces = (n_dim+1) lines */
	double* F[3];
	long nfaces[3];
	/* causal lists */
	int* causal; long ncausal;
	int* wind; long nwind;
	int* nonwind; long nnonwind;
	int starCell;
	/* ghost storage along each dim: [dim][side][layer][7][face cells] */
	double* ghostQ[3][2];
	long gcount[3];
	/* splines */
	spline_t rad_recomb, rad_cool, th_cxhi, th_recomb;
	/* thermo constants (Thermodynamics.cpp:24-57) */
	double z0, th_excess, T1, T2, T3, T4, imlc, nmlc, ciec_minT, ciec, cxhi_damp, n0, nmc;
	double fuvh_a, fuvh_b, fuvh_c, irh_a, irh_b, crh, th_Tmin;
	/* driver state */
	double time;
	int first_time, rad_once, stepCounter;
	int active[3], nactive;
	char err[512];
};

static int fail(orc_ctx* c, int code, const char* fmt, ...) {
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(c->err, sizeof(c->err), fmt, ap);
	va_end(ap);
	return code;
}

#define FLD(a, f, i) ((a)[(long)(f) * c->N + (i)])

static inline void cell_coords(const orc_ctx* c, long id, int* ijk) {
	ijk[0] = (int)(id % c->nx);
	ijk[1] = (int)((id / c->nx) % c->ny);
	ijk[2] = (int)(id / ((long)c->nx * c->ny));
}
static inline long flat(const orc_ctx* c, int i, int j, int k) {
	return i + (long)c->nx * (j + (long)c->ny * k);
}
static inline void cell_xc(const orc_ctx* c, long id, double* xc) {
	/* Grid::buildCells, Grid.cpp:525-548: centre at index+0.5 for dims < nd, 0 otherwise */
	int ijk[3];
	cell_coords(c, id, ijk);
	for (int i = 0; i < 3; ++i)
		xc[i] = (double)ijk[i];
	for (int i = 0; i < c->nd; ++i)
		xc[i] += 0.5;
}
static inline int ncell_dim(const orc_ctx* c, int d) { return d == 0 ? c->nx : (d == 1 ? c->ny : c->nz); }

/* -------------------------------------------------------------- geometry --- */
static double cell_volume(const orc_ctx* c, double rc) {
	/* Grid::computeCellVolume, Grid.cpp:876-905 */
	double PI = 3.14159265359, volume = 0, r1, r2;
	const double* dx = c->dx;
	if (c->geometry == G_CART) {
		volume = 1.0;
		for (int i = 0; i < c->nd; ++i) volume *= dx[i];
	} else if (c->geometry == G_CYL) {
		r2 = rc * dx[0] + 0.5 * dx[0];
		r1 = rc * dx[0] - 0.5 * dx[0];
		volume = PI * (r2 - r1) * (r2 + r1);
		if (c->nd >= 2) volume *= dx[1];
	} else if (c->geometry == G_SPH) {
		r2 = rc * dx[0] + 0.5 * dx[0];
		r1 = rc * dx[0] - 0.5 * dx[0];
		volume = 4.0 * PI * (r2 - r1) * (r2 * r2 + r1 * r2 + r1 * r1) / 3.0;
	}
	return volume;
}

static double join_area(const orc_ctx* c, const double* xj, int dim) {
	/* Grid::computeJoinArea, Grid.cpp:846-874 */
	double PI = 3.14159265359, area = 0, r1, r2;
	const double* dx = c->dx;
	if (c->geometry == G_CART) {
		area = 1.0;
		for (int i = 0; i < c->nd; ++i)
			if (i != dim) area *= dx[i];
	} else if (c->geometry == G_CYL) {
		if (dim == 0) {
			r1 = xj[0] * dx[0];
			area = 2.0 * PI * r1;
			if (c->nd >= 2) area *= dx[1];
		} else if (dim == 1) {
			r1 = xj[0] * dx[0] - 0.5 * dx[0];
			r2 = xj[0] * dx[0] + 0.5 * dx[0];
			area = PI * (r2 - r1) * (r2 + r1);
		}
	} else if (c->geometry == G_SPH) {
		r1 = xj[0] * dx[0];
		area = 4.0 * PI * r1 * r1;
	}
	return area;
}

/* Area of the face on the left (side 0) or right (side 1) of interior cell id
 * along dim.  The join coordinate is the right-hand cell's centre moved back by
 * half a cell along dim (Grid::weakLink, Grid.cpp:405-411). */
static double face_area(const orc_ctx* c, long id, int dim, int side) {
	double xj[3];
	cell_xc(c, id, xj);
	xj[dim] += side ? 0.5 : -0.5;
	return join_area(c, xj, dim);
}

/* ----------------------------------------------------------- causal order --- */
static int within(const orc_ctx* c, const int* x) {
	return x[0] >= 0 && x[0] < c->nx && x[1] >= 0 && x[1] < c->ny && x[2] >= 0 && x[2] < c->nz;
}

static void next_snake(const orc_ctx* c, const int* from, const int* src, int dxc, int dyc, int dzc, int* nxt) {
	/* Grid::nextSnakeCoords, Grid.cpp:255-283 */
	if (from[0] + dxc >= 0 && from[0] + dxc < c->nx) {
		nxt[0] = from[0] + dxc; nxt[1] = from[1]; nxt[2] = from[2];
	} else if (from[1] + dyc >= 0 && from[1] + dyc < c->ny) {
		nxt[0] = src[0]; nxt[1] = from[1] + dyc; nxt[2] = from[2];
	} else if (from[2] + dzc >= 0 && from[2] + dzc < c->nz) {
		nxt[0] = src[0]; nxt[1] = src[1]; nxt[2] = from[2] + dzc;
	} else {
		nxt[0] = nxt[1] = nxt[2] = -1;
	}
}

static void next_causal(const orc_ctx* c, const int* from, const int* src, int* nxt) {
	/* Grid::nextCausalCoords, Grid.cpp:294-356 */
	int dir[3], begin[3], i, nd = c->nd;
	for (i = 0; i < 3; ++i)
		dir[i] = (from[i] != src[i]) ? (int)((from[i] - src[i]) / fabs((double)(from[i] - src[i]))) : 1;
	for (i = 0; i < 3; ++i)
		begin[i] = src[i] - (dir[i] < 0 ? 1 : 0);
	next_snake(c, from, begin, dir[0], dir[1], dir[2], nxt);
#define SET(a, b, cc) do { nxt[0] = src[0] - (a); nxt[1] = src[1] - (b); nxt[2] = src[2] - (cc); } while (0)
	if (!within(c, nxt) && dir[0] == 1 && dir[1] == 1 && dir[2] == 1) { SET(1, 0, 0); dir[0] = -1; }
	if (!within(c, nxt) && dir[0] == -1 && dir[1] == 1 && dir[2] == 1 && nd > 1) { SET(0, 1, 0); dir[0] = 1; dir[1] = -1; }
	if (!within(c, nxt) && dir[0] == 1 && dir[1] == -1 && dir[2] == 1 && nd > 1) { SET(1, 1, 0); dir[0] = -1; }
	if (!within(c, nxt) && dir[0] == -1 && dir[1] == -1 && dir[2] == 1 && nd > 2) { SET(0, 0, 1); dir[0] = 1; dir[1] = 1; dir[2] = -1; }
	if (!within(c, nxt) && dir[0] == 1 && dir[1] == 1 && dir[2] == -1 && nd > 2) { SET(1, 0, 1); dir[0] = -1; }
	if (!within(c, nxt) && dir[0] == -1 && dir[1] == 1 && dir[2] == -1 && nd > 2) { SET(0, 1, 1); dir[0] = 1; dir[1] = -1; }
	if (!within(c, nxt) && dir[0] == 1 && dir[1] == -1 && dir[2] == -1 && nd > 2) { SET(1, 1, 1); dir[0] = -1; }
#undef SET
}

static void build_causal(orc_ctx* c) {
	/* Grid::buildCausal (Grid.cpp:568-574) from nearestCoord(position) (:234-240) */
	int start[3], cur[3], nxt[3];
	start[0] = (int)smin(smax(0, c->p.star_pos[0]), c->nx - 1);
	start[1] = (int)smin(smax(0, c->p.star_pos[1]), c->ny - 1);
	start[2] = (int)smin(smax(0, c->p.star_pos[2]), c->nz - 1);
	c->causal = (int*)malloc(sizeof(int) * c->N);
	c->ncausal = 0;
	memcpy(cur, start, sizeof(cur));
	while (within(c, cur) && c->ncausal < c->N) {
		c->causal[c->ncausal++] = (int)flat(c, cur[0], cur[1], cur[2]);
		next_causal(c, cur, start, nxt);
		memcpy(cur, nxt, sizeof(cur));
	}
}

/* ------------------------------------------------------ C2-Ray neighbours --- */
static void nearest_neighbours(orc_ctx* c) {
	/* Grid::calculateNearestNeighbours, Grid.cpp:922-952.  A traversal that
	 * leaves the interior lands on a ghost cell or on -1; both contribute a
	 * zero optical depth (ghost R/T fields are never written), so they are
	 * stored as -1 here. */
	for (long id = 0; id < c->N; ++id) {
		double xc[3];
		int ijk[3];
		cell_xc(c, id, xc);
		cell_coords(c, id, ijk);
		int plane = 0;
		double dmax = 0;
		for (int i = 0; i < c->nd; ++i) {
			double dd = fabs(xc[i] - c->sxc[i]);
			if (dd > dmax) { dmax = dd; plane = i; }
		}
		int irot[3] = {(plane + 1) % 3, (plane + 2) % 3, plane % 3};
		double d[3];
		for (int i = 0; i < 3; i++) d[i] = xc[irot[i]] - c->sxc[irot[i]];
		int s[3], LR[3];
		for (int i = 0; i < 3; ++i) {
			s[i] = d[i] < -1.0 / 10.0 ? -1 : 1;
			LR[i] = fabs(d[i]) < 1.0 / 10.0 ? 0 : s[i];
		}
		int off[4][3] = {{0, 0, -LR[2]}, {0, -LR[1], -LR[2]}, {-LR[0], 0, -LR[2]}, {-LR[0], -LR[1], -LR[2]}};
		for (int n = 0; n < 4; ++n) {
			int t[3] = {ijk[0], ijk[1], ijk[2]};
			for (int r = 0; r < 3; ++r) t[irot[r]] += off[n][r];
			FLD(c->nbr, n, id) = within(c, t) ? (int)flat(c, t[0], t[1], t[2]) : -1;
		}
		double ic0 = (int)xc[irot[0]] - 0.5 * (s[2] * d[0] / d[2]);
		double ic1 = (int)xc[irot[1]] - 0.5 * (s[2] * d[1] / d[2]);
		double delta0 = fabs(2.0 * ic0 - 2.0 * (int)xc[irot[0]] + s[0]);
		double delta1 = fabs(2.0 * ic1 - 2.0 * (int)xc[irot[1]] + s[1]);
		FLD(c->nbw, 0, id) = (fabs(d[2]) > 0.9) ? delta0 * delta1 : 0;
		FLD(c->nbw, 1, id) = ((fabs(d[1]) > 0.9) && (fabs(d[2]) > 0.9)) ? delta0 * (1.0 - delta1) : 0;
		FLD(c->nbw, 2, id) = ((fabs(d[0]) > 0.9) && (fabs(d[2]) > 0.9)) ? (1.0 - delta0) * delta1 : 0;
		FLD(c->nbw, 3, id) = ((fabs(d[0]) > 0.9) && (fabs(d[1]) > 0.9) && (fabs(d[2]) > 0.9)) ? (1.0 - delta0) * (1.0 - delta1) : 0;
	}
}

/* ----------------------------------------------------------- fluid algebra --- */
static void UfromQ(double* u, const double* q, double gamma, int nd) {
	/* GridCell.cpp:163-173 */
	double ke = 0;
	u[DEN] = q[DEN];
	for (int dim = 0; dim < nd; ++dim) {
		u[VEL + dim] = q[VEL + dim] * q[DEN];
		ke += 0.5 * q[DEN] * q[VEL + dim] * q[VEL + dim];
	}
	u[PRE] = q[PRE] / (gamma - 1.0) + ke;
	u[HII] = q[HII] * q[DEN];
	u[ADV] = q[ADV] * q[DEN];
}

static void QfromU(double* q, const double* u, double gamma, int nd) {
	/* GridCell.cpp:175-185 */
	q[DEN] = u[DEN];
	double ke = 0;
	for (int dim = 0; dim < nd; ++dim) {
		q[VEL + dim] = u[VEL + dim] / u[DEN];
		ke += 0.5 * u[VEL + dim] * u[VEL + dim] / u[DEN];
	}
	q[PRE] = (u[PRE] - ke) * (gamma - 1.0);
	q[HII] = u[HII] / u[DEN];
	q[ADV] = u[ADV] / u[DEN];
}

static void FfromQ(double* f, const double* q, double gamma, int nd, int dim) {
	/* GridCell.cpp:200-213 */
	f[DEN] = q[DEN] * q[VEL + dim];
	double ke = 0;
	for (int id = 0; id < nd; ++id) {
		ke += q[VEL + id] * q[VEL + id];
		f[VEL + (dim + id) % nd] = q[DEN] * q[VEL + (dim + id) % nd] * q[VEL + dim];
	}
	ke *= 0.5 * q[DEN];
	f[VEL + dim] += q[PRE];
	double g2 = gamma / (gamma - 1.0);
	f[PRE] = q[VEL + dim] * (g2 * q[PRE] + ke);
	f[HII] = q[DEN] * q[VEL + dim] * q[HII];
	f[ADV] = q[DEN] * q[VEL + dim] * q[ADV];
}

static double calc_temperature(const orc_ctx* c, double hii, double pre, double den) {
	/* Fluid::calcTemperature, Fluid.cpp:71-74 */
	double mu_inv = c->X * (hii + 1.0) + (1.0 - c->X) * 0.25;
	return (pre / den) * (1.0 / mu_inv) / c->specificGasConstant;
}

static void get7(const orc_ctx* c, const double* a, long id, double* v) {
	for (int f = 0; f < NU; ++f) v[f] = FLD(a, f, id);
}
static void put7(const orc_ctx* c, double* a, long id, const double* v) {
	for (int f = 0; f < NU; ++f) FLD(a, f, id) = v[f];
}

static void global_QfromU(orc_ctx* c) {
	/* Fluid::globalQfromU, Fluid.cpp:162-165 */
	for (long id = 0; id < c->N; ++id) {
		double q[7], u[7];
		get7(c, c->Q, id, q);
		get7(c, c->U, id, u);
		QfromU(q, u, c->gamma, c->nd);
		put7(c, c->Q, id, q);
	}
}

static void global_UfromQ(orc_ctx* c) {
	/* Fluid::globalUfromQ, Fluid.cpp:167-170 */
	for (long id = 0; id < c->N; ++id) {
		double q[7], u[7];
		get7(c, c->Q, id, q);
		get7(c, c->U, id, u);
		UfromQ(u, q, c->gamma, c->nd);
		put7(c, c->U, id, u);
	}
}

static void fix_primitives(orc_ctx* c) {
	/* Fluid::fixPrimitives, Fluid.cpp:138-150 (the temperature floor uses U[DEN]) */
	for (long id = 0; id < c->N; ++id) {
		double* q = c->Q;
		FLD(q, HII, id) = smax(smin(FLD(q, HII, id), 1.0), 0.0);
		FLD(q, ADV, id) = smax(smin(FLD(q, ADV, id), 1.0), 0.0);
		FLD(q, DEN, id) = smax(FLD(q, DEN, id), c->dfloor);
		FLD(q, PRE, id) = smax(FLD(q, PRE, id), c->pfloor);
		double mu_inv = c->X * (FLD(q, HII, id) + 1.0) + (1.0 - c->X) * 0.25;
		double temperature = FLD(q, PRE, id) / (mu_inv * c->specificGasConstant * FLD(q, DEN, id));
		if (temperature < c->tfloor)
			FLD(q, PRE, id) = mu_inv * c->specificGasConstant * FLD(c->U, DEN, id) * c->tfloor;
	}
}

static void adv_solution(orc_ctx* c, double dt) {
	/* Fluid::advSolution, Fluid.cpp:80-87 */
	for (long i = 0; i < NU * c->N; ++i) {
		c->U[i] += dt * c->UDOT[i];
		c->UDOT[i] = 0;
	}
}

static int fix_solution(orc_ctx* c) {
	/* Fluid::fixSolution, Fluid.cpp:89-136 */
	for (long id = 0; id < c->N; ++id) {
		double u[7];
		get7(c, c->U, id, u);
		if (!isfinite(u[DEN]) || !isfinite(u[PRE]))
			return fail(c, ORC_ERR_NAN, "fixSolution: non-finite density/energy at cell %ld", id);
		double hii = smax(smin(u[HII] / u[DEN], 1.0), 0.0);
		double adv = smax(smin(u[ADV] / u[DEN], 1.0), 0.0);
		double v[3];
		double den = smax(u[DEN], c->dfloor);
		for (int dim = 0; dim < c->nd; ++dim) v[dim] = u[VEL + dim] / u[DEN];
		double ke = 0.0;
		for (int dim = 0; dim < c->nd; ++dim) ke += v[dim] * v[dim];
		ke *= 0.5 * u[DEN];
		double pre = (u[PRE] - ke) * (c->gamma - 1.0);
		ke *= den / u[DEN];
		if (pre < c->pfloor) pre = c->pfloor;
		double mu_inv = c->X * (hii + 1.0) + (1.0 - c->X) * 0.25;
		double temperature = pre / (mu_inv * c->specificGasConstant * den);
		if (temperature < c->tfloor)
			pre = mu_inv * c->specificGasConstant * den * c->tfloor;
		u[DEN] = den;
		u[PRE] = pre / (c->gamma - 1.0) + ke;
		u[HII] = hii * den;
		u[ADV] = adv * den;
		for (int dim = 0; dim < c->nd; ++dim) u[VEL + dim] = den * v[dim];
		if (u[DEN] == 0 || u[PRE] == 0)
			return fail(c, ORC_ERR_NAN, "fixSolution: zero density or energy at cell %ld", id);
		for (int f = 0; f < NU; ++f)
			if (u[f] != u[f] || isinf(u[f]))
				return fail(c, ORC_ERR_NAN, "fixSolution: invalid value at cell %ld", id);
		put7(c, c->U, id, u);
	}
	return 0;
}

static int check_values(orc_ctx* c) {
	/* Torch::checkValues, Torch.cpp:420-443 */
	for (long id = 0; id < c->N; ++id) {
		for (int f = 0; f < NU; ++f) {
			double u = FLD(c->U, f, id);
			if (u != u || isinf(u) || FLD(c->Q, DEN, id) == 0 || FLD(c->Q, PRE, id) == 0)
				return fail(c, ORC_ERR_NAN, "checkValues: invalid state at cell %ld", id);
		}
	}
	return 0;
}

/* ------------------------------------------------------------- limiters --- */
static inline double minmod(double a, double b) { return (a * b > 0) ? (fabs(a) < fabs(b) ? a : b) : 0; }
static inline double maxmod(double a, double b) { return (a * b > 0) ? (fabs(a) > fabs(b) ? a : b) : 0; }

static double limiter(int kind, double a, double b) {
	/* SlopeLimiter.cpp:5-54 */
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

/* -------------------------------------------------------- Riemann solvers --- */
static void wave_speeds(double a_l2, double a_r2, const double* Ql, const double* Qr, int dim, double* Sl, double* Sr) {
	/* characteristicWaveSpeeds, Riemann.cpp:27-42 */
	double sqrtrho_l = sqrt(Ql[DEN]);
	double sqrtrho_r = sqrt(Qr[DEN]);
	double u_tilde = (sqrtrho_l * Ql[VEL + dim] + sqrtrho_r * Qr[VEL + dim]) / (sqrtrho_l + sqrtrho_r);
	double nu2 = 0.5 * sqrtrho_r * sqrtrho_l / ((sqrtrho_l + sqrtrho_r) * (sqrtrho_l + sqrtrho_r));
	double dsqrd = (sqrtrho_l * a_l2 + sqrtrho_r * a_r2) / (sqrtrho_l + sqrtrho_r);
	dsqrd += nu2 * (Qr[VEL + dim] - Ql[VEL + dim]) * (Qr[VEL + dim] - Ql[VEL + dim]);
	double d = sqrt(dsqrd);
	*Sl = u_tilde - d;
	*Sr = u_tilde + d;
}

static int hllc(double* F, const double* Ql, const double* Qr, double a_l2, double a_r2, double gamma, int nd, int dim) {
	/* HartenLaxLeerContactSolver::solve, Riemann.cpp:52-104 */
	double S_l, S_r;
	wave_speeds(a_l2, a_r2, Ql, Qr, dim, &S_l, &S_r);
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
		double U_lr[7] = {0}, F_lr[7] = {0}, U_clr[7] = {0};
		UfromQ(U_lr, Qlr, gamma, nd);
		FfromQ(F_lr, Qlr, gamma, nd, dim);
		double A_lr = Qlr[DEN] * (S_lr - Qlr[VEL + dim]) / (S_lr - S_c);
		U_clr[DEN] = A_lr;
		for (int id = 0; id < nd; ++id) U_clr[VEL + id] = A_lr * Qlr[VEL + id];
		U_clr[VEL + dim] = A_lr * S_c;
		U_clr[PRE] = A_lr * ((U_lr[PRE] / Qlr[DEN]) + (S_c - Qlr[VEL + dim]) * (S_c + Qlr[PRE] / (Qlr[DEN] * (S_lr - Qlr[VEL + dim]))));
		U_clr[HII] = A_lr * Qlr[HII];
		U_clr[ADV] = A_lr * Qlr[ADV];
		for (int i = 0; i < NU; ++i) F[i] = F_lr[i] + S_lr * (U_clr[i] - U_lr[i]);
		if (nd < 3) F[VEL + 2] = 0;
		if (nd < 2) F[VEL + 1] = 0;
	}
	return F[HII] != F[HII] ? ORC_ERR_FLUX : 0;
}

static int hll(double* F, const double* Ql, const double* Qr, double a_l2, double a_r2, double gamma, int nd, int dim) {
	/* HartenLaxLeerSolver::solve, Riemann.cpp:108-140 */
	double S_l, S_r;
	wave_speeds(a_l2, a_r2, Ql, Qr, dim, &S_l, &S_r);
	if (S_r <= 0) {
		FfromQ(F, Qr, gamma, nd, dim);
	} else if (S_l >= 0) {
		FfromQ(F, Ql, gamma, nd, dim);
	} else {
		double U_l[7] = {0}, U_r[7] = {0}, F_l[7] = {0}, F_r[7] = {0};
		UfromQ(U_l, Ql, gamma, nd);
		UfromQ(U_r, Qr, gamma, nd);
		FfromQ(F_l, Ql, gamma, nd, dim);
		FfromQ(F_r, Qr, gamma, nd, dim);
		for (int i = 0; i < NU; ++i)
			F[i] = (S_r * F_l[i] - S_l * F_r[i] + S_l * S_r * (U_r[i] - U_l[i])) / (S_r - S_l);
	}
	return F[HII] != F[HII] ? ORC_ERR_FLUX : 0;
}

/* 3-vector algebra in the evaluation order of the vendored Eigen 3.2.1
 * (lib/Eigen, SSE2 packets of two doubles), established by compiling it here:
 *   - dot/squaredNorm reduce three terms as x + (y + z);
 *   - v /= s multiplies by the reciprocal 1/s (so normalize() does);
 *   - 3x3 * 3-vector and 3x3 * 3x3 coefficients accumulate (a + b) + c. */
static void cross3(const double* a, const double* b, double* r) {
	r[0] = a[1] * b[2] - a[2] * b[1];
	r[1] = a[2] * b[0] - a[0] * b[2];
	r[2] = a[0] * b[1] - a[1] * b[0];
}
static double dot3(const double* a, const double* b) { return a[0] * b[0] + (a[1] * b[1] + a[2] * b[2]); }
static double norm3(const double* a) { return sqrt(dot3(a, a)); }
static void normalize3(double* a) {
	double r = 1.0 / norm3(a);
	a[0] *= r; a[1] *= r; a[2] *= r;
}

static void rotation_a2b(const double* A, const double* B, double R[3][3]) {
	/* getRotationFromA2B, Riemann.cpp:161-171: I + [v]x + (1-c)/s^2 [v]x[v]x */
	double v[3];
	cross3(A, B, v);
	double s = norm3(v);
	double cc = dot3(A, B);
	double vx[3][3] = {{0, -v[2], v[1]}, {v[2], 0, -v[0]}, {-v[1], v[0], 0}};
	double k = (1.0 - cc) / (s * s);
	double kvx[3][3];
	for (int i = 0; i < 3; ++i)
		for (int j = 0; j < 3; ++j) kvx[i][j] = k * vx[i][j];
	for (int i = 0; i < 3; ++i)
		for (int j = 0; j < 3; ++j) {
			double prod = kvx[i][0] * vx[0][j] + kvx[i][1] * vx[1][j] + kvx[i][2] * vx[2][j];
			double id = (i == j) ? 1.0 : 0.0;
			R[i][j] = (id + vx[i][j]) + prod;
		}
}

static void rotate(double R[3][3], double* v) {
	/* rotate, Riemann.cpp:154-159 */
	double x = v[VEL + 0], y = v[VEL + 1], z = v[VEL + 2];
	for (int i = 0; i < 3; ++i)
		v[VEL + i] = R[i][0] * x + R[i][1] * y + R[i][2] * z;
}

static int rotated_hllc(double* F, const double* Ql, const double* Qr, double a_l2, double a_r2, double gamma, int nd, int dim) {
	/* RotatedHartenLaxLeerSolver::solve, Riemann.cpp:181-244 */
	int pureHLLC = 0, pureHLL = 0;
	double d[3] = {dim == 0 ? 1 : 0, dim == 1 ? 1 : 0, dim == 2 ? 1 : 0};
	double n1[3] = {Qr[VEL + 0] - Ql[VEL + 0], Qr[VEL + 1] - Ql[VEL + 1], Qr[VEL + 2] - Ql[VEL + 2]};
	double n2[3] = {0, 0, 0}, t[3];
	if (n1[dim] < 0)
		for (int i = 0; i < 3; ++i) n1[i] = -1.0 * n1[i];
	if (norm3(n1) < 1.0e-6)
		pureHLLC = 1;
	else {
		normalize3(n1);
		cross3(n1, d, t);
		if (norm3(t) == 0)
			pureHLL = 1;
		else {
			cross3(t, n1, n2);
			if (norm3(n2) == 0)
				pureHLL = 1;
			else {
				if (n2[dim] < 0)
					for (int i = 0; i < 3; ++i) n2[i] = -1.0 * n2[i];
				normalize3(n2);
				cross3(n2, d, t);
				if (norm3(t) == 0)
					pureHLLC = 1;
			}
		}
	}
	if (!pureHLLC && !pureHLL) {
		double F1[7] = {0}, F2[7] = {0}, QlR[7], QrR[7], Rm[3][3];
		memcpy(QlR, Ql, sizeof(QlR));
		memcpy(QrR, Qr, sizeof(QrR));
		rotation_a2b(n1, d, Rm);
		rotate(Rm, QlR);
		rotate(Rm, QrR);
		int e = hll(F1, QlR, QrR, a_l2, a_r2, gamma, nd, dim);
		rotation_a2b(d, n1, Rm);
		rotate(Rm, QlR);
		rotate(Rm, QrR);
		rotate(Rm, F1);
		rotation_a2b(n2, d, Rm);
		rotate(Rm, QlR);
		rotate(Rm, QrR);
		e |= hllc(F2, QlR, QrR, a_l2, a_r2, gamma, nd, dim);
		rotation_a2b(d, n2, Rm);
		rotate(Rm, F2);
		for (int iu = 0; iu < NU; ++iu)
			F[iu] = fabs(dot3(d, n1)) * F1[iu] + fabs(dot3(d, n2)) * F2[iu];
		return e;
	} else if (pureHLL)
		return hll(F, Ql, Qr, a_l2, a_r2, gamma, nd, dim);
	return hllc(F, Ql, Qr, a_l2, a_r2, gamma, nd, dim);
}

static int riemann(const orc_ctx* c, double* F, const double* Ql, const double* Qr, double a_l2, double a_r2, int dim) {
	for (int i = 0; i < NU; ++i) F[i] = 0;
	switch (c->p.riemann) {
	case RS_HLLC: return hllc(F, Ql, Qr, a_l2, a_r2, c->gamma, c->nd, dim);
	case RS_HLL: return hll(F, Ql, Qr, a_l2, a_r2, c->gamma, c->nd, dim);
	default: return rotated_hllc(F, Ql, Qr, a_l2, a_r2, c->gamma, c->nd, dim);
	}
}

/* ------------------------------------------------------------------ hydro --- */
/* Ghost layers: ghostQ[dim][side] holds ng layers x 7 fields x (cells in the
 * face), layer 0 adjacent to the boundary.  Face cell index = flat index with
 * the dim coordinate dropped. */
static long face_index(const orc_ctx* c, int dim, const int* ijk) {
	if (dim == 0) return ijk[1] + (long)c->ny * ijk[2];
	if (dim == 1) return ijk[0] + (long)c->nx * ijk[2];
	return ijk[0] + (long)c->nx * ijk[1];
}
static double* ghost_ptr(orc_ctx* c, int dim, int side, int layer, int f, long fi) {
	return &c->ghostQ[dim][side][((long)layer * NU + f) * c->gcount[dim] + fi];
}

static void apply_bcs(orc_ctx* c) {
	/* Grid::applyBCs, Grid.cpp:649-836 (single rank: no PARTITION) */
	for (int dim = 0; dim < c->nd; ++dim) {
		int n = ncell_dim(c, dim);
		for (int side = 0; side < 2; ++side) {
			int cond = side == 0 ? c->lbc[dim] : c->rbc[dim];
			int ijk[3];
			int lo[3] = {0, 0, 0}, hi[3] = {c->nx, c->ny, c->nz};
			hi[dim] = 1;
			for (ijk[2] = lo[2]; ijk[2] < hi[2]; ++ijk[2])
			for (ijk[1] = lo[1]; ijk[1] < hi[1]; ++ijk[1])
			for (ijk[0] = lo[0]; ijk[0] < hi[0]; ++ijk[0]) {
				long fi = face_index(c, dim, ijk);
				for (int layer = 0; layer < c->ng; ++layer) {
					int src;
					int k = layer + 1;
					switch (cond) {
					case BC_PERIODIC: src = side == 0 ? n - k : k - 1; break;
					case BC_REFLECTING: src = side == 0 ? k : n - 1 - k; break;
					default: src = side == 0 ? 0 : n - 1; break;
					}
					int t[3] = {ijk[0], ijk[1], ijk[2]};
					t[dim] = src;
					long sid = flat(c, t[0], t[1], t[2]);
					double q[7];
					get7(c, c->Q, sid, q);
					double v = q[VEL + dim];
					if (cond == BC_INFLOW) {
						if (side == 0 ? v < 0 : v > 0) q[VEL + dim] = -1.0 * v;
					} else if (cond == BC_OUTFLOW) {
						if (side == 0 ? v > 0 : v < 0) q[VEL + dim] = -1.0 * v;
					} else if (cond == BC_REFLECTING) {
						q[VEL + dim] = -v;
					}
					for (int f = 0; f < NU; ++f) *ghost_ptr(c, dim, side, layer, f, fi) = q[f];
				}
			}
		}
	}
}

/* Q of the cell at offset o (|o| <= ng) along dim from interior cell ijk. */
static void q_along(orc_ctx* c, const int* ijk, int dim, int o, double* q) {
	int n = ncell_dim(c, dim);
	int x = ijk[dim] + o;
	if (x >= 0 && x < n) {
		int t[3] = {ijk[0], ijk[1], ijk[2]};
		t[dim] = x;
		get7(c, c->Q, flat(c, t[0], t[1], t[2]), q);
		return;
	}
	long fi = face_index(c, dim, ijk);
	int side = x < 0 ? 0 : 1;
	int layer = x < 0 ? -x - 1 : x - n;
	for (int f = 0; f < NU; ++f) q[f] = *ghost_ptr(c, dim, side, layer, f, fi);
}

static void piecewise_linear(const orc_ctx* c, const double* Ql, const double* Qc, const double* Qr, double* left, double* right) {
	/* Hydrodynamics::piecewiseLinear, Hydro.cpp:44-50 */
	for (int iq = 0; iq < NU; ++iq) {
		double dQdr = limiter(c->p.limiter, Qc[iq] - Ql[iq], Qr[iq] - Qc[iq]);
		left[iq] = Qc[iq] - 0.5 * dQdr;
		right[iq] = Qc[iq] + 0.5 * dQdr;
	}
}

static int hydro_fluxes(orc_ctx* c) {
	/* Hydrodynamics::integrate (Hydro.cpp:31-34) = applyBCs + calcFluxes (:91-115)
	 * with the reconstruction of Hydro.cpp:52-67.  Face f along dim sits between
	 * line positions f-1 and f (f = 0 is the left boundary face). */
	apply_bcs(c);
	for (int dim = 0; dim < c->nd; ++dim) {
		int n = ncell_dim(c, dim);
		int ijk[3], hi[3] = {c->nx, c->ny, c->nz};
		hi[dim] = 1;
		for (ijk[2] = 0; ijk[2] < hi[2]; ++ijk[2])
		for (ijk[1] = 0; ijk[1] < hi[1]; ++ijk[1])
		for (ijk[0] = 0; ijk[0] < hi[0]; ++ijk[0]) {
			long fi = face_index(c, dim, ijk);
			for (int f = 0; f <= n; ++f) {
				double Ls[7], Rs[7], F[7];
				int pos[3] = {ijk[0], ijk[1], ijk[2]};
				if (c->order == 1) {
					double a[7], b[7], cq[7], e[7], unused[7];
					pos[dim] = 0;
					q_along(c, pos, dim, f - 2, a);
					q_along(c, pos, dim, f - 1, b);
					q_along(c, pos, dim, f, cq);
					q_along(c, pos, dim, f + 1, e);
					/* left state: QR of the cell at f-1; right state: QL of the cell at f */
					piecewise_linear(c, a, b, cq, unused, Ls);
					piecewise_linear(c, b, cq, e, Rs, unused);
				} else {
					pos[dim] = 0;
					q_along(c, pos, dim, f - 1, Ls);
					q_along(c, pos, dim, f, Rs);
				}
				double a_l2 = c->gamma * Ls[PRE] / Ls[DEN];
				double a_r2 = c->gamma * Rs[PRE] / Rs[DEN];
				if (riemann(c, F, Ls, Rs, a_l2, a_r2, dim))
					return fail(c, ORC_ERR_FLUX, "Riemann solver: HII flux is NaN (dim %d face %d)", dim, f);
				for (int q = 0; q < NU; ++q)
					c->F[dim][((long)q * c->gcount[dim] + fi) * (n + 1) + f] = F[q];
			}
		}
	}
	return 0;
}

static void hydro_source_terms(orc_ctx* c) {
	/* Hydrodynamics::updateSourceTerms, Hydro.cpp:117-156 */
	for (long id = 0; id < c->N; ++id) {
		int ijk[3];
		cell_coords(c, id, ijk);
		double vol = c->vol[id];
		for (int dim = 0; dim < c->nd; ++dim) {
			int n = ncell_dim(c, dim);
			long fi = face_index(c, dim, ijk);
			double al = face_area(c, id, dim, 0), ar = face_area(c, id, dim, 1);
			for (int i = 0; i < NU; ++i) {
				const double* Fd = c->F[dim] + ((long)i * c->gcount[dim] + fi) * (n + 1);
				FLD(c->UDOT, i, id) += (al / vol) * Fd[ijk[dim]];
				FLD(c->UDOT, i, id) -= (ar / vol) * Fd[ijk[dim] + 1];
			}
		}
		for (int i = 0; i < 3; ++i) {
			FLD(c->UDOT, VEL + i, id) += FLD(c->grav, i, id);
			FLD(c->UDOT, PRE, id) += FLD(c->Q, VEL + i, id) * FLD(c->grav, i, id);
		}
		if (c->geometry == G_CYL) {
			double xc[3];
			cell_xc(c, id, xc);
			double r = c->dx[0] * xc[0];
			FLD(c->UDOT, VEL + 0, id) += FLD(c->Q, PRE, id) / r;
		} else if (c->geometry == G_SPH) {
			double area1 = face_area(c, id, 0, 1), area2 = face_area(c, id, 0, 0);
			double r = vol / (area1 - area2);
			FLD(c->UDOT, VEL + 0, id) += FLD(c->Q, PRE, id) / r;
		}
	}
	/* Star::injectEnergyMomentum, Star.cpp:57-68 */
	if (c->p.star_on && c->mdot != 0) {
		for (long w = 0; w < c->nwind; ++w) {
			long id = c->wind[w];
			FLD(c->UDOT, DEN, id) += c->mdot;
			FLD(c->UDOT, PRE, id) += c->edot;
			FLD(c->UDOT, HII, id) += (FLD(c->U, HII, id) / FLD(c->U, DEN, id)) * c->mdot;
			FLD(c->UDOT, ADV, id) += c->mdot;
		}
	}
}

static double hydro_dt(orc_ctx* c) {
	/* Hydrodynamics::calculateTimeStep, Hydro.cpp:77-89 */
	double tmin = c->dt_max;
	for (long id = 0; id < c->N; ++id) {
		double inv_t = 0;
		double ss = sqrt(c->gamma * FLD(c->Q, PRE, id) / FLD(c->Q, DEN, id));
		for (int dim = 0; dim < c->nd; ++dim)
			inv_t += (fabs(FLD(c->Q, VEL + dim, id)) + ss) / c->dx[dim];
		if (inv_t == 0) inv_t = 1.0 / c->dt_max;
		tmin = smin(tmin, 0.5 / inv_t);
	}
	return smin(tmin, c->dt_max);
}

/* -------------------------------------------------------------- radiation --- */
static double photoionisation_rate(double nHI, double T, double delT, double shellVol, double photonRate) {
	/* Radiation.cpp:243-251 */
	if (nHI == 0 || shellVol == 0) return 0.0;
	double emT = m_exp(-T);
	double emdT = m_exp(-delT);
	return photonRate * emT * (1.0 - emdT) / (nHI * shellVol);
}

static double collisional_ionisation_rate(const orc_ctx* c, double T) {
	/* Radiation.cpp:231-237 */
	if (!c->p.collisions_on || T < 5.0e3) return 0.0;
	double U = c->voronov_DE / T;
	return c->voronov_A * (1. + c->voronov_P * sqrt(U)) * m_exp(c->voronov_K * m_log(U) - U) / (c->voronov_X + U);
}

static void doric(double dt, double* HII_avg, double* HII, double Api, double nHII_aB, double nHII_Aci) {
	/* Radiation::doric, Radiation.cpp:140-179 */
	double xeq, inv_ti, epsilon = 1.0e-8;
	double HII_old = *HII;
	if (nHII_aB == 0.0) xeq = 1.0;
	else xeq = (Api + nHII_Aci) / (Api + nHII_Aci + nHII_aB);
	inv_ti = Api + nHII_Aci + nHII_aB;
	if (dt * inv_ti < 1.0e-8) {
		*HII = HII_old;
		*HII = smax(smin(*HII, 1.0), 0.0);
		if (1.0 - *HII < epsilon) *HII = 1.0 - epsilon;
		*HII_avg = *HII;
	} else {
		double e = m_exp(-dt * inv_ti);
		*HII = xeq + (HII_old - xeq) * e;
		*HII = smax(smin(*HII, 1.0), 0.0);
		if (1.0 - *HII < epsilon) *HII = 1.0 - epsilon;
		*HII_avg = xeq + (HII_old - xeq) * (1.0 - e) / (dt * inv_ti);
		*HII_avg = smax(smin(*HII_avg, 1.0), 0.0);
		if (1.0 - *HII_avg < epsilon) *HII_avg = 1.0 - epsilon;
	}
}

static double cell_dist2(const orc_ctx* c, long id) {
	double xc[3], d2 = 0;
	cell_xc(c, id, xc);
	for (int i = 0; i < c->nd; ++i) d2 += (xc[i] - c->sxc[i]) * (xc[i] - c->sxc[i]);
	return d2;
}

static void update_tau_sc(orc_ctx* c, int average, long id, double dist2) {
	/* Radiation::updateTauSC, Radiation.cpp:353-373 */
	int rt = average ? R_TAU_A : R_TAU, rd = average ? R_DTAU_A : R_DTAU;
	if (dist2 > 0.95) {
		double tau[4] = {0, 0, 0, 0}, w[4];
		for (int i = 0; i < 4; ++i) {
			int nb = FLD(c->nbr, i, id);
			if (nb >= 0) tau[i] = FLD(c->R, rt, nb) + FLD(c->R, rd, nb);
			w[i] = FLD(c->nbw, i, id) / smax(c->p.tau0, tau[i]);
		}
		double sum_w = w[0] + w[1] + w[2] + w[3];
		double newtau = 0.0;
		for (int i = 0; i < 4; ++i) {
			w[i] = w[i] / sum_w;
			newtau += w[i] * tau[i];
		}
		FLD(c->R, rt, id) = newtau;
	} else
		FLD(c->R, rt, id) = 0;
}

static int is_star(const orc_ctx* c, long id) {
	/* Radiation::isStar, Radiation.cpp:682-684 (z compared int against double) */
	double xc[3];
	cell_xc(c, id, xc);
	return (int)xc[0] == (int)c->sxc[0] && (int)xc[1] == (int)c->sxc[1] && (double)(int)xc[2] == c->sxc[2];
}

static int update_hii_frac(orc_ctx* c, double dt, long id) {
	/* Radiation::update_HIIfrac (implicit scheme), Radiation.cpp:375-478 */
	if (is_star(c, id)) {
		FLD(c->R, R_HEAT, id) = 0;
		FLD(c->Q, HII, id) = 1;
		FLD(c->R, R_HII_A, id) = 1;
		return 0;
	}
	double n_H = c->X * FLD(c->Q, DEN, id) / c->hydrogenMass;
	double A_pi = 0;
	double x_new = FLD(c->Q, HII, id);
	double HII_avg = x_new;
	double T = calc_temperature(c, FLD(c->Q, HII, id), FLD(c->Q, PRE, id), FLD(c->Q, DEN, id));
	double alphaB = spline_eval(&c->rad_recomb, T);
	double A_ci = collisional_ionisation_rate(c, T);
	double convergence2 = 1.0e-3, convergence_frac = 1.0e-5, HII_avg_old;
	int niter = 0, miter = 0, converged = 0;
	double tau_avg = FLD(c->R, R_TAU_A, id);
	while (!converged) {
		niter++;
		HII_avg_old = HII_avg;
		x_new = FLD(c->Q, HII, id);
		double dtau_avg = (1.0 - HII_avg) * n_H * c->photoIonXsec * c->ds[id];
		double nHI = (1.0 - HII_avg) * n_H;
		A_pi = photoionisation_rate(nHI, tau_avg, dtau_avg, c->shellVol[id], c->photonRate);
		double nHII_aB = HII_avg * n_H * alphaB;
		double nHII_Aci = HII_avg * n_H * A_ci;
		doric(dt, &HII_avg, &x_new, A_pi, nHII_aB, nHII_Aci);
		if ((fabs((HII_avg - HII_avg_old) / HII_avg) < convergence2 || (HII_avg < convergence_frac) || A_pi == 0))
			converged = 1;
		if (niter > 10005) {
			miter++;
			niter = 0;
			HII_avg = 0.5 * (HII_avg + HII_avg_old);
		}
		if (miter > 5 || x_new != x_new)
			return fail(c, ORC_ERR_PICARD, "update_HIIfrac: implicit method not converging at cell %ld", id);
	}
	FLD(c->R, R_HII_A, id) = HII_avg;
	FLD(c->Q, HII, id) = x_new;
	if (x_new > 0.001) FLD(c->Q, ADV, id) = 1;
	return 0;
}

static int update_hii_frac2(orc_ctx* c, double dt, long id) {
	/* Radiation::update_HIIfrac for the implicit2 and explicit schemes,
	 * Radiation.cpp:375-478: implicit2 iterates with tau_avg = TAU; explicit
	 * takes one doric step whose time-averaged result becomes Q[HII]. */
	if (is_star(c, id)) {
		FLD(c->R, R_HEAT, id) = 0;
		FLD(c->Q, HII, id) = 1;
		FLD(c->R, R_HII_A, id) = 1;
		return 0;
	}
	if (c->p.rt_scheme == 1) {
		double saved = FLD(c->R, R_TAU_A, id);
		FLD(c->R, R_TAU_A, id) = FLD(c->R, R_TAU, id);  /* the iteration's tau_avg */
		int e = update_hii_frac(c, dt, id);
		FLD(c->R, R_TAU_A, id) = saved;
		return e;
	}
	double n_H = c->X * FLD(c->Q, DEN, id) / c->hydrogenMass;
	double x = FLD(c->Q, HII, id);
	double x_avg = x;
	double T = calc_temperature(c, FLD(c->Q, HII, id), FLD(c->Q, PRE, id), FLD(c->Q, DEN, id));
	double alphaB = spline_eval(&c->rad_recomb, T);
	double A_ci = collisional_ionisation_rate(c, T);
	double tau = FLD(c->R, R_TAU, id), dtau = FLD(c->R, R_DTAU, id);
	double nHI = (1.0 - x) * (c->X * FLD(c->Q, DEN, id) / c->hydrogenMass);
	double A_pi = photoionisation_rate(nHI, tau, dtau, c->shellVol[id], c->photonRate);
	double nHII_aB = x_avg * n_H * alphaB;
	double nHII_Aci = x_avg * n_H * A_ci;
	double x_dummy = x;
	doric(dt, &x, &x_dummy, A_pi, nHII_aB, nHII_Aci);
	FLD(c->Q, HII, id) = x;
	if (x > 0.001) FLD(c->Q, ADV, id) = 1;
	return 0;
}

static int transfer_radiation2(orc_ctx* c, double dt) {
	/* Radiation::transferRadiation2, Radiation.cpp:508-567, with rayTrace,
	 * :480-506 (single rank): the causal sweep only interpolates TAU and sets
	 * the cell optical depths from the current fractions; the fractions are
	 * then updated cell by cell, independently.  Star on (the caller's test). */
	for (long w = 0; w < c->nwind; ++w) {
		long id = c->wind[w];
		FLD(c->R, R_TAU, id) = 0;
		FLD(c->R, R_TAU_A, id) = 0;
		FLD(c->R, R_DTAU, id) = 0;
		FLD(c->R, R_DTAU_A, id) = 0;
		FLD(c->Q, HII, id) = 1;
		FLD(c->R, R_HII_A, id) = 1;
	}
	for (long k = 0; k < c->nnonwind; ++k) {
		long id = c->nonwind[k];
		update_tau_sc(c, 0, id, cell_dist2(c, id));
		double nH = c->X * FLD(c->Q, DEN, id) / c->hydrogenMass;
		FLD(c->R, R_DTAU, id) = (1.0 - FLD(c->Q, HII, id)) * nH * c->photoIonXsec * c->ds[id];
		FLD(c->R, R_DTAU_A, id) = (1.0 - FLD(c->R, R_HII_A, id)) * nH * c->photoIonXsec * c->ds[id];
	}
	for (long k = 0; k < c->nnonwind; ++k) {
		int e = update_hii_frac2(c, dt, c->nonwind[k]);
		if (e) return e;
	}
	return 0;
}

static int transfer_radiation(orc_ctx* c, double dt) {
	/* Radiation::transferRadiation, Radiation.cpp:569-651 (single rank) */
	if (c->p.rt_scheme != 0 && c->p.star_on) return transfer_radiation2(c, dt);
	if (c->p.star_on) {
		for (long w = 0; w < c->nwind; ++w) {
			long id = c->wind[w];
			FLD(c->R, R_TAU, id) = 0;
			FLD(c->R, R_TAU_A, id) = 0;
			FLD(c->R, R_DTAU, id) = 0;
			FLD(c->R, R_DTAU_A, id) = 0;
			FLD(c->Q, HII, id) = 1;
			FLD(c->R, R_HII_A, id) = 1;
		}
		for (long k = 0; k < c->nnonwind; ++k) {
			long id = c->nonwind[k];
			double dist2 = cell_dist2(c, id);
			update_tau_sc(c, 0, id, dist2);
			update_tau_sc(c, 1, id, dist2);
			int e = update_hii_frac(c, dt, id);
			if (e) return e;
			double nH = c->X * FLD(c->Q, DEN, id) / c->hydrogenMass;
			FLD(c->R, R_DTAU, id) = (1.0 - FLD(c->Q, HII, id)) * nH * c->photoIonXsec * c->ds[id];
			FLD(c->R, R_DTAU_A, id) = (1.0 - FLD(c->R, R_HII_A, id)) * nH * c->photoIonXsec * c->ds[id];
		}
	} else {
		for (long id = 0; id < c->N; ++id) {
			double x_new = FLD(c->Q, HII, id), x_dummy = x_new;
			double n_H = c->X * FLD(c->Q, DEN, id) / c->hydrogenMass;
			double T = calc_temperature(c, FLD(c->Q, HII, id), FLD(c->Q, PRE, id), FLD(c->Q, DEN, id));
			double nHII_aB = x_new * n_H * spline_eval(&c->rad_recomb, T);
			double nHII_Aci = x_new * n_H * collisional_ionisation_rate(c, T);
			doric(dt, &x_new, &x_dummy, 0, nHII_aB, nHII_Aci);
			FLD(c->Q, HII, id) = x_new;
		}
	}
	return 0;
}

static int rad_pre(orc_ctx* c) {
	/* Radiation::preTimeStepCalculations, Radiation.cpp:257-296 */
	for (long k = 0; k < c->nnonwind; ++k) {
		long id = c->nonwind[k];
		double q_hii = FLD(c->Q, HII, id), q_pre = FLD(c->Q, PRE, id), q_den = FLD(c->Q, DEN, id);
		double n_H = (c->X * q_den / c->hydrogenMass);
		double excessEnergy = c->photonEnergy - c->rydbergEnergy;
		double T = calc_temperature(c, q_hii, q_pre, q_den);
		double nHI = (1.0 - q_hii) * n_H;
		double A_pi = photoionisation_rate(nHI, FLD(c->R, R_TAU, id), FLD(c->R, R_DTAU, id), c->shellVol[id], c->photonRate);
		double photoion = n_H * (1.0 - q_hii) * A_pi * excessEnergy;
		double rate_rc = spline_eval(&c->rad_cool, T);
		double recombination = q_hii * q_hii * n_H * n_H * c->boltzmannConst * T * rate_rc;
		double collisions = q_hii * (1.0 - q_hii) * n_H * n_H * collisional_ionisation_rate(c, T);
		double rate = photoion - recombination - collisions;
		double softrate = rate;
		if (T < c->Tmin[id] + 200 && rate < 0.0)
			softrate = smin(0.0, softrate * (T - c->Tmin[id]) / 200.0);
		softrate *= c->p.heating_amp;
		FLD(c->R, R_HEAT, id) = softrate;
		if (rate != rate)
			return fail(c, ORC_ERR_NAN, "radiation heating rate is NaN at cell %ld", id);
	}
	return 0;
}

static int rad_dt(orc_ctx* c, double* out) {
	/* Radiation::calculateTimeStep, Radiation.cpp:298-351 */
	double dt_max = c->dt_max, dt = dt_max;
	if (c->p.star_on) {
		for (long k = 0; k < c->nnonwind; ++k) {
			long id = c->nonwind[k];
			double dtc, dt1, dt2, dt3, dt4;
			dtc = dt1 = dt2 = dt3 = dt4 = dt_max;
			double q_hii = FLD(c->Q, HII, id), q_pre = FLD(c->Q, PRE, id), q_den = FLD(c->Q, DEN, id);
			if (c->p.coupling == CP_NEQ) {
				if (FLD(c->R, R_HEAT, id) != 0) dtc = fabs(FLD(c->U, PRE, id) / FLD(c->R, R_HEAT, id));
			}
			if (c->p.K1 != 0.0) {
				double T = calc_temperature(c, q_hii, q_pre, q_den);
				if (!c->rad_once) {
					dt1 = c->p.K1 * c->hydrogenMass / (c->X * q_den * spline_eval(&c->rad_recomb, T));
					c->rad_once = 1;
				} else if (q_hii != 0) {
					dt1 = c->p.K1 * c->hydrogenMass / (c->X * q_den * q_hii * spline_eval(&c->rad_recomb, T));
				}
			}
			if (c->p.K2 != 0.0) dt2 = dt_max;
			if (c->p.K3 != 0.0 || c->p.K4 != 0.0) {
				double nH = c->X * q_den / c->hydrogenMass;
				double nHI = (1.0 - q_hii) * nH;
				double A_pi = photoionisation_rate(nHI, FLD(c->R, R_TAU, id), FLD(c->R, R_DTAU, id), c->shellVol[id], c->photonRate);
				double Tq = calc_temperature(c, q_hii, q_pre, q_den);
				double A_ci = collisional_ionisation_rate(c, Tq);
				double A_rr = spline_eval(&c->rad_recomb, Tq);
				double fracRate = (1.0 - q_hii) * (A_pi + q_hii * nH * A_ci) - q_hii * q_hii * nH * A_rr;
				if (c->p.K3 != 0.0 && fracRate != 0.0) dt3 = c->p.K3 * smax(0.05, 1.0 - q_hii) / fabs(fracRate);
				if (c->p.K4 != 0.0 && fracRate != 0.0) dt4 = c->p.K4 * 1.0 / fabs(fracRate);
			}
			dt = smin(dt, smin(dt_max, smin(dtc, smin(dt1, smin(dt2, smin(dt3, dt4))))));
			if (dt == 0.0 || dt != dt || isinf(dt))
				return fail(c, ORC_ERR_DT, "Radiation::calculateTimeStep: invalid timestep %g", dt);
		}
	}
	*out = dt;
	return 0;
}

static void rad_source_terms(orc_ctx* c, double dt) {
	/* Radiation::updateSourceTerms, Radiation.cpp:653-680 */
	if (!c->p.star_on) return;
	for (long id = 0; id < c->N; ++id) {
		if (c->p.coupling == CP_TTI) {
			double HII_new = FLD(c->Q, HII, id);
			double mu_inv_new = c->X * (HII_new + 1.0) + (1.0 - c->X) * 0.25;
			double T_new = c->p.THI + (c->p.THII - c->p.THI) * HII_new;
			double pre_new = c->specificGasConstant * mu_inv_new * FLD(c->Q, DEN, id) * T_new;
			double ke = 0.0;
			for (int dim = 0; dim < c->nd; ++dim)
				ke += 0.5 * FLD(c->U, VEL + dim, id) * FLD(c->U, VEL + dim, id) / FLD(c->U, DEN, id);
			double E_new = pre_new / (c->gamma - 1.0) + ke;
			FLD(c->UDOT, PRE, id) += (E_new - FLD(c->U, PRE, id)) / dt;
		} else if (c->p.coupling == CP_NEQ) {
			FLD(c->UDOT, PRE, id) += FLD(c->R, R_HEAT, id);
		}
		FLD(c->UDOT, HII, id) += (FLD(c->Q, HII, id) * FLD(c->Q, DEN, id) - FLD(c->U, HII, id)) / dt;
		FLD(c->UDOT, ADV, id) += (FLD(c->Q, ADV, id) * FLD(c->Q, DEN, id) - FLD(c->U, ADV, id)) / dt;
	}
}

/* ---------------------------------------------------------- thermodynamics --- */
static double flux_fuv(const orc_ctx* c, double Q_FUV, double dist_sqrd) {
	/* Thermodynamics.cpp:117-122 */
	return dist_sqrd != 0 ? Q_FUV / (1.2e7 * 4 * c->pi * dist_sqrd) : 0;
}
static double imlc(const orc_ctx* c, double ne, double T) {
	return c->imlc * c->z0 * ne * ne * m_exp(-c->T1 / T - (c->T2 / T) * (c->T2 / T));
}
static double nmlc(const orc_ctx* c, double ne, double nn, double T) {
	return c->nmlc * c->z0 * ne * nn * m_exp(-c->T3 / T - (c->T4 / T) * (c->T4 / T));
}
static double ciec(const orc_ctx* c, double ne, double T) {
	/* Thermodynamics.cpp:135-143 */
	if (T > c->ciec_minT) {
		double cie_rate = c->ciec * ne * ne * c->z0 * m_exp(-0.63 * m_log(T)) * (1.0 - m_exp(-m_pow(1.0e-5 * T, 1.63)));
		double smoothing = smin(1.0, (T - 5.0e4) / (2.0e4));
		return cie_rate * smoothing;
	}
	return 0;
}
static double nmc(const orc_ctx* c, double nH, double x, double T) {
	/* Thermodynamics.cpp:146-149 */
	double T0 = 70.0 + 220.0 * m_pow(nH / c->n0, 0.2);
	return c->nmc * (1.0 - x) * (1.0 - x) * m_pow(nH, 1.6) * sqrt(T) * m_exp(-T0 / T);
}
static double cxhi(const orc_ctx* c, double nH, double x, double T) {
	/* Thermodynamics.cpp:161-166 */
	double rate = spline_eval(&c->th_cxhi, m_log10(T));
	return x * (1.0 - x) * nH * nH * m_exp((2.302585093 * rate) - ((T / c->cxhi_damp) * (T / c->cxhi_damp)));
}
static double fuvh(const orc_ctx* c, double nH, double Av, double F) {
	return c->fuvh_a * nH * F * m_exp(-1.9 * Av) / (c->fuvh_b + c->fuvh_c * F * m_exp(-1.9 * Av) / nH);
}
static double irh(const orc_ctx* c, double nH, double Av, double F) {
	return c->irh_a * nH * F * m_exp(-0.05 * Av) * m_exp(-2.0 * m_log(1.0 + c->irh_b / nH));
}
static double soft_landing(double rate, double T, double T_min) {
	/* Thermodynamics.cpp:202-211 */
	double result = rate;
	if (rate < 0.0) {
		if (T <= T_min) result = 0;
		else if (T <= T_min + 200) result = rate * (T - T_min) / 200;
	}
	return result;
}

static void update_colden(orc_ctx* c, long id, double dist2) {
	/* Thermodynamics::updateColDen, Thermodynamics.cpp:339-363 */
	if (dist2 > 0.95 * 0.95) {
		double colden[4] = {0, 0, 0, 0}, w[4];
		for (int i = 0; i < 4; ++i) {
			int nb = FLD(c->nbr, i, id);
			if (nb != -1) colden[i] = FLD(c->T, T_COL_DEN, nb) + FLD(c->T, T_DCOL_DEN, nb);
			w[i] = colden[i] == 0 ? 0 : FLD(c->nbw, i, id) / colden[i];
		}
		double sum_w = w[0] + w[1] + w[2] + w[3];
		double newcolden = 0.0;
		for (int i = 0; i < 4 && sum_w != 0; ++i) {
			w[i] = w[i] / sum_w;
			newcolden += w[i] * colden[i];
		}
		FLD(c->T, T_COL_DEN, id) = newcolden;
		FLD(c->T, T_DCOL_DEN, id) = (FLD(c->Q, DEN, id) / c->hydrogenMass) * c->ds[id];
	} else {
		FLD(c->T, T_COL_DEN, id) = 0;
		FLD(c->T, T_DCOL_DEN, id) = (FLD(c->Q, DEN, id) / c->hydrogenMass) * c->ds[id];
	}
}

static void thermo_ray_trace(orc_ctx* c) {
	/* Thermodynamics::rayTrace, Thermodynamics.cpp:365-417 (single rank) */
	for (long w = 0; w < c->nwind; ++w) update_colden(c, c->wind[w], cell_dist2(c, c->wind[w]));
	for (long k = 0; k < c->nnonwind; ++k) update_colden(c, c->nonwind[k], cell_dist2(c, c->nonwind[k]));
}

static void thermo_pre(orc_ctx* c) {
	/* Thermodynamics::preTimeStepCalculations, Thermodynamics.cpp:218-264 */
	if (c->p.star_on) thermo_ray_trace(c);
	for (long k = 0; k < c->nnonwind; ++k) {
		long id = c->nonwind[k];
		if (FLD(c->Q, ADV, id) < c->p.thermo_hii_switch) {
			FLD(c->T, T_RATE, id) = 0;
			continue;
		}
		double nH = c->X * FLD(c->Q, DEN, id) / c->hydrogenMass;
		double x = FLD(c->Q, HII, id);
		double ne = nH * (x);
		double nn = nH * (1.0 - x);
		double T = calc_temperature(c, FLD(c->Q, HII, id), FLD(c->Q, PRE, id), FLD(c->Q, DEN, id));
		double rsqrd = 0, F_FUV = 0;
		if (c->p.star_on) {
			double xc[3];
			cell_xc(c, id, xc);
			for (int i = 0; i < c->nd; ++i)
				rsqrd += (xc[i] - c->sxc[i]) * (xc[i] - c->sxc[i]) * c->dx[i] * c->dx[i];
			F_FUV = flux_fuv(c, 0.5 * c->photonRate, rsqrd);
		}
		double tau = FLD(c->T, T_COL_DEN, id);
		double Av_FUV = 1.086 * c->dustXsec * tau;
		double rate = 0;
		rate += fuvh(c, nH, Av_FUV, F_FUV);
		rate += irh(c, nH, Av_FUV, F_FUV);
		rate += c->crh * nH;
		FLD(c->T, T_HEAT, id) = rate;
		rate -= imlc(c, ne, T);
		rate -= nmlc(c, ne, nn, T);
		rate -= cxhi(c, nH, x, T);
		rate -= ciec(c, ne, T);
		rate -= nmc(c, nH, x, T);
		rate = soft_landing(rate, T, c->Tmin[id]);
		FLD(c->T, T_RATE, id) = c->p.heating_amp * rate;
	}
}

static void thermo_integrate(orc_ctx* c, double dt) {
	/* Thermodynamics::integrate, Thermodynamics.cpp:266-337 */
	if (!c->p.thermo_subcycling) return;
	for (long k = 0; k < c->nnonwind; ++k) {
		long id = c->nonwind[k];
		if (FLD(c->Q, ADV, id) < c->p.thermo_hii_switch) {
			FLD(c->T, T_RATE, id) = 0;
			continue;
		}
		double qden = FLD(c->Q, DEN, id), qpre = FLD(c->Q, PRE, id), x = FLD(c->Q, HII, id);
		double Tmin = c->Tmin[id];
		double nH = c->X * qden / c->hydrogenMass;
		double ne = nH * (x);
		double nn = nH * (1.0 - x);
		double dti = fabs(0.10 * FLD(c->U, PRE, id) / FLD(c->T, T_RATE, id));
		double mu_inv = c->X * (x + 1.0) + (1.0 - c->X) * 0.25;
		double pre2temp = 1.0 / (mu_inv * c->specificGasConstant * qden);
		double temp2pre = (mu_inv * c->specificGasConstant * qden);
		double rate2dpre = smin(dt, dti) * (c->gamma - 1.0);
		double dpre2rate = 1.0 / rate2dpre;
		double pressure = qpre + FLD(c->T, T_RATE, id) * rate2dpre;
		double subcycleT = pressure * pre2temp;
		if (pressure < c->pfloor || subcycleT < Tmin) {
			double pfl = smax(Tmin * temp2pre, c->pfloor);
			subcycleT = pfl * pre2temp;
			pressure = pfl;
		}
		if (dt > dti) {
			double dtdti = dt / dti;
			int nsteps = dtdti - (int)dtdti > 0 ? (int)(dtdti + 1.0) : (int)(dtdti + 0.5);
			--nsteps;
			for (int i = 0; i < nsteps; ++i) {
				double r = FLD(c->T, T_HEAT, id);
				r -= imlc(c, ne, subcycleT);
				r -= nmlc(c, ne, nn, subcycleT);
				r -= cxhi(c, nH, x, subcycleT);
				r -= ciec(c, ne, subcycleT);
				r -= nmc(c, nH, x, subcycleT);
				r = c->p.heating_amp * soft_landing(r, subcycleT, Tmin);
				pressure += r * rate2dpre;
				subcycleT = pressure * pre2temp;
				if (pressure < c->pfloor || subcycleT < Tmin) {
					double pfl = smax(Tmin * temp2pre, c->pfloor);
					subcycleT = pfl * pre2temp;
					pressure = pfl;
				}
			}
		}
		FLD(c->T, T_RATE, id) = (pressure - qpre) * dpre2rate;
	}
}

static double thermo_dt(orc_ctx* c) {
	/* Thermodynamics::calculateTimeStep, Thermodynamics.cpp:463-476 */
	double dt = c->dt_max;
	for (long id = 0; id < c->N; ++id) {
		double rate = FLD(c->T, T_RATE, id);
		if (rate != 0) {
			double frac = c->p.thermo_subcycling ? 1.0 : 0.1;
			double dti = fabs(frac * FLD(c->U, PRE, id) / rate);
			if (dti < dt) dt = dti;
		}
	}
	return dt;
}

static void thermo_source_terms(orc_ctx* c) {
	/* Thermodynamics::updateSourceTerms, Thermodynamics.cpp:478-485 */
	for (long k = 0; k < c->nnonwind; ++k) {
		long id = c->nonwind[k];
		FLD(c->UDOT, PRE, id) += FLD(c->T, T_RATE, id);
		FLD(c->T, T_RATE, id) = FLD(c->T, T_HEAT, id) = 0;
	}
}

/* ------------------------------------------------------------------ driver --- */
static int calculate_time_step(orc_ctx* c, double* dt_out) {
	/* Torch::calculateTimeStep, Torch.cpp:304-339 */
	double dt;
	if (c->first_time) {
		dt = c->dt_max * 1.0e-20;
		c->first_time = 0;
	} else {
		double dt_hydro = hydro_dt(c);
		double dt_rad = dt_hydro, dt_thermo = dt_hydro;
		if (c->p.radiation_on) {
			int e = rad_dt(c, &dt_rad);
			if (e) return e;
		}
		if (c->p.cooling_on) dt_thermo = thermo_dt(c);
		dt = smin(smin(dt_hydro, dt_rad), dt_thermo);
	}
	*dt_out = dt;
	return 0;
}

static int comp_pre(orc_ctx* c, int comp) {
	if (comp == COMP_RAD) return rad_pre(c);
	if (comp == COMP_THERMO) thermo_pre(c);
	return 0;
}

static int sub_step(orc_ctx* c, double dt, int hasCalculatedHeatFlux, int comp) {
	/* Torch::subStep, Torch.cpp:352-364 */
	int e = check_values(c);
	if (e) return e;
	if (!hasCalculatedHeatFlux) {
		global_QfromU(c);
		fix_primitives(c);
		if ((e = comp_pre(c, comp))) return e;
	}
	switch (comp) {
	case COMP_HYDRO:
		if ((e = hydro_fluxes(c))) return e;
		hydro_source_terms(c);
		break;
	case COMP_RAD:
		if ((e = transfer_radiation(c, dt))) return e;
		rad_source_terms(c, dt);
		break;
	default:
		thermo_integrate(c, dt);
		thermo_source_terms(c);
		break;
	}
	adv_solution(c, dt);
	if ((e = fix_solution(c))) return e;
	return check_values(c);
}

static int hydro_step(orc_ctx* c, double dt) {
	/* Torch::hydroStep (hasCalculatedHeatFlux = true), Torch.cpp:366-387 */
	int e = check_values(c);
	if (e) return e;
	memcpy(c->W, c->U, sizeof(double) * NU * c->N);
	if ((e = hydro_fluxes(c))) return e;
	hydro_source_terms(c);
	adv_solution(c, dt / 2.0);
	if ((e = fix_solution(c))) return e;
	global_QfromU(c);
	memcpy(c->U, c->W, sizeof(double) * NU * c->N);
	if ((e = hydro_fluxes(c))) return e;
	hydro_source_terms(c);
	adv_solution(c, dt);
	return fix_solution(c);
}

int orc_full_step(orc_ctx* c, double dt_next_checkpoint, double* dt_out) {
	/* Torch::fullStep, Torch.cpp:389-418 */
	int e;
	global_QfromU(c);
	fix_primitives(c);
	if (c->p.cooling_on) thermo_pre(c);
	if (c->p.radiation_on && (e = rad_pre(c))) return e;
	double dtc;
	if ((e = calculate_time_step(c, &dtc))) return e;
	double dt = smin(dt_next_checkpoint, dtc);
	if (c->nactive == 1) {
		if ((e = hydro_step(c, dt))) return e;
	} else {
		int ncomps = c->nactive;
		c->stepCounter = (c->stepCounter + 1) % ncomps;
		for (int i = 0; i < ncomps; ++i) {
			double h = (i == ncomps - 1) ? 1.0 : 0.5;
			if ((e = sub_step(c, h * dt, i == 0, c->active[(i + c->stepCounter) % ncomps]))) return e;
		}
		for (int i = ncomps - 2; i >= 0; --i)
			if ((e = sub_step(c, dt / 2.0, 0, c->active[(i + c->stepCounter) % ncomps]))) return e;
	}
	c->time += dt;
	*dt_out = dt;
	return 0;
}

/* ------------------------------------------------------------------- setup --- */
static void init_tables(orc_ctx* c) {
	/* Radiation::initRecombinationHummer, Radiation.cpp:184-207 */
	static const double alphab[31] = {9.283e-11, 8.823e-11, 8.361e-11, 7.898e-11, 7.435e-11,
		6.973e-11, 6.512e-11, 6.054e-11, 5.599e-11, 5.147e-11, 4.700e-11,
		4.258e-11, 3.823e-11, 3.397e-11, 2.983e-11, 2.584e-11, 2.204e-11,
		1.847e-11, 1.520e-11, 1.226e-11, 9.696e-12, 7.514e-12, 5.710e-12,
		4.257e-12, 3.117e-12, 2.244e-12, 1.590e-12, 1.110e-12, 7.642e-13,
		5.199e-13, 3.498e-13};
	static const double coolb[31] = {8.287e-11, 7.821e-11, 7.356e-11, 6.892e-11, 6.430e-11,
		5.971e-11, 5.515e-11, 5.062e-11, 4.614e-11, 4.170e-11, 3.734e-11,
		3.306e-11, 2.888e-11, 2.484e-11, 2.098e-11, 1.736e-11, 1.402e-11,
		1.103e-11, 8.442e-12, 6.279e-12, 4.539e-12, 3.192e-12, 2.185e-12,
		1.458e-12, 9.484e-13, 6.023e-13, 3.738e-13, 2.268e-13, 1.348e-13,
		7.859e-14, 4.499e-14};
	double xs[31], yr[31], yc[31];
	for (int i = 0; i < 31; i++) {
		double T = exp(log(10.0) * (1.0 + 0.2 * (double)i));
		double sqrt_T = sqrt(T);
		xs[i] = T;
		yr[i] = TO_CODE(&c->cv, alphab[i] / sqrt_T, 0, 3, -1);
		yc[i] = TO_CODE(&c->cv, coolb[i] / sqrt_T, 0, 3, -1);
	}
	spline_init(&c->rad_recomb, xs, yr, 31, 0);
	spline_init(&c->rad_cool, xs, yc, 31, 0);
	/* Thermodynamics::initRecombinationHII uses the first 26 points, Thermodynamics.cpp:83-100 */
	spline_init(&c->th_recomb, xs, yc, 26, 0);
	/* Thermodynamics::initCollisionalExcitationHI, Thermodynamics.cpp:59-77 */
	static const double Tc[26] = {3162.2776602, 3981.0717055, 5011.8723363, 6309.5734448, 7943.2823472,
		10000.0000000, 12589.2541179, 15848.9319246, 19952.6231497, 25118.8643151,
		31622.7766017, 39810.7170553, 50118.7233627, 63095.7344480, 79432.8234724,
		100000.0000000, 125892.5411794, 158489.3192461, 199526.2314969, 251188.6431510,
		316227.7660168, 398107.1705535, 501187.2336273, 630957.3444802, 794328.2347243,
		1000000.0000000};
	static const double Rc[26] = {1.150800e-34, 2.312065e-31, 9.571941e-29, 1.132400e-26, 4.954502e-25,
		9.794900e-24, 1.035142e-22, 6.652732e-22, 2.870781e-21, 9.036495e-21, 2.218196e-20,
		4.456562e-20, 7.655966e-20, 1.158777e-19, 1.588547e-19, 2.013724e-19, 2.393316e-19,
		2.710192e-19, 2.944422e-19, 3.104560e-19, 3.191538e-19, 3.213661e-19, 3.191538e-19,
		3.126079e-19, 3.033891e-19, 2.917427e-19};
	double lx[26], ly[26];
	for (int i = 0; i < 26; i++) {
		lx[i] = log10(Tc[i]);
		ly[i] = log10(TO_CODE(&c->cv, Rc[i], 1, 5, -3));
	}
	spline_init(&c->th_cxhi, lx, ly, 26, 1);
}

static int setup(orc_ctx* c, const double* den, const double* pre, const double* hii,
                 const double* v0, const double* v1, const double* v2, const double* grav) {
	orc_params* p = &c->p;
	conv_t* cv = &c->cv;
	/* Constants::initialise_DPT, Constants.cpp:27-50 */
	conv_init(cv);
	conv_set_dpt(cv, p->dscale, p->pscale, p->tscale);
	c->hydrogenMass = TO_CODE(cv, 1.674e-24, 1, 0, 0);
	c->specificGasConstant = TO_CODE(cv, 8.314462e7, 0, 2, -2);
	c->boltzmannConst = TO_CODE(cv, 1.3806488e-16, 1, 2, -2);
	c->rydbergEnergy = TO_CODE(cv, 13.6 * 1.60217646e-12, 1, 2, -2);
	c->dustXsec = TO_CODE(cv, 5.0e-22, 0, 2, 0);
	c->pi = 3.14159265359;
	c->voronov_A = TO_CODE(cv, 2.91e-8, 0, 3, -1);
	c->voronov_X = 0.232;
	c->voronov_K = 0.39;
	c->voronov_P = 0.0;
	c->voronov_DE = c->rydbergEnergy / c->boltzmannConst;
	/* TorchParameters::initialise, Parameters.cpp:9-27 */
	c->tmax = TO_CODE(cv, p->tmax, 0, 0, 1);
	c->dt_max = c->tmax / 10.0;
	c->side = TO_CODE(cv, p->side_length, 0, 1, 0);
	for (int i = 0; i < 3; ++i) { c->lbc[i] = p->left_bc[i]; c->rbc[i] = p->right_bc[i]; }
	if (p->geometry == G_SPH || p->geometry == G_CYL) c->lbc[0] = BC_REFLECTING;
	c->photoIonXsec = TO_CODE(cv, p->photoion_xsec, 0, 2, 0);
	c->alphaB = TO_CODE(cv, p->alphaB, 0, 3, -1);
	c->dfloor = TO_CODE(cv, p->dfloor, 1, -3, 0);
	c->tfloor = p->tfloor;
	c->pfloor = 0.1 * c->specificGasConstant * c->dfloor * c->tfloor;
	c->photonEnergy = TO_CODE(cv, p->photon_energy, 1, 2, -2);
	c->photonRate = TO_CODE(cv, p->photon_rate, 0, 0, -1);
	c->massLossRate = TO_CODE(cv, p->mass_loss_rate, 1, 0, -1);
	c->windVelocity = TO_CODE(cv, p->wind_velocity, 0, 1, -1);
	if (!p->star_on) {
		/* TorchParameters::getStarParameters leaves these at zero (Parameters.cpp:80-95) */
		c->photonEnergy = c->photonRate = c->massLossRate = c->windVelocity = 0;
	}
	c->gamma = p->gamma;
	c->X = p->mass_frac_h;
	c->nd = p->nd;
	c->nx = p->ncells[0]; c->ny = p->ncells[1]; c->nz = p->ncells[2];
	c->order = p->spatial_order;
	if (c->order != 0 && c->order != 1)
		return fail(c, ORC_ERR_PARAM, "spatial_order must be 0 or 1");
	c->ng = c->order + 1;
	c->geometry = p->geometry;
	c->N = (long)c->nx * c->ny * c->nz;
	/* Grid::initialise, Grid.cpp:470-471 */
	for (int i = 0; i < 3; ++i) c->dx[i] = 0;
	for (int i = 0; i < c->nd; ++i) c->dx[i] = c->side / (double)c->nx;

	long N = c->N;
	c->U = (double*)calloc(NU * N, sizeof(double));
	c->Q = (double*)calloc(NU * N, sizeof(double));
	c->W = (double*)calloc(NU * N, sizeof(double));
	c->UDOT = (double*)calloc(NU * N, sizeof(double));
	c->R = (double*)calloc(NR * N, sizeof(double));
	c->T = (double*)calloc(NT * N, sizeof(double));
	c->Tmin = (double*)calloc(N, sizeof(double));
	c->grav = (double*)calloc(3 * N, sizeof(double));
	c->vol = (double*)calloc(N, sizeof(double));
	c->ds = (double*)calloc(N, sizeof(double));
	c->shellVol = (double*)calloc(N, sizeof(double));
	c->nbr = (int*)calloc(4 * N, sizeof(int));
	c->nbw = (double*)calloc(4 * N, sizeof(double));
	for (int d = 0; d < 3; ++d) {
		int n = ncell_dim(c, d);
		c->gcount[d] = N / n;
		c->nfaces[d] = c->gcount[d] * (n + 1);
		if (d < c->nd) {
			c->F[d] = (double*)calloc(NU * c->nfaces[d], sizeof(double));
			c->ghostQ[d][0] = (double*)calloc((size_t)c->ng * NU * c->gcount[d], sizeof(double));
			c->ghostQ[d][1] = (double*)calloc((size_t)c->ng * NU * c->gcount[d], sizeof(double));
		}
	}
	for (long id = 0; id < N; ++id) {
		double xc[3];
		cell_xc(c, id, xc);
		c->vol[id] = cell_volume(c, xc[0]);
	}

	/* Star::initialise, Star.cpp:13-40 */
	for (int i = 0; i < 3; ++i) {
		double mod = (p->face_snap[i] && (p->star_pos[i] == 0)) ? 0.5 : 0;
		c->sxc[i] = p->star_pos[i] + 0.5 - mod;
	}
	if (c->nd < 3) c->sxc[2] = 0;
	if (c->nd < 2) c->sxc[1] = 0;

	/* Fluid::initialiseGrid, Fluid.cpp:31-57 */
	build_causal(c);
	c->starCell = within(c, p->star_pos) ? (int)flat(c, p->star_pos[0], p->star_pos[1], p->star_pos[2]) : -1;
	c->wind = (int*)malloc(sizeof(int) * (c->ncausal + 1));
	c->nonwind = (int*)malloc(sizeof(int) * (c->ncausal + 1));
	c->nwind = c->nnonwind = 0;
	int wr = p->star_on ? p->wind_cell_radius : 0;
	for (long k = 0; k < c->ncausal; ++k) {
		long id = c->causal[k];
		double xc[3], dist2 = 0;
		cell_xc(c, id, xc);
		for (int i = 0; i < c->nd; ++i)
			dist2 += ((int)xc[i] - p->star_pos[i]) * (xc[i] - p->star_pos[i]);
		if (dist2 <= wr * wr || id == c->starCell) c->wind[c->nwind++] = (int)id;
		else c->nonwind[c->nnonwind++] = (int)id;
	}
	/* Star::setWindCells, Star.cpp:42-51 */
	{
		double volume = 0;
		for (long w = 0; w < c->nwind; ++w) volume += c->vol[c->wind[w]];
		c->mdot = c->massLossRate / volume;
		c->edot = 0.5 * c->mdot * c->windVelocity * c->windVelocity;
	}
	init_tables(c);
	/* Thermodynamics::initialise constants, Thermodynamics.cpp:33-54 */
	c->z0 = 5.0e-4;
	c->th_excess = TO_CODE(cv, 5 * 1.60217646e-12, 1, 2, -2);
	c->T1 = 33610; c->T2 = 2180; c->T3 = 28390; c->T4 = 1780;
	c->imlc = TO_CODE(cv, 2.905e-19, 1.0, 5.0, -3.0);
	c->nmlc = TO_CODE(cv, 4.477e-20, 1.0, 5.0, -3.0);
	c->ciec_minT = 5.0e4;
	c->ciec = TO_CODE(cv, 3.485e-15, 1.0, 5.0, -3.0);
	c->cxhi_damp = 5.0e5;
	c->n0 = TO_CODE(cv, 1.0e6, 0.0, -3.0, 0.0);
	c->nmc = TO_CODE(cv, 3.981e-27, 1.0, 3.8, -3.0);
	c->fuvh_a = TO_CODE(cv, 1.9e-26, 1.0, 4.0, -2.0);
	c->fuvh_b = TO_CODE(cv, 1.00000, 0.0, 0.0, -1.0);
	c->fuvh_c = TO_CODE(cv, 6.40000, 0.0, -1.0, 0.0);
	c->irh_a = TO_CODE(cv, 7.7e-32, 1.0, 4.0, -2.0);
	c->irh_b = TO_CODE(cv, 3.0e4, 0.0, -3.0, 0.0);
	c->crh = TO_CODE(cv, 5.0e-27, 1.0, 2.0, -3.0);
	c->th_Tmin = 100;

	/* DataReader::readGrid (DataReader.cpp:70-125) / setUpLua: primitives in cgs */
	for (long id = 0; id < N; ++id) {
		FLD(c->Q, DEN, id) = den[id];
		FLD(c->Q, PRE, id) = pre[id];
		FLD(c->Q, HII, id) = hii[id];
		FLD(c->Q, VEL + 0, id) = (c->nd > 0 && v0) ? v0[id] : 0;
		FLD(c->Q, VEL + 1, id) = (c->nd > 1 && v1) ? v1[id] : 0;
		FLD(c->Q, VEL + 2, id) = (c->nd > 2 && v2) ? v2[id] : 0;
		if (grav)
			for (int d = 0; d < 3; ++d) FLD(c->grav, d, id) = grav[d * N + id];
	}
	/* Thermodynamics::initialiseMinTempField, Thermodynamics.cpp:103-112 (before code units) */
	for (long id = 0; id < N; ++id)
		c->Tmin[id] = p->min_temp_initial_state
			? calc_temperature(c, FLD(c->Q, HII, id), FLD(c->Q, PRE, id), FLD(c->Q, DEN, id))
			: c->th_Tmin;
	/* Torch::toCodeUnits, Torch.cpp:146-155 */
	for (long id = 0; id < N; ++id) {
		FLD(c->Q, DEN, id) = TO_CODE(cv, FLD(c->Q, DEN, id), 1, -3, 0);
		FLD(c->Q, PRE, id) = TO_CODE(cv, FLD(c->Q, PRE, id), 1, -1, -2);
		for (int d = 0; d < c->nd; ++d)
			FLD(c->Q, VEL + d, id) = TO_CODE(cv, FLD(c->Q, VEL + d, id), 0, 1, -1);
		for (int d = 0; d < c->nd; ++d)
			FLD(c->grav, d, id) = TO_CODE(cv, FLD(c->grav, d, id), 1, -2, -2);
	}
	fix_primitives(c);
	global_UfromQ(c);
	/* Radiation::initField, Radiation.cpp:78-96 */
	nearest_neighbours(c);
	for (long id = 0; id < N; ++id) {
		double xc[3], d[3] = {0, 0, 0}, denom;
		cell_xc(c, id, xc);
		for (int i = 0; i < c->nd; ++i) d[i] = fabs(xc[i] - c->sxc[i]);
		/* Radiation::cellPathLength, Radiation.cpp:102-117 */
		if (d[2] >= d[1] && d[2] >= d[0]) denom = d[2];
		else if (d[1] > d[2] && d[1] >= d[0]) denom = d[1];
		else denom = d[0];
		c->ds[id] = denom != 0
			? sqrt(d[0] * d[0] * c->dx[0] * c->dx[0] + d[1] * d[1] * c->dx[1] * c->dx[1] + d[2] * d[2] * c->dx[2] * c->dx[2]) / denom
			: 0.0;
		double r_sqrd = 0;
		for (int i = 0; i < c->nd; ++i)
			r_sqrd += (xc[i] - c->sxc[i]) * (xc[i] - c->sxc[i]) * c->dx[i] * c->dx[i];
		/* Radiation::shellVolume, Radiation.cpp:119-138 */
		double dsv = c->ds[id];
		if (r_sqrd <= 100.0 * dsv * dsv) {
			double r = sqrt(r_sqrd);
			double r_min = r - 0.5 * dsv, r_max = r + 0.5 * dsv;
			c->shellVol[id] = 4.0 * c->pi * (r_max * r_max * r_max - r_min * r_min * r_min) / 3.0;
		} else
			c->shellVol[id] = 4.0 * c->pi * r_sqrd * dsv;
		double nH = c->X * FLD(c->Q, DEN, id) / c->hydrogenMass;
		FLD(c->R, R_DTAU, id) = (1.0 - FLD(c->Q, HII, id)) * nH * c->photoIonXsec * c->ds[id];
		FLD(c->R, R_DTAU_A, id) = (1.0 - FLD(c->R, R_HII_A, id)) * nH * c->photoIonXsec * c->ds[id];
	}
	/* Torch::run prologue, Torch.cpp:245-264 */
	global_QfromU(c);
	fix_primitives(c);
	c->nactive = 0;
	c->active[c->nactive++] = COMP_HYDRO;
	if (p->cooling_on) c->active[c->nactive++] = COMP_THERMO;
	if (p->radiation_on) c->active[c->nactive++] = COMP_RAD;
	if (p->star_on) thermo_ray_trace(c); /* fillHeatingArrays' ray trace, Thermodynamics.cpp:420-421 */
	c->time = 0;
	c->first_time = 1;
	c->rad_once = 0;
	c->stepCounter = 0;
	return 0;
}

orc_ctx* orc_create(const orc_params* p, const double* den, const double* pre, const double* hii,
                    const double* v0, const double* v1, const double* v2, const double* grav,
                    char* err, int errlen) {
	orc_ctx* c = (orc_ctx*)calloc(1, sizeof(orc_ctx));
	c->p = *p;
	if (setup(c, den, pre, hii, v0, v1, v2, grav)) {
		if (err && errlen > 0) snprintf(err, errlen, "%s", c->err);
		orc_destroy(c);
		return NULL;
	}
	return c;
}

void orc_get_state(const orc_ctx* c, double* U, double* Q, double* R, double* T, double* Tmin) {
	if (U) memcpy(U, c->U, sizeof(double) * NU * c->N);
	if (Q) memcpy(Q, c->Q, sizeof(double) * NU * c->N);
	if (R) memcpy(R, c->R, sizeof(double) * NR * c->N);
	if (T) memcpy(T, c->T, sizeof(double) * NT * c->N);
	if (Tmin) memcpy(Tmin, c->Tmin, sizeof(double) * c->N);
}

double orc_time(const orc_ctx* c) { return c->time; }
double orc_dt_max(const orc_ctx* c) { return c->dt_max; }
long orc_ncells(const orc_ctx* c) { return c->N; }
const char* orc_last_error(const orc_ctx* c) { return c->err; }

long orc_causal_order(const orc_ctx* c, int* out, long cap) {
	long n = c->ncausal < cap ? c->ncausal : cap;
	if (out) memcpy(out, c->causal, sizeof(int) * n);
	return c->ncausal;
}

long orc_cell_volumes(const orc_ctx* c, double* out, long cap) {
	long n = c->N < cap ? c->N : cap;
	if (out) memcpy(out, c->vol, sizeof(double) * n);
	return c->N;
}

void orc_destroy(orc_ctx* c) {
	if (!c) return;
	free(c->U); free(c->Q); free(c->W); free(c->UDOT); free(c->R); free(c->T);
	free(c->Tmin); free(c->grav); free(c->vol); free(c->ds); free(c->shellVol);
	free(c->nbr); free(c->nbw); free(c->causal); free(c->wind); free(c->nonwind);
	for (int d = 0; d < 3; ++d) {
		free(c->F[d]);
		free(c->ghostQ[d][0]);
		free(c->ghostQ[d][1]);
	}
	free(c);
}
