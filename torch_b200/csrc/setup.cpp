// Host-side set-up of a run (compiled with -ffp-contract=off so that the
// FP64 arithmetic rounds like the reference's host code).
//
// Restates, in order:
//   Converter / Constants                  src/Torch/Converter.cpp:17-63, src/Torch/Constants.cpp:27-50
//   TorchParameters::initialise            src/Torch/Parameters.cpp:9-27
//   Grid geometry, Star, wind cells        src/Fluid/Grid.cpp:461-566, src/Fluid/Star.cpp:13-51,
//                                          src/Fluid/Fluid.cpp:31-57
//   Radiation / Thermodynamics tables      src/Integrators/Radiation.cpp:184-207,
//                                          src/Integrators/Thermodynamics.cpp:24-100,
//                                          src/Integrators/SplineData.cpp:15-140
//   initial state                          src/Torch/Torch.cpp:101-118 (readGrid/setUpLua,
//                                          initialiseMinTempField, toCodeUnits, fixPrimitives,
//                                          globalUfromQ) and Radiation::initField (Radiation.cpp:78-138)
// and builds the shell order of the causal sweeps.
#include "setup.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace trg {
namespace {

struct Converter {
	double M = 1.0 * 2.0e33, L = 14.6 * 3.09e18, T = 10000.0 * 3.15569e7;

	void set_rho_pressure_time(double rho, double pressure, double time) {
		double rho_0 = (rho > 0) ? rho : M / (L * L * L);
		double pressure_0 = (pressure > 0) ? pressure : rho_0 * L * L / (T * T);
		double time_0 = (time > 0) ? time : T;
		T = time_0;
		M = std::sqrt((pressure_0 / rho_0) * pressure_0 * pressure_0) * T * T * T;
		L = std::sqrt(pressure_0 / rho_0) * T;
	}

	double to_code(double val, double mi, double li, double ti) const {
		double MM = mi >= 0 ? M : 1.0 / M;
		MM = 1.0 / MM;
		double LL = li >= 0 ? L : 1.0 / L;
		LL = 1.0 / LL;
		double TT = ti >= 0 ? T : 1.0 / T;
		TT = 1.0 / TT;
		int im = (int)std::abs(mi), il = (int)std::abs(li), it = (int)std::abs(ti);
		double result = val;
		while (im >= 1 || il >= 1 || it >= 1) {
			if (im-- >= 1) result *= MM;
			if (il-- >= 1) result *= LL;
			if (it-- >= 1) result *= TT;
		}
		double left = std::abs(mi) - (int)std::abs(mi);
		if (left != 0) result *= std::pow(MM, left);
		left = std::abs(li) - (int)std::abs(li);
		if (left != 0) result *= std::pow(LL, left);
		left = std::abs(ti) - (int)std::abs(ti);
		if (left != 0) result *= std::pow(TT, left);
		return result;
	}
};

inline double smin(double a, double b) { return (b < a) ? b : a; }
inline double smax(double a, double b) { return (a < b) ? b : a; }

void spline_build(Spline& s, const double* x, const double* y, int n, int log_mode) {
	s.n = n;
	s.log_mode = log_mode;
	for (int i = 0; i < n; ++i) { s.x[i] = x[i]; s.y[i] = y[i]; s.y2[i] = 0.0; }
	// natural cubic spline, SplineData::spline with yp1 = ypn = 1e99
	double u[32] = {0};
	for (int i = 1; i < n - 1; i++) {
		double sig = (s.x[i] - s.x[i - 1]) / (s.x[i + 1] - s.x[i - 1]);
		double p = sig * s.y2[i - 1] + 2.0;
		s.y2[i] = (sig - 1.0) / p;
		u[i] = (s.y[i + 1] - s.y[i]) / (s.x[i + 1] - s.x[i]) - (s.y[i] - s.y[i - 1]) / (s.x[i] - s.x[i - 1]);
		u[i] = (6.0 * u[i] / (s.x[i + 1] - s.x[i - 1]) - sig * u[i - 1]) / p;
	}
	double qn = 0.0, un = 0.0;
	s.y2[n - 1] = (un - qn * u[n - 2]) / (qn * s.y2[n - 2] + 1.0);
	for (int k = n - 2; k >= 0; k--) s.y2[k] = s.y2[k] * s.y2[k + 1] + u[k];
	if (log_mode) {
		s.min_slope = (s.y[1] - s.y[0]) / (s.x[1] - s.x[0]);
		s.max_slope = (s.y[n - 1] - s.y[n - 2]) / (s.x[n - 1] - s.x[n - 2]);
	} else {
		s.min_slope = (std::log10(s.y[1]) - std::log10(s.y[0])) / (std::log10(s.x[1]) - std::log10(s.x[0]));
		s.max_slope = (std::log10(s.y[n - 1]) - std::log10(s.y[n - 2])) / (std::log10(s.x[n - 1]) - std::log10(s.x[n - 2]));
	}
}

void build_tables(const Converter& cv, Tables& t) {
	static const double alphab[31] = {9.283e-11, 8.823e-11, 8.361e-11, 7.898e-11, 7.435e-11, 6.973e-11, 6.512e-11,
		6.054e-11, 5.599e-11, 5.147e-11, 4.700e-11, 4.258e-11, 3.823e-11, 3.397e-11, 2.983e-11, 2.584e-11, 2.204e-11,
		1.847e-11, 1.520e-11, 1.226e-11, 9.696e-12, 7.514e-12, 5.710e-12, 4.257e-12, 3.117e-12, 2.244e-12,
		1.590e-12, 1.110e-12, 7.642e-13, 5.199e-13, 3.498e-13};
	static const double coolb[31] = {8.287e-11, 7.821e-11, 7.356e-11, 6.892e-11, 6.430e-11, 5.971e-11, 5.515e-11,
		5.062e-11, 4.614e-11, 4.170e-11, 3.734e-11, 3.306e-11, 2.888e-11, 2.484e-11, 2.098e-11, 1.736e-11, 1.402e-11,
		1.103e-11, 8.442e-12, 6.279e-12, 4.539e-12, 3.192e-12, 2.185e-12, 1.458e-12, 9.484e-13, 6.023e-13,
		3.738e-13, 2.268e-13, 1.348e-13, 7.859e-14, 4.499e-14};
	// Hummer (1994) tables at log10 T = 1.0, 1.2, ..., 7.0 (Radiation.cpp:184-207)
	double xs[31], yr[31], yc[31];
	for (int i = 0; i < 31; i++) {
		double T = std::exp(std::log(10.0) * (1.0 + 0.2 * static_cast<double>(i)));
		double sqrt_T = std::sqrt(T);
		xs[i] = T;
		yr[i] = cv.to_code(alphab[i] / sqrt_T, 0, 3, -1);
		yc[i] = cv.to_code(coolb[i] / sqrt_T, 0, 3, -1);
	}
	spline_build(t.rad_recomb, xs, yr, 31, 0);
	spline_build(t.rad_cool, xs, yc, 31, 0);
	spline_build(t.th_recomb, xs, yc, 26, 0);  // the thermodynamics copy keeps 26 points (Thermodynamics.cpp:94)
	// H I collisional excitation, log-log (Thermodynamics.cpp:59-77)
	static const double Tc[26] = {3162.2776602, 3981.0717055, 5011.8723363, 6309.5734448, 7943.2823472,
		10000.0000000, 12589.2541179, 15848.9319246, 19952.6231497, 25118.8643151, 31622.7766017, 39810.7170553,
		50118.7233627, 63095.7344480, 79432.8234724, 100000.0000000, 125892.5411794, 158489.3192461,
		199526.2314969, 251188.6431510, 316227.7660168, 398107.1705535, 501187.2336273, 630957.3444802,
		794328.2347243, 1000000.0000000};
	static const double Rc[26] = {1.150800e-34, 2.312065e-31, 9.571941e-29, 1.132400e-26, 4.954502e-25,
		9.794900e-24, 1.035142e-22, 6.652732e-22, 2.870781e-21, 9.036495e-21, 2.218196e-20, 4.456562e-20,
		7.655966e-20, 1.158777e-19, 1.588547e-19, 2.013724e-19, 2.393316e-19, 2.710192e-19, 2.944422e-19,
		3.104560e-19, 3.191538e-19, 3.213661e-19, 3.191538e-19, 3.126079e-19, 3.033891e-19, 2.917427e-19};
	double lx[26], ly[26];
	for (int i = 0; i < 26; i++) {
		lx[i] = std::log10(Tc[i]);
		ly[i] = std::log10(cv.to_code(Rc[i], 1, 5, -3));
	}
	spline_build(t.th_cxhi, lx, ly, 26, 1);
}

struct Geo {
	const Params& P;
	explicit Geo(const Params& p) : P(p) {}
	void xc(long long id, double* x, int* ijk) const {
		ijk[0] = (int)(id % P.nx);
		ijk[1] = (int)((id / P.nx) % P.ny);
		ijk[2] = (int)(id / ((long long)P.nx * P.ny));
		for (int i = 0; i < 3; ++i) x[i] = (double)ijk[i];
		x[0] += (double)P.x0;  // a slab's cells at their global x
		for (int i = 0; i < P.nd; ++i) x[i] += 0.5;
	}
	double volume(double rc) const {
		const double PI = 3.14159265359;
		double volume = 0, r1, r2;
		if (P.geometry == G_CART) {
			volume = 1.0;
			for (int i = 0; i < P.nd; ++i) volume *= P.dx[i];
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
	bool within(const int* c) const {
		return c[0] >= 0 && c[0] < P.nx && c[1] >= 0 && c[1] < P.ny && c[2] >= 0 && c[2] < P.nz;
	}
};

// Grid::nextCausalCoords (Grid.cpp:255-356): the order of the reference's serial sweep.
void next_causal(const Geo& g, const int* from, const int* src, int* nxt) {
	const Params& P = g.P;
	int dir[3], begin[3];
	for (int i = 0; i < 3; ++i)
		dir[i] = (from[i] != src[i]) ? (int)((from[i] - src[i]) / std::fabs((double)(from[i] - src[i]))) : 1;
	for (int i = 0; i < 3; ++i) begin[i] = src[i] - (dir[i] < 0 ? 1 : 0);
	if (from[0] + dir[0] >= 0 && from[0] + dir[0] < P.nx) {
		nxt[0] = from[0] + dir[0]; nxt[1] = from[1]; nxt[2] = from[2];
	} else if (from[1] + dir[1] >= 0 && from[1] + dir[1] < P.ny) {
		nxt[0] = begin[0]; nxt[1] = from[1] + dir[1]; nxt[2] = from[2];
	} else if (from[2] + dir[2] >= 0 && from[2] + dir[2] < P.nz) {
		nxt[0] = begin[0]; nxt[1] = begin[1]; nxt[2] = from[2] + dir[2];
	} else {
		nxt[0] = nxt[1] = nxt[2] = -1;
	}
	const int nd = P.nd;
	auto jump = [&](int a, int b, int c) { nxt[0] = src[0] - a; nxt[1] = src[1] - b; nxt[2] = src[2] - c; };
	if (!g.within(nxt) && dir[0] == 1 && dir[1] == 1 && dir[2] == 1) { jump(1, 0, 0); dir[0] = -1; }
	if (!g.within(nxt) && dir[0] == -1 && dir[1] == 1 && dir[2] == 1 && nd > 1) { jump(0, 1, 0); dir[0] = 1; dir[1] = -1; }
	if (!g.within(nxt) && dir[0] == 1 && dir[1] == -1 && dir[2] == 1 && nd > 1) { jump(1, 1, 0); dir[0] = -1; }
	if (!g.within(nxt) && dir[0] == -1 && dir[1] == -1 && dir[2] == 1 && nd > 2) { jump(0, 0, 1); dir[0] = 1; dir[1] = 1; dir[2] = -1; }
	if (!g.within(nxt) && dir[0] == 1 && dir[1] == 1 && dir[2] == -1 && nd > 2) { jump(1, 0, 1); dir[0] = -1; }
	if (!g.within(nxt) && dir[0] == -1 && dir[1] == 1 && dir[2] == -1 && nd > 2) { jump(0, 1, 1); dir[0] = 1; dir[1] = -1; }
	if (!g.within(nxt) && dir[0] == 1 && dir[1] == -1 && dir[2] == -1 && nd > 2) { jump(1, 1, 1); dir[0] = -1; }
}

// Upwind neighbours and weights of Grid::calculateNearestNeighbours
// (Grid.cpp:922-952), used here only to verify the shell order.
void neighbour_cells(const Params& P, const int* ijk, const double* xc, long long* nb, double* w) {
	int plane = 0;
	double dmax = 0;
	for (int i = 0; i < P.nd; ++i) {
		double dd = std::fabs(xc[i] - P.sxc[i]);
		if (dd > dmax) { dmax = dd; plane = i; }
	}
	int irot[3] = {(plane + 1) % 3, (plane + 2) % 3, plane % 3};
	double d[3];
	int s[3], LR[3];
	for (int i = 0; i < 3; i++) {
		d[i] = xc[irot[i]] - P.sxc[irot[i]];
		s[i] = d[i] < -1.0 / 10.0 ? -1 : 1;
		LR[i] = std::fabs(d[i]) < 1.0 / 10.0 ? 0 : s[i];
	}
	const int off[4][3] = {{0, 0, -LR[2]}, {0, -LR[1], -LR[2]}, {-LR[0], 0, -LR[2]}, {-LR[0], -LR[1], -LR[2]}};
	for (int n = 0; n < 4; ++n) {
		int t[3] = {ijk[0], ijk[1], ijk[2]};
		for (int r = 0; r < 3; ++r) t[irot[r]] += off[n][r];
		bool in = t[0] >= 0 && t[0] < P.nx && t[1] >= 0 && t[1] < P.ny && t[2] >= 0 && t[2] < P.nz;
		nb[n] = in ? t[0] + (long long)P.nx * (t[1] + (long long)P.ny * t[2]) : -1;
	}
	double ic0 = (int)xc[irot[0]] - 0.5 * (s[2] * d[0] / d[2]);
	double ic1 = (int)xc[irot[1]] - 0.5 * (s[2] * d[1] / d[2]);
	double delta0 = std::fabs(2.0 * ic0 - 2.0 * (int)xc[irot[0]] + s[0]);
	double delta1 = std::fabs(2.0 * ic1 - 2.0 * (int)xc[irot[1]] + s[1]);
	w[0] = (std::fabs(d[2]) > 0.9) ? delta0 * delta1 : 0;
	w[1] = ((std::fabs(d[1]) > 0.9) && (std::fabs(d[2]) > 0.9)) ? delta0 * (1.0 - delta1) : 0;
	w[2] = ((std::fabs(d[0]) > 0.9) && (std::fabs(d[2]) > 0.9)) ? (1.0 - delta0) * delta1 : 0;
	w[3] = ((std::fabs(d[0]) > 0.9) && (std::fabs(d[1]) > 0.9) && (std::fabs(d[2]) > 0.9)) ? (1.0 - delta0) * (1.0 - delta1) : 0;
}

}  // namespace

std::string host_setup(const trg_params& p, const double* den, const double* pre, const double* hii, const double* v0,
                       const double* v1, const double* v2, const double* grav, HostSetup& out, const SlabSpec* slab) {
	Params& P = out.P;
	std::memset(&P, 0, sizeof(P));
	if (p.nd < 1 || p.nd > 3) return "nd must be 1, 2 or 3";
	for (int i = 0; i < 3; ++i)
		if (p.ncells[i] < 1) return "ncells must be positive";
	if ((p.nd < 3 && p.ncells[2] != 1) || (p.nd < 2 && p.ncells[1] != 1)) return "ncells beyond nd must be 1";
	if (p.spatial_order != 0 && p.spatial_order != 1)
		return "spatial_order must be 0 or 1 (Hydrodynamics::calcFluxes, Hydro.cpp:94-112)";
	if (p.rt_scheme < 0 || p.rt_scheme > 2) return "rt_scheme must be 0 (implicit), 1 (implicit2) or 2 (explicit)";
	if (!den || !pre || !hii || !v0) return "den, pre, hii and v0 are required";
	if (slab) {
		if ((p.radiation_on || p.cooling_on || p.star_on) && p.precision != TRG_PRECISION_FP64)
			return "slabs of a run with radiation, cooling or a star take the FP64 form";
		if (p.star_on && (p.mass_loss_rate != 0 || p.wind_cell_radius > 0))
			return "slabs take no stellar wind (its injection volume would be split over slabs)";
		if (slab->nx < 2 || slab->x0 < 0 || slab->x0 + slab->nx > p.ncells[0])
			return "a slab lies inside the grid and holds at least two x layers";
	}
	Converter cv;
	cv.set_rho_pressure_time(p.dscale, p.pscale, p.tscale);
	P.hydrogenMass = cv.to_code(1.674e-24, 1, 0, 0);
	P.specificGasConstant = cv.to_code(8.314462e7, 0, 2, -2);
	P.boltzmannConst = cv.to_code(1.3806488e-16, 1, 2, -2);
	P.rydbergEnergy = cv.to_code(13.6 * 1.60217646e-12, 1, 2, -2);
	P.dustXsec = cv.to_code(5.0e-22, 0, 2, 0);
	P.pi = 3.14159265359;
	P.voronov_A = cv.to_code(2.91e-8, 0, 3, -1);
	P.voronov_X = 0.232;
	P.voronov_K = 0.39;
	P.voronov_P = 0.0;
	P.voronov_DE = P.rydbergEnergy / P.boltzmannConst;

	out.tmax = cv.to_code(p.tmax, 0, 0, 1);
	out.dt_max = out.tmax / 10.0;
	P.dt_max = out.dt_max;
	double side = cv.to_code(p.side_length, 0, 1, 0);
	for (int i = 0; i < 3; ++i) { P.lbc[i] = p.left_bc[i]; P.rbc[i] = p.right_bc[i]; }
	if (p.geometry == G_SPH || p.geometry == G_CYL) P.lbc[0] = BC_REFLECTING;
	P.photoIonXsec = cv.to_code(p.photoion_xsec, 0, 2, 0);
	P.dfloor = cv.to_code(p.dfloor, 1, -3, 0);
	P.tfloor = p.tfloor;
	P.pfloor = 0.1 * P.specificGasConstant * P.dfloor * P.tfloor;
	double photonEnergy = cv.to_code(p.photon_energy, 1, 2, -2);
	double photonRate = cv.to_code(p.photon_rate, 0, 0, -1);
	double massLossRate = cv.to_code(p.mass_loss_rate, 1, 0, -1);
	double windVelocity = cv.to_code(p.wind_velocity, 0, 1, -1);
	if (!p.star_on) photonEnergy = photonRate = massLossRate = windVelocity = 0;  // Parameters.cpp:80-95
	P.photonEnergy = photonEnergy;
	P.photonRate = photonRate;
	P.gamma = p.gamma;
	P.X = p.mass_frac_h;
	P.nd = p.nd;
	P.nx = slab ? slab->nx : p.ncells[0]; P.ny = p.ncells[1]; P.nz = p.ncells[2];
	P.N = (long long)P.nx * P.ny * P.nz;
	P.x0 = slab ? slab->x0 : 0;
	if (slab) {
		// Grid.cpp:804-833: a face between two slabs takes its ghosts from the
		// neighbour (PARTITION); with periodic x the two ends are neighbours too
		const bool many = slab->nx < p.ncells[0];
		if (slab->x0 > 0 || (many && P.lbc[0] == BC_PERIODIC)) P.lbc[0] = BC_PARTITION;
		if (slab->x0 + slab->nx < p.ncells[0] || (many && P.rbc[0] == BC_PERIODIC)) P.rbc[0] = BC_PARTITION;
	}
	P.geometry = p.geometry;
	P.order = p.spatial_order;
	P.ng = P.order + 1;
	P.riemann = p.riemann;
	P.limiter = p.limiter;
	for (int i = 0; i < 3; ++i) P.dx[i] = 0;
	for (int i = 0; i < P.nd; ++i) P.dx[i] = side / (double)p.ncells[0];  // Grid.cpp:470-471 (ncells[0] for every dim)
	for (int d = 0; d < P.nd; ++d) {
		int n = d == 0 ? P.nx : (d == 1 ? P.ny : P.nz);
		bool mirror = P.lbc[d] == BC_REFLECTING || P.lbc[d] == BC_PERIODIC || P.rbc[d] == BC_REFLECTING ||
		              P.rbc[d] == BC_PERIODIC;
		if (mirror && n < P.ng + 1) return "reflecting/periodic boundaries need more cells than ghost layers";
	}
	P.tau0 = p.tau0;
	P.THI = p.THI;
	P.THII = p.THII;
	P.heating_amp = p.heating_amp;
	P.thermo_hii_switch = p.thermo_hii_switch;
	P.K1 = p.K1; P.K2 = p.K2; P.K3 = p.K3; P.K4 = p.K4;
	P.radiation_on = p.radiation_on;
	P.cooling_on = p.cooling_on;
	P.star_on = p.star_on;
	P.collisions_on = p.collisions_on;
	P.coupling = p.coupling;
	P.rt_scheme = p.rt_scheme;
	P.thermo_subcycling = p.thermo_subcycling;
	P.hydro_tma = 1;
	for (int i = 0; i < 3; ++i) P.star_pos[i] = p.star_pos[i];
	P.wind_radius = p.star_on ? p.wind_cell_radius : 0;
	// Star::initialise, Star.cpp:13-40
	for (int i = 0; i < 3; ++i) {
		double mod = (p.face_snap[i] && (p.star_pos[i] == 0)) ? 0.5 : 0;
		P.sxc[i] = p.star_pos[i] + 0.5 - mod;
	}
	if (P.nd < 3) P.sxc[2] = 0;
	if (P.nd < 2) P.sxc[1] = 0;
	Geo g(P);
	// the star's cell in this grid's (a slab's) own indices
	const int sp_loc[3] = {p.star_pos[0] - P.x0, p.star_pos[1], p.star_pos[2]};
	P.star_cell = g.within(sp_loc) ? sp_loc[0] + (long long)P.nx * (sp_loc[1] + (long long)P.ny * sp_loc[2]) : -1;

	const long long N = P.N;
	// Causal order (Grid::buildCausal, Grid.cpp:568-574) -> wind list and the
	// first non-wind cell; wind volume summed in that order (Star.cpp:42-51).
	// (a slab walks its own cells from the one nearest the star,
	// Grid::nearestCoord / buildCausal, Grid.cpp:252-258, :568-574)
	int start[3] = {(int)smin(smax(0, sp_loc[0]), P.nx - 1), (int)smin(smax(0, sp_loc[1]), P.ny - 1),
	                (int)smin(smax(0, sp_loc[2]), P.nz - 1)};
	int cur[3] = {start[0], start[1], start[2]}, nxt[3];
	std::vector<char> wind(N, 0);
	double wind_volume = 0;
	long long visited = 0;
	while (g.within(cur) && visited < N) {
		long long id = cur[0] + (long long)P.nx * (cur[1] + (long long)P.ny * cur[2]);
		double xc[3];
		int ijk[3];
		g.xc(id, xc, ijk);
		double dist2 = 0;
		for (int i = 0; i < P.nd; ++i) dist2 += ((int)xc[i] - p.star_pos[i]) * (xc[i] - p.star_pos[i]);
		if (dist2 <= P.wind_radius * P.wind_radius || id == P.star_cell) {
			wind[id] = 1;
			out.wind_cells.push_back((int)id);
			wind_volume += g.volume(xc[0]);
		} else if (out.first_nonwind_cell < 0) {
			out.first_nonwind_cell = id;
		}
		next_causal(g, cur, start, nxt);
		cur[0] = nxt[0]; cur[1] = nxt[1]; cur[2] = nxt[2];
		++visited;
	}
	if (visited != N) return "causal order does not cover the grid";
	// (a slab without the star's cell has no wind cells: no injection)
	P.mdot = (slab && wind_volume == 0) ? 0.0 : massLossRate / wind_volume;
	P.edot = 0.5 * P.mdot * windVelocity * windVelocity;

	build_tables(cv, out.tables);
	// Thermodynamics::initialise constants (Thermodynamics.cpp:33-54)
	P.z0 = 5.0e-4;
	P.T1 = 33610; P.T2 = 2180; P.T3 = 28390; P.T4 = 1780;
	P.imlc = cv.to_code(2.905e-19, 1.0, 5.0, -3.0);
	P.nmlc = cv.to_code(4.477e-20, 1.0, 5.0, -3.0);
	P.ciec_minT = 5.0e4;
	P.ciec = cv.to_code(3.485e-15, 1.0, 5.0, -3.0);
	P.cxhi_damp = 5.0e5;
	P.n0 = cv.to_code(1.0e6, 0.0, -3.0, 0.0);
	P.nmc = cv.to_code(3.981e-27, 1.0, 3.8, -3.0);
	P.fuvh_a = cv.to_code(1.9e-26, 1.0, 4.0, -2.0);
	P.fuvh_b = cv.to_code(1.00000, 0.0, 0.0, -1.0);
	P.fuvh_c = cv.to_code(6.40000, 0.0, -1.0, 0.0);
	P.irh_a = cv.to_code(7.7e-32, 1.0, 4.0, -2.0);
	P.irh_b = cv.to_code(3.0e4, 0.0, -3.0, 0.0);
	P.crh = cv.to_code(5.0e-27, 1.0, 2.0, -3.0);

	// Initial state (primitives in cgs, then code units).
	out.U.assign(7 * N, 0.0);
	out.Q.assign(7 * N, 0.0);
	out.R.assign(6 * N, 0.0);
	out.T.assign(4 * N, 0.0);
	out.Tmin.assign(N, 0.0);
	out.ds.assign(N, 0.0);
	out.shellVol.assign(N, 0.0);
	out.has_grav = grav != nullptr;
	if (grav) out.grav.assign(grav, grav + 3 * N);
	double* Q = out.Q.data();
	double* U = out.U.data();
	const double X = P.X, Rg = P.specificGasConstant;
	for (long long id = 0; id < N; ++id) {
		Q[DEN * N + id] = den[id];
		Q[PRE * N + id] = pre[id];
		Q[HII * N + id] = hii[id];
		Q[(VEL + 0) * N + id] = P.nd > 0 ? v0[id] : 0;
		Q[(VEL + 1) * N + id] = (P.nd > 1 && v1) ? v1[id] : 0;
		Q[(VEL + 2) * N + id] = (P.nd > 2 && v2) ? v2[id] : 0;
		// Thermodynamics::initialiseMinTempField (Thermodynamics.cpp:103-112), before code units
		if (p.min_temp_initial_state) {
			double mu_inv = X * (Q[HII * N + id] + 1.0) + (1.0 - X) * 0.25;
			out.Tmin[id] = (Q[PRE * N + id] / Q[DEN * N + id]) * (1.0 / mu_inv) / Rg;
		} else {
			out.Tmin[id] = 100;
		}
		// Torch::toCodeUnits (Torch.cpp:146-155)
		Q[DEN * N + id] = cv.to_code(Q[DEN * N + id], 1, -3, 0);
		Q[PRE * N + id] = cv.to_code(Q[PRE * N + id], 1, -1, -2);
		for (int d = 0; d < P.nd; ++d) Q[(VEL + d) * N + id] = cv.to_code(Q[(VEL + d) * N + id], 0, 1, -1);
		if (grav)
			for (int d = 0; d < P.nd; ++d) out.grav[d * N + id] = cv.to_code(out.grav[d * N + id], 1, -2, -2);
		// Fluid::fixPrimitives (Fluid.cpp:138-150) while U is still zero, then globalUfromQ
		double q[7], u[7];
		for (int f = 0; f < 7; ++f) q[f] = Q[f * N + id];
		q[HII] = smax(smin(q[HII], 1.0), 0.0);
		q[ADV] = smax(smin(q[ADV], 1.0), 0.0);
		q[DEN] = smax(q[DEN], P.dfloor);
		q[PRE] = smax(q[PRE], P.pfloor);
		double mu_inv = X * (q[HII] + 1.0) + (1.0 - X) * 0.25;
		double temperature = q[PRE] / (mu_inv * Rg * q[DEN]);
		if (temperature < P.tfloor) q[PRE] = mu_inv * Rg * 0.0 * P.tfloor;
		double ke = 0;
		u[DEN] = q[DEN];
		for (int d = 0; d < P.nd; ++d) {
			u[VEL + d] = q[VEL + d] * q[DEN];
			ke += 0.5 * q[DEN] * q[VEL + d] * q[VEL + d];
		}
		for (int d = P.nd; d < 3; ++d) u[VEL + d] = 0;
		u[PRE] = q[PRE] / (P.gamma - 1.0) + ke;
		u[HII] = q[HII] * q[DEN];
		u[ADV] = q[ADV] * q[DEN];
		for (int f = 0; f < 7; ++f) { Q[f * N + id] = q[f]; U[f * N + id] = u[f]; }
		// Radiation::initField: path length, shell volume, optical depths (Radiation.cpp:78-138)
		double xc[3];
		int ijk[3];
		g.xc(id, xc, ijk);
		double dd[3] = {0, 0, 0}, denom;
		for (int i = 0; i < P.nd; ++i) dd[i] = std::abs(xc[i] - P.sxc[i]);
		if (dd[2] >= dd[1] && dd[2] >= dd[0]) denom = dd[2];
		else if (dd[1] > dd[2] && dd[1] >= dd[0]) denom = dd[1];
		else denom = dd[0];
		double ds = denom != 0 ? std::sqrt(dd[0] * dd[0] * P.dx[0] * P.dx[0] + dd[1] * dd[1] * P.dx[1] * P.dx[1] +
		                                   dd[2] * dd[2] * P.dx[2] * P.dx[2]) / denom
		                       : 0.0;
		double r_sqrd = 0;
		for (int i = 0; i < P.nd; ++i) r_sqrd += (xc[i] - P.sxc[i]) * (xc[i] - P.sxc[i]) * P.dx[i] * P.dx[i];
		double shell;
		if (r_sqrd <= 100.0 * ds * ds) {
			double r = std::sqrt(r_sqrd);
			double r_min = r - 0.5 * ds, r_max = r + 0.5 * ds;
			shell = 4.0 * P.pi * (r_max * r_max * r_max - r_min * r_min * r_min) / 3.0;
		} else {
			shell = 4.0 * P.pi * r_sqrd * ds;
		}
		out.ds[id] = ds;
		out.shellVol[id] = shell;
		double nH = X * q[DEN] / P.hydrogenMass;
		out.R[R_DTAU * N + id] = (1.0 - q[HII]) * nH * P.photoIonXsec * ds;
		out.R[R_DTAU_A * N + id] = (1.0 - out.R[R_HII_A * N + id]) * nH * P.photoIonXsec * ds;
	}

	// Shell order.  Key = 2L, L the max-norm distance from the star in cell
	// units (cell and star centres sit on integers or half-integers, so 2L is
	// an integer).  An upwind neighbour with a non-zero weight always has a
	// smaller key: it is one cell nearer along the dominant axis, and a
	// neighbour left level with the cell along another axis ties only when
	// that axis is as far from the star as the dominant one, in which case its
	// weight is exactly zero (delta = 0 in calculateNearestNeighbours).  The
	// kernels skip zero-weight neighbours (their contribution is 0 * finite),
	// so each shell reads only finished inner shells.  Checked below.
	std::vector<int> shell_of(N);
	int nshell = 0;
	for (long long id = 0; id < N; ++id) {
		double xc[3];
		int ijk[3];
		g.xc(id, xc, ijk);
		double L = 0;
		for (int i = 0; i < P.nd; ++i) L = std::max(L, std::fabs(xc[i] - P.sxc[i]));
		int s = (int)std::lround(2.0 * L);
		shell_of[id] = s;
		nshell = std::max(nshell, s + 1);
	}
	for (long long id = 0; id < N; ++id) {
		double xc[3];
		int ijk[3];
		g.xc(id, xc, ijk);
		double d2 = 0;
		for (int i = 0; i < P.nd; ++i) d2 += (xc[i] - P.sxc[i]) * (xc[i] - P.sxc[i]);
		if (!(d2 > 0.95 * 0.95)) continue;
		long long nb[4];
		double w[4];
		neighbour_cells(P, ijk, xc, nb, w);
		for (int k = 0; k < 4; ++k)
			if (nb[k] >= 0 && w[k] != 0 && shell_of[nb[k]] >= shell_of[id])
				return "internal: shell order violates a sweep dependency";
	}
	// drop empty shells (odd keys are empty for a cell-centred star)
	{
		std::vector<int> remap(nshell, -1);
		std::vector<char> used(nshell, 0);
		for (long long id = 0; id < N; ++id) used[shell_of[id]] = 1;
		int k = 0;
		for (int s = 0; s < nshell; ++s)
			if (used[s]) remap[s] = k++;
		for (long long id = 0; id < N; ++id) shell_of[id] = remap[shell_of[id]];
		nshell = k;
	}
	std::vector<long long> cnt_all(nshell + 1, 0), cnt_nw(nshell + 1, 0);
	for (long long id = 0; id < N; ++id) {
		cnt_all[shell_of[id] + 1]++;
		if (!wind[id]) cnt_nw[shell_of[id] + 1]++;
	}
	for (int s = 0; s < nshell; ++s) { cnt_all[s + 1] += cnt_all[s]; cnt_nw[s + 1] += cnt_nw[s]; }
	out.off_all = cnt_all;
	out.off_nonwind = cnt_nw;
	out.sweep_all.assign(N, 0);
	out.sweep_nonwind.assign(cnt_nw[nshell], 0);
	std::vector<long long> pa(cnt_all.begin(), cnt_all.end() - 1), pn(cnt_nw.begin(), cnt_nw.end() - 1);
	for (long long id = 0; id < N; ++id) {
		int s = shell_of[id];
		out.sweep_all[pa[s]++] = (int)id;
		if (!wind[id]) out.sweep_nonwind[pn[s]++] = (int)id;
	}
	// reference values of the FP32 form: medians of the initial density and pressure
	{
		std::vector<double> d(Q + DEN * N, Q + DEN * N + N), pr(Q + PRE * N, Q + PRE * N + N);
		std::nth_element(d.begin(), d.begin() + N / 2, d.end());
		std::nth_element(pr.begin(), pr.begin() + N / 2, pr.end());
		P.f32_rho0 = d[N / 2] > 0 ? d[N / 2] : 1.0;
		P.f32_p0 = pr[N / 2] > 0 ? pr[N / 2] : 1.0;
		if (slab && slab->f32_rho0 > 0 && slab->f32_p0 > 0) {
			P.f32_rho0 = slab->f32_rho0;
			P.f32_p0 = slab->f32_p0;
		}
		P.f32_v0 = std::sqrt(P.f32_p0 / P.f32_rho0);
	}
	out.nactive = 0;
	out.active[out.nactive++] = 0;                      // HYDRO
	if (p.cooling_on) out.active[out.nactive++] = 2;    // THERMO
	if (p.radiation_on) out.active[out.nactive++] = 1;  // RAD
	return "";
}

// The arguments Torch::setUpLua passes to the Lua setup function
// initialise(x, y, z, xs, ys, zs) (src/Torch/Torch.cpp:196-228): each cell's
// centre and the star's position, cell index coordinates times the grid
// spacing in code units, converted back to cgs (Converter::fromCodeUnits,
// length index 1).  Coordinates beyond nd are 0.
std::string setup_positions(const trg_params& p, double* x, double* y, double* z, double* star) {
	if (p.nd < 1 || p.nd > 3) return "nd must be 1, 2 or 3";
	for (int i = 0; i < 3; ++i)
		if (p.ncells[i] < 1) return "ncells must be positive";
	if ((p.nd < 3 && p.ncells[2] != 1) || (p.nd < 2 && p.ncells[1] != 1)) return "ncells beyond nd must be 1";
	Converter cv;
	cv.set_rho_pressure_time(p.dscale, p.pscale, p.tscale);
	const double side = cv.to_code(p.side_length, 0, 1, 0);
	double dx[3] = {0, 0, 0};
	for (int i = 0; i < p.nd; ++i) dx[i] = side / (double)p.ncells[0];  // Grid.cpp:470-471
	// fromCodeUnits(v, 0, 1, 0) multiplies by the length unit once (Converter.cpp:35-62)
	auto from_code_length = [&](double v) { return v * cv.L; };
	double sxc[3];
	for (int i = 0; i < 3; ++i) {  // Star::initialise, Star.cpp:13-25
		const double mod = (p.face_snap[i] && (p.star_pos[i] == 0)) ? 0.5 : 0;
		sxc[i] = p.star_pos[i] + 0.5 - mod;
	}
	if (p.nd < 3) sxc[2] = 0;
	if (p.nd < 2) sxc[1] = 0;
	if (star)
		for (int i = 0; i < 3; ++i) star[i] = from_code_length(sxc[i] * dx[i]);
	const long long nx = p.ncells[0], ny = p.ncells[1], nz = p.ncells[2];
	double* out[3] = {x, y, z};
	for (long long k = 0; k < nz; ++k)
		for (long long j = 0; j < ny; ++j)
			for (long long i = 0; i < nx; ++i) {
				const long long id = i + nx * (j + ny * k);
				const long long ijk[3] = {i, j, k};
				for (int d = 0; d < 3; ++d) {
					if (!out[d]) continue;
					double xc = (double)ijk[d];  // Grid::buildCells, Grid.cpp:525-548
					if (d < p.nd) xc += 0.5;
					out[d][id] = from_code_length(xc * dx[d]);
				}
			}
	return "";
}

}  // namespace trg
