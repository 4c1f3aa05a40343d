// Plain data types shared by host set-up code and device kernels of torch_b200.
#pragma once

#include <cstdint>

namespace trg {

enum { DEN = 0, PRE = 1, HII = 2, ADV = 3, VEL = 4, NU = 7 };
enum { R_HII_A = 0, R_TAU, R_TAU_A, R_DTAU, R_DTAU_A, R_HEAT, NR };
enum { T_COL_DEN = 0, T_DCOL_DEN, T_HEAT, T_RATE, NT };

// Device layout of the radiation fields R (6 N doubles): the optical depths
// TAU, DTAU, TAU_A, DTAU_A of a cell side by side (one 32-byte sector, which
// the causal sweep reads from each inner neighbour), then HII_A and HEAT as
// plain arrays.  The thermodynamics fields T (4 N): COL_DEN, DCOL_DEN of a
// cell side by side, then HEAT and RATE.  The C ABI exchanges both as field
// after field ([6][N], [4][N]).
#ifdef __CUDACC__
#define TRG_HD __host__ __device__
#else
#define TRG_HD
#endif
TRG_HD inline constexpr int r_quad_slot(int f) { return f == R_TAU ? 0 : (f == R_DTAU ? 1 : (f == R_TAU_A ? 2 : 3)); }
TRG_HD inline constexpr long long r_index(long long N, int f, long long id) {
	return f == R_HII_A ? 4 * N + id : (f == R_HEAT ? 5 * N + id : id * 4 + r_quad_slot(f));
}
TRG_HD inline constexpr long long t_index(long long N, int f, long long id) {
	return f <= T_DCOL_DEN ? id * 2 + f : (long long)f * N + id;
}
// heating / cooling diagnostics (HID, src/Torch/Common.hpp:32-34)
enum { H_IMLC = 0, H_NMLC, H_RHII, H_CEHI, H_CIEC, H_NMC, H_EUVH, H_FUVH, H_IRH, H_CRH, H_TOT, NH };
enum { G_CART = 0, G_CYL = 1, G_SPH = 2 };
enum { BC_FREE = 0, BC_REFLECTING = 1, BC_OUTFLOW = 2, BC_INFLOW = 3, BC_PERIODIC = 4 };
// an x face that borders another slab of an x-slab decomposition
// (Condition::PARTITION, Grid.cpp:804-833): its ghost layers come from the
// neighbour's halo, held in State::halo_recv
constexpr int BC_PARTITION = 5;
enum { CP_TTI = 0, CP_NEQ = 1, CP_OFF = 2 };
enum { RS_HLLC = 0, RS_ROTATED = 1, RS_HLL = 2 };

// Device error word bits (host maps them to TRG_ERR_*).
enum : unsigned {
	ERRB_NAN = 1u, ERRB_PICARD = 2u, ERRB_DT = 4u, ERRB_FLUX = 8u, ERRB_TC = 16u, ERRB_SUBCYCLE = 32u,
	ERRB_ASYNC = 64u,  // an asynchronous (TMA) copy did not complete within its wait limit
	ERRB_SLAB = 128u,  // a slab's sweep met a partition-face neighbour before any boundary layer was exchanged
};

// Work queue of the thermal sub-cycles: control words (State::thq_ctl) and
// limits.  Bins hold counts of bit length b (2^b .. 2^(b+1) - 1 sub-cycles).
constexpr int THQ_BINS = 32;
enum { THQ_COUNT = 0, THQ_HEAD = 1, THQ_BIN = 2, THQ_CURSOR = THQ_BIN + THQ_BINS, THQ_CTL = THQ_CURSOR + THQ_BINS };
constexpr int THQ_MAX_SUBCYCLES = 1 << 26;

// Rows of State::sw_rad beyond the six per-cell inputs, and the largest
// candidate list the learned start serves in one sweep.
constexpr int SW_TAU_A = 6, SW_LSTART = 7, SW_RAD_ROWS = 8;
constexpr int LCAND_MAX = 1 << 21;
// persistent grid of the learned-start inference (4 CTAs per SM of a B200)
constexpr int INFER_CTAS = 148 * 4;

// Planes per CTA of the FP32 form's fallback flag pass (k_fb_flags).
constexpr int FB_ZCHUNK = 16;

// Cubic spline table (SplineData, src/Integrators/SplineData.cpp) built on the host.
struct Spline {
	int n, log_mode;
	double min_slope, max_slope;
	double x[32], y[32], y2[32];
};

struct Tables {
	Spline rad_recomb, rad_cool, th_cxhi, th_recomb;
};

// Code-unit parameters of one run (the reference's Constants, TorchParameters
// after initialise(), Star, Thermodynamics constants).
struct BatchTable;

struct Params {
	int nd, nx, ny, nz;
	long long N;
	// x-slab decomposition: global x index of this grid's first cell (0 for a
	// whole grid); cell centres and the geometry use global positions
	int x0;
	int geometry, order, ng;
	int lbc[3], rbc[3];
	int riemann, limiter;
	double dx[3];
	double gamma, X;
	double hydrogenMass, specificGasConstant, boltzmannConst, rydbergEnergy, dustXsec, pi;
	double voronov_A, voronov_X, voronov_K, voronov_P, voronov_DE;
	double dt_max, dfloor, pfloor, tfloor;
	double photoIonXsec, photonEnergy, photonRate;
	double tau0, THI, THII, heating_amp, thermo_hii_switch;
	double K1, K2, K3, K4;
	int radiation_on, cooling_on, star_on, collisions_on, coupling, thermo_subcycling;
	int rt_scheme;  // 0 implicit, 1 implicit2, 2 explicit (Radiation.cpp:48-53)
	int star_pos[3];
	int wind_radius;     // Star::windCellRadius when the star is on, else 0
	long long star_cell; // flat index of the star cell or -1
	double sxc[3];       // Star::xc
	double mdot, edot;
	// thermodynamics constants (Thermodynamics::initialise, Thermodynamics.cpp:24-57)
	double z0, T1, T2, T3, T4, imlc, nmlc, ciec_minT, ciec, cxhi_damp, n0, nmc;
	double fuvh_a, fuvh_b, fuvh_c, irh_a, irh_b, crh;
	// FP32 form: the hydro state is stored divided by these reference values
	// (density rho0, pressure / energy density p0, velocity v0 = sqrt(p0/rho0)),
	// so that FP32 holds it far from its range limits whatever the code units.
	double f32_rho0, f32_p0, f32_v0;
	// diagnostic counters (State::stats) are updated only when this is set
	int stats_on;
	// FP32 hydro pass on the FP64 state: stage planes by TMA where possible
	// (else per-cell cp.async)
	int hydro_tma;
	// batched launch over many grids (null for one grid): kernels take each
	// grid's Params and State from this table
	const BatchTable* batch;
};

// Device pointers of one context (FP64 state).
struct State {
	double* U;      // [7][N]
	double* Q;      // [7][N]
	double* U1;     // [7][N] scratch (RK2 intermediate state)
	double* UDOT;   // [7][N] (component-phase interface only)
	double* R;      // [6][N]
	double* T;      // [4][N]
	double* Tmin;   // [N]
	double* ds;     // [N]
	double* shellVol;
	double* grav;   // [3][N] or nullptr
	// x-slab decomposition (caller-owned device buffers, null for a whole
	// grid): the two boundary x layers of each partition face packed for the
	// neighbour, and the neighbours' layers received, both
	// [side 2][layer 2][field 7][ny * nz] (layer 0 next to the face); doubles
	// (primitives of the FP64 form) or floats (the hydro-only FP32 state)
	void* halo_send;
	const void* halo_recv;
	// x-slab decomposition with a star: the star-side neighbour's boundary x
	// layer, received before each causal sweep, [side 2][ny * nz][4] doubles
	// (the four optical depths in the R quad order, or COL_DEN, DCOL_DEN and
	// two unused), read where an upwind neighbour lies across a partition
	// face; null for a whole grid
	const double* sweep_recv;
	double* F[3];   // face fluxes per dimension [7][faces]
	long long nfaces[3];
	const Tables* tables;
	unsigned* err;
	// scalars: [0] dt, [1] time, [2..4] per-component dt minima (as uint64 bits)
	double* scal;
	double* dt_hist;
	// diagnostic counters, TRG_STAT_* indices of the C ABI header
	unsigned long long* stats;
	// heating / cooling diagnostics [NH][N], kept up to date during the step
	// when non-null (trg_heating_enable)
	double* H;
	// learned starting iterate: the network's inference image (null = plain
	// solve); when set, lstart is non-null (the predictions live in sw_rad
	// row SW_LSTART) and lcand lists the candidate sweep positions
	const unsigned char* mlp_img;
	double* lstart;
	int* lcand;
	unsigned* lcand_n;
	// FP32 form, radiation-hydro runs: cells whose hydro stencil spans a
	// pressure contrast FP32 cannot difference are updated in FP64 instead
	// (flag per cell, compacted list and its length)
	unsigned char* fb_flag;
	int* fb_list;
	unsigned* fb_count;
	// training-set recording by the plain solve: records of 8 floats
	float* harvest;
	long long harvest_cap;
	unsigned long long* harvest_n;
	// Causal sweeps of a single grid: each cell's own inputs in sweep order
	// (index = the cell's position in the sweep list), so that the
	// latency-bound shell kernels read them contiguously; a parallel pass
	// refreshes the per-step ones before each sweep.
	//   sw_rad [8][sw_rad_n] over the non-wind sweep list: n_H, the case-B
	//          recombination rate, the collisional ionisation rate, x_HII
	//          (per sweep), path length ds, shell volume (fixed), TAU_A of the
	//          last sweep, the learned starting fraction of the coming sweep
	//          (NaN: none);
	//   sw_col [2][sw_col_n] over the sweep list of all cells: the cell's own
	//          column density ds rho / m_H (per sweep), ds (fixed).
	// Thermal sub-cycle work queue (null: every cell runs its sub-cycles in
	// place): cells with at least thq_min sub-cycles, their bins, the cells
	// laid out bin by bin, and the control words (THQ_*)
	int* thq;
	unsigned char* thq_binof;
	int* thq_sorted;
	unsigned* thq_ctl;
	int thq_min;
	double* sw_rad;
	long long sw_rad_n;
	double* sw_col;
	long long sw_col_n;
	// global FP64 mass and energy sums (null: off): the time-step reduction
	// also leaves per-block double-double partials of sum(rho V) and sum(E V)
	// here, 4 doubles per 256-cell block (mass hi, lo, energy hi, lo)
	double* cons_part;
};

// Many independent grids advanced by one launch per stage.  Cell and face
// ranges of the grids are laid end to end, each padded to a whole number of
// 256-thread blocks, so that a block belongs to one grid (found by binary
// search in the offsets); shell and wind lists hold (grid << BATCH_CELL_BITS) |
// cell entries.
constexpr int BATCH_CELL_BITS = 22;
constexpr int BATCH_CELL_MASK = (1 << BATCH_CELL_BITS) - 1;
constexpr int BATCH_MAX_GRIDS = 1 << (31 - BATCH_CELL_BITS);
struct BatchTable {
	int G;
	const Params* P;             // per grid (their batch field is null)
	const State* S;
	const long long* cell_off;   // [G + 1]
	const long long* face_off[3];  // [G + 1] per dimension
	const long long* first_cell;   // [G] first non-wind cell in causal order
	// FP32 form (2-D grids): the CTA tiles of all grids' FP32 hydro pass
	const struct BatchTile* tiles;
	int ntiles;
};
struct BatchTile {
	int g, tx, ty, pad;  // grid, tile index along x and y
};

}  // namespace trg
