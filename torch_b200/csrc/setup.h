// Host-side set-up of a run: code units, tables, initial state, sweep order.
#pragma once
#include <string>
#include <vector>

#include "../../include/torch_b200.h"
#include "trg_types.h"

namespace trg {

struct HostSetup {
	Params P;
	Tables tables;
	std::vector<double> U, Q, R, T, Tmin, ds, shellVol, grav;  // field-major [f][N]
	bool has_grav = false;
	// Sweep order: cells grouped into shells of the max-norm distance from
	// the star; a shell only reads cells of inner shells.
	std::vector<int> sweep_all, sweep_nonwind;          // cell ids, shell by shell
	std::vector<long long> off_all, off_nonwind;        // shell offsets (size nshell+1)
	std::vector<int> wind_cells;
	long long first_nonwind_cell = -1;                   // first non-wind cell in causal order
	double dt_max = 0, tmax = 0;
	int nactive = 1;
	int active[3] = {0, 0, 0};
};

// One slab of an x-slab decomposition: global x of its first cell, its
// width, and the FP32 form's reference density and pressure (the whole
// grid's, so that every slab scales its state alike; 0: this slab's medians).
struct SlabSpec {
	int x0 = 0, nx = 0;
	double f32_rho0 = 0, f32_p0 = 0;
};

// Returns an empty string on success, else the reason for refusing the input.
// With `slab`, p describes the whole grid and the arrays hold the slab's cells.
std::string host_setup(const trg_params& p, const double* den, const double* pre, const double* hii, const double* v0,
                       const double* v1, const double* v2, const double* grav, HostSetup& out,
                       const SlabSpec* slab = nullptr);

// Cell and star positions (cgs) as Torch::setUpLua passes them to the Lua
// setup function; empty string on success.
std::string setup_positions(const trg_params& p, double* x, double* y, double* z, double* star);

}  // namespace trg
