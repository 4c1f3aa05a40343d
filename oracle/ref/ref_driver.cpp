/*
 * Step-capped driver around the UNMODIFIED reference TORCH sources.
 *
 * Test infrastructure only (the CPU oracle): it is compiled together with the
 * reference's own src/*.cpp by oracle/ref/Makefile into oracle/_ref/torch_ref,
 * and is never linked into the product library.
 *
 * What it runs, in the reference's own order:
 *   - parseParameters()            src/main.cpp:126-208 (Lua config via Selene)
 *   - Torch::initialise()          src/Torch/Torch.cpp:29-144 (initial conditions
 *                                  from the DataReader text format when --ic is given)
 *   - the Torch::run() prologue    src/Torch/Torch.cpp:245-264 without the
 *                                  snapshot I/O: globalQfromU, fixPrimitives,
 *                                  active component list, fillHeatingArrays
 *   - N x Torch::fullStep(dt_max)  src/Torch/Torch.cpp:389-418, advancing
 *                                  Grid::currentTime like run() does (:285-286).
 *                                  The checkpoint scheduler is not run: every
 *                                  step is offered dt_next_checkpoint = dt_max.
 *
 * With --setup-dump=FILE (and --setup) it also writes the raw values the Lua
 * setup function returned for every cell (see below).
 *
 * Output: a binary state dump (format "TRGS", see write_state below) of the
 * interior cells in the reference's flat index order (x fastest); with
 * --print2d=DIR also the reference's own checkpoint files of the final state
 * (DataPrinter::print2D and ::printHeating after fillHeatingArrays).
 *
 * Each invocation is one fresh process, because the reference keeps
 * function-local statics (Torch.cpp:305, Radiation.cpp:79, Radiation.cpp:300).
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#define private public
#define protected public
#include "Torch/Torch.hpp"
#include "Fluid/Fluid.hpp"
#include "Fluid/Grid.hpp"
#include "Fluid/GridCell.hpp"
#include "Fluid/Star.hpp"
#include "Integrators/Radiation.hpp"
#include "Integrators/Thermodynamics.hpp"
#include "MPI/MPI_Wrapper.hpp"
#include "selene/include/selene.h"
#undef private
#undef protected

/* Defined in the reference's src/main.cpp, compiled with -Dmain=torch_reference_main. */
void parseParameters(const std::string& filename, TorchParameters& p);

static const char* arg_value(const char* arg, const char* key) {
	size_t n = strlen(key);
	return strncmp(arg, key, n) == 0 ? arg + n : nullptr;
}

/*
 * TRGS v1 layout (little endian):
 *   char magic[4] = "TRGS"; int32 version = 1;
 *   int32 nx, ny, nz, nd, nsteps, flags;
 *   double time, dx;
 *   double U[7][N], Q[7][N], R[6][N], T[4][N], T_min[N]   (N = nx*ny*nz, x fastest)
 *   double dt[nsteps]
 */
static void write_state(const std::string& path, Torch& torch, const std::vector<double>& dts) {
	Grid& grid = torch.fluid.getGrid();
	const int nx = grid.ncells[0], ny = grid.ncells[1], nz = grid.ncells[2];
	const size_t N = (size_t)nx * ny * nz;
	FILE* f = fopen(path.c_str(), "wb");
	if (!f)
		throw std::runtime_error("cannot open " + path);
	int32_t hdr[8] = {0, 1, nx, ny, nz, torch.consts->nd, (int32_t)dts.size(), 0};
	memcpy(hdr, "TRGS", 4);
	fwrite(hdr, sizeof(int32_t), 8, f);
	double t = grid.currentTime, dx = grid.dx[0];
	fwrite(&t, sizeof(double), 1, f);
	fwrite(&dx, sizeof(double), 1, f);
	std::vector<double> buf(N);
	typedef double (*Getter)(GridCell&, int);
	auto dump = [&](Getter getter, int count) {
		for (int c = 0; c < count; ++c) {
			for (size_t i = 0; i < N; ++i)
				buf[i] = getter(grid.getCell((int)i), c);
			fwrite(buf.data(), sizeof(double), N, f);
		}
	};
	dump([](GridCell& cell, int c) { return cell.U[c]; }, UID::N);
	dump([](GridCell& cell, int c) { return cell.Q[c]; }, UID::N);
	dump([](GridCell& cell, int c) { return cell.R[c]; }, RID::N);
	dump([](GridCell& cell, int c) { return cell.T[c]; }, TID::N);
	dump([](GridCell& cell, int) { return cell.T_min; }, 1);
	if (!dts.empty())
		fwrite(dts.data(), sizeof(double), dts.size(), f);
	fclose(f);
}

int main(int argc, char** argv) {
	std::string params, setup, ic, out, out0, print2d, setup_dump;
	long steps = 0;
	int print_params = 0;
	for (int i = 1; i < argc; ++i) {
		const char* v;
		if ((v = arg_value(argv[i], "--params="))) params = v;
		else if ((v = arg_value(argv[i], "--setup="))) setup = v;
		else if ((v = arg_value(argv[i], "--ic="))) ic = v;
		else if ((v = arg_value(argv[i], "--steps="))) steps = atol(v);
		else if ((v = arg_value(argv[i], "--out="))) out = v;
		else if ((v = arg_value(argv[i], "--out0="))) out0 = v;
		else if ((v = arg_value(argv[i], "--print2d="))) print2d = v;
		else if ((v = arg_value(argv[i], "--setup-dump="))) setup_dump = v;
		else if (strcmp(argv[i], "--print-params") == 0) print_params = 1;
		else {
			fprintf(stderr, "usage: torch_ref --params=P.lua [--setup=S.lua] [--ic=IC_000.txt] "
			                "--steps=N --out=final.bin [--out0=initial.bin] [--print2d=DIR] [--setup-dump=FILE]\n");
			return 2;
		}
	}
	if (params.empty() || (!print_params && setup.empty() && ic.empty())) {
		fprintf(stderr, "torch_ref: --params and one of --setup/--ic are required\n");
		return 2;
	}
	try {
		MPIW::Instance();
		TorchParameters p;
		parseParameters(params, p);
		p.setupFile = setup;
		if (!ic.empty())
			p.initialConditions = ic;
		if (print_params) {
			/* The values the reference's own Lua front end produced. */
			printf("dscale %.17g\npscale %.17g\ntscale %.17g\nspatial_order %d\ntemporal_order %d\n"
			       "tmax %.17g\nradiation_on %d\ncooling_on %d\nnd %d\nncells %d %d %d\n"
			       "side_length %.17g\ngeometry %s\nleft_bc %s %s %s\nright_bc %s %s %s\n"
			       "gamma %.17g\ndfloor %.17g\npfloor %.17g\ntfloor %.17g\nriemann %s\nlimiter %s\n"
			       "K %.17g %.17g %.17g %.17g\nphotoion_xsec %.17g\nalphaB %.17g\ntau0 %.17g\n"
			       "minX %.17g\nTHI %.17g\nTHII %.17g\nmass_frac_h %.17g\ncollisions_on %d\n"
			       "coupling %s\nrt_scheme %s\nthermo_hii_switch %.17g\nheating_amp %.17g\n"
			       "thermo_subcycling %d\nmin_temp_initial_state %d\nstar_on %d\nstar_pos %d %d %d\n"
			       "face_snap %d %d %d\nphoton_energy %.17g\nphoton_rate %.17g\nwind_cell_radius %d\n"
			       "mass_loss_rate %.17g\nwind_velocity %.17g\nwind_temperature %.17g\n",
			       p.dscale, p.pscale, p.tscale, p.spatialOrder, p.temporalOrder, p.tmax,
			       (int)p.radiation_on, (int)p.cooling_on, p.nd, p.ncells[0], p.ncells[1], p.ncells[2],
			       p.sideLength, p.geometry.c_str(), p.leftBC[0].c_str(), p.leftBC[1].c_str(),
			       p.leftBC[2].c_str(), p.rightBC[0].c_str(), p.rightBC[1].c_str(), p.rightBC[2].c_str(),
			       p.heatCapacityRatio, p.dfloor, p.pfloor, p.tfloor, p.riemannSolver.c_str(),
			       p.slopeLimiter.c_str(), p.K1, p.K2, p.K3, p.K4, p.photoIonCrossSection, p.alphaB,
			       p.tau0, p.minX, p.THI, p.THII, p.massFractionH, (int)p.collisions_on,
			       p.rt_coupling.c_str(), p.rt_scheme.c_str(), p.thermoHII_Switch,
			       p.heatingAmplification, (int)p.thermoSubcycling, (int)p.minTempInitialState,
			       (int)p.star_on, p.star_position[0], p.star_position[1], p.star_position[2],
			       (int)p.faceSnap[0], (int)p.faceSnap[1], (int)p.faceSnap[2], p.photonEnergy,
			       p.photonRate, p.windCellRadius, p.massLossRate, p.windVelocity, p.windTemperature);
			return 0;
		}

		Torch torch;
		torch.initialise(p);
		if (!setup_dump.empty() && !setup.empty()) {
			/* The raw values of the Lua setup function (cgs, before toCodeUnits),
			 * evaluated with the arguments Torch::setUpLua passes
			 * (src/Torch/Torch.cpp:196-228): [9][N] doubles, x fastest. */
			Grid& grid = torch.fluid.getGrid();
			const size_t N = (size_t)grid.ncells[0] * grid.ncells[1] * grid.ncells[2];
			std::vector<double> vals(9 * N);
			sel::State luaState{true};
			if (!luaState.Load(setup))
				throw std::runtime_error("cannot load " + setup);
			for (size_t id = 0; id < N; ++id) {
				GridCell& cell = grid.getCell((int)id);
				std::array<double, 3> xc, xs;
				for (int i = 0; i < 3; ++i) {
					xc[i] = torch.consts->converter.fromCodeUnits(cell.xc[i] * grid.dx[i], 0, 1, 0);
					xs[i] = torch.consts->converter.fromCodeUnits(torch.fluid.getStar().xc[i] * grid.dx[i], 0, 1, 0);
				}
				double r[9];
				sel::tie(r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7], r[8]) =
					luaState["initialise"](xc[0], xc[1], xc[2], xs[0], xs[1], xs[2]);
				for (int k = 0; k < 9; ++k) vals[k * N + id] = r[k];
			}
			FILE* f = fopen(setup_dump.c_str(), "wb");
			if (!f || fwrite(vals.data(), sizeof(double), vals.size(), f) != vals.size())
				throw std::runtime_error("cannot write " + setup_dump);
			fclose(f);
		}

		/* Torch::run() prologue, src/Torch/Torch.cpp:245-264, minus snapshot I/O. */
		torch.fluid.globalQfromU();
		torch.fluid.fixPrimitives();
		torch.activeComponents.push_back(ComponentID::HYDRO);
		if (torch.cooling_on)
			torch.activeComponents.push_back(ComponentID::THERMO);
		if (torch.radiation_on)
			torch.activeComponents.push_back(ComponentID::RAD);
		torch.thermodynamics.fillHeatingArrays(torch.fluid);

		std::vector<double> dts;
		if (!out0.empty())
			write_state(out0, torch, dts);
		for (long s = 0; s < steps; ++s) {
			double dt = torch.fullStep(torch.dt_max);
			torch.fluid.getGrid().deltatime = dt;
			torch.fluid.getGrid().currentTime += dt;
			dts.push_back(dt);
		}
		if (!out.empty())
			write_state(out, torch, dts);
		if (!print2d.empty()) {
			/* What Torch::run writes at a checkpoint (src/Torch/Torch.cpp:270-281):
			 * fillHeatingArrays, then DataPrinter::printHeating and ::print2D,
			 * here into <print2d>/heating_final.txt.gz and data2D_final.txt.gz. */
			torch.thermodynamics.fillHeatingArrays(torch.fluid);
			torch.inputOutput.dir2D = print2d;
			torch.inputOutput.printing_on = true;
			std::remove((print2d + "/heating_final.txt.gz").c_str());
			std::remove((print2d + "/data2D_final.txt.gz").c_str());
			torch.inputOutput.printHeating("final", torch.fluid.getGrid().currentTime, torch.fluid.getGrid());
			torch.inputOutput.print2D("final", torch.fluid.getGrid().currentTime, torch.fluid.getGrid());
		}
	}
	catch (std::exception& e) {
		fprintf(stderr, "torch_ref: reference threw: %s\n", e.what());
		return 3;
	}
	return 0;
}
