/*
 * CPU oracle: a sequential, plain-C restatement of the reference TORCH
 * operator-split timestep (src/Torch/Torch.cpp:304-443 and everything it
 * calls).  TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load it as the checker; the product library
 * never links it.
 *
 * Parity is pinned against the reference itself: oracle/ref builds the
 * unmodified reference sources into oracle/_ref/torch_ref, and the CPU tests
 * compare this restatement with that binary bit for bit (FP64, no FP
 * contraction on either side).
 *
 * Layout: structure-of-arrays over the interior cells, flat index
 * i + nx*(j + ny*k) (the reference's Grid::flatIndex, Grid.cpp:153-155).
 * Field order U/Q: DEN, PRE(=E in U), HII, ADV, VEL0, VEL1, VEL2
 * (src/Torch/Common.hpp:23-34).
 */
#ifndef TORCH_ORACLE_H
#define TORCH_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Raw run parameters as read from the Lua config (cgs where the reference
 * keeps cgs), i.e. TorchParameters before TorchParameters::initialise
 * (src/Torch/Parameters.hpp:25-97).  Enum values follow src/Torch/Common.hpp. */
typedef struct orc_params {
	double dscale, pscale, tscale;
	int spatial_order, temporal_order;
	double tmax;
	int radiation_on, cooling_on;
	int nd;
	int ncells[3];
	double side_length;
	int geometry;               /* 0 cartesian, 1 cylindrical, 2 spherical */
	int left_bc[3], right_bc[3];/* 0 free, 1 reflecting, 2 outflow, 3 inflow, 4 periodic */
	double gamma, dfloor, tfloor;
	int riemann;                /* 0 HLLC, 1 RotatedHLLC, 2 HLL */
	int limiter;                /* 0 monotonised_central, 1 superbee, 2 minmod, 3 maxmod, 4 leer, 5 ospre, 6 albada */
	double K1, K2, K3, K4;
	double photoion_xsec, alphaB, tau0, minX, THI, THII, mass_frac_h;
	int rt_scheme;              /* 0 implicit, 1 implicit2, 2 explicit */
	int collisions_on;
	int coupling;               /* 0 tti, 1 neq, 2 off */
	double heating_amp, thermo_hii_switch;
	int thermo_subcycling, min_temp_initial_state;
	int star_on;
	int star_pos[3];
	int face_snap[3];
	double photon_energy, photon_rate, mass_loss_rate, wind_velocity, wind_temperature;
	int wind_cell_radius;
} orc_params;

typedef struct orc_ctx orc_ctx;

/* Torch::initialise (Torch.cpp:29-144) + the Torch::run prologue (:245-264).
 * den/pre/hii/v0..v2 are the initial primitives in cgs over the interior
 * cells (the DataReader/Lua setup values); v1/v2/grav may be NULL (zero).
 * grav is [3][N] or NULL.  Returns NULL and fills err on failure. */
orc_ctx* orc_create(const orc_params* p, const double* den, const double* pre,
                    const double* hii, const double* v0, const double* v1,
                    const double* v2, const double* grav, char* err, int errlen);

/* One Torch::fullStep(dt_next_checkpoint) (Torch.cpp:389-418) plus the
 * currentTime advance of Torch::run (:285-286).  Returns 0 or an error code;
 * *dt_out receives the step size. */
int orc_full_step(orc_ctx* c, double dt_next_checkpoint, double* dt_out);

/* Copies U[7][N], Q[7][N], R[6][N], T[4][N], Tmin[N] (any may be NULL). */
void orc_get_state(const orc_ctx* c, double* U, double* Q, double* R, double* T, double* Tmin);
double orc_time(const orc_ctx* c);
double orc_dt_max(const orc_ctx* c);
long orc_ncells(const orc_ctx* c);
const char* orc_last_error(const orc_ctx* c);
void orc_destroy(orc_ctx* c);
/* Test hook of the host-libm build: moves a fixed, input-determined fraction
 * of the step's exp/log/log10/pow results by one ulp (0: off). */
void orc_set_libm_noise(double fraction);

/* Order in which the reference visits interior cells in its causal sweeps
 * (Grid::buildCausal, Grid.cpp:568-574): writes up to cap flat indices and
 * returns the list length. */
long orc_causal_order(const orc_ctx* c, int* out, long cap);

/* Cell volumes (Grid::computeCellVolume, Grid.cpp:876-905) in code units:
 * writes up to cap values in flat-index order and returns the cell count. */
long orc_cell_volumes(const orc_ctx* c, double* out, long cap);

#ifdef __cplusplus
}
#endif
#endif
