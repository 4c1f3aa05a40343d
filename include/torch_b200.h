/*
 * torch_b200: B200 (sm_100a) implementation of the TORCH operator-split
 * radiation-hydrodynamics timestep, behind a plain C ABI.
 *
 * The entry points replace the Fluid/Integrators step of the reference:
 *
 *   trg_create         Torch::initialise (src/Torch/Torch.cpp:29-144) followed by
 *                      the Torch::run prologue (src/Torch/Torch.cpp:245-264).
 *                      Input: the raw Lua parameters (TorchParameters,
 *                      src/Torch/Parameters.hpp:25-97, before
 *                      TorchParameters::initialise) and the initial primitive
 *                      fields in cgs, as DataReader::readGrid
 *                      (src/IO/DataReader.cpp:70-125) or the Lua setup callback
 *                      (src/Torch/Torch.cpp:192-228) would produce them.
 *   trg_full_step      Torch::fullStep(dt_next_checkpoint)
 *                      (src/Torch/Torch.cpp:389-418) plus the currentTime advance
 *                      of Torch::run (src/Torch/Torch.cpp:285-286).
 *   trg_run_steps      nsteps consecutive trg_full_step calls enqueued without a
 *                      host round trip between steps.
 *   trg_component      one phase of one Integrator (src/Integrators/Integrator.hpp:26-29:
 *                      preTimeStepCalculations / calculateTimeStep / integrate /
 *                      updateSourceTerms) or of the Fluid bookkeeping
 *                      (Fluid::globalQfromU+fixPrimitives, advSolution+fixSolution,
 *                      src/Fluid/Fluid.cpp:80-170), for callers that drive the
 *                      operator split themselves.
 *   trg_get_state /    read or replace the cell state (code units, SoA, flat
 *   trg_set_conserved  index i + nx*(j + ny*k), Grid::flatIndex, src/Fluid/Grid.cpp:153-155).
 *   trg_last_error     the text of the last failure (the reference throws
 *                      std::runtime_error with a message, src/main.cpp:101-105).
 *
 * Conventions: every call returns 0 on success or a TRG_ERR_* code; the
 * context owns all device memory; one context per host thread, all work on the
 * context's own CUDA stream.  Field order for U and Q is DEN, PRE (total energy
 * E in U), HII, ADV, VEL0, VEL1, VEL2 (src/Torch/Common.hpp:23-34); R is
 * HII_A, TAU, TAU_A, DTAU, DTAU_A, HEAT; T is COL_DEN, DCOL_DEN, HEAT, RATE.
 */
#ifndef TORCH_B200_H
#define TORCH_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TRG_OK 0
#define TRG_ERR_ARG 1          /* invalid argument or unsupported parameter */
#define TRG_ERR_CUDA 2         /* a CUDA runtime call failed */
#define TRG_ERR_NAN 3          /* checkValues / fixSolution found an invalid state */
#define TRG_ERR_PICARD 4       /* implicit ionisation solve did not converge */
#define TRG_ERR_DT 5           /* invalid radiation time step */
#define TRG_ERR_FLUX 6         /* Riemann solver produced a NaN HII flux */
#define TRG_ERR_OOM 7          /* device allocation failed */
#define TRG_ERR_TC 8           /* a tensor-core (tcgen05) wait expired */
#define TRG_ERR_SUBCYCLE 9     /* a cell needs more thermal sub-cycles than the work queue runs */

#define TRG_PRECISION_FP64 0   /* every kernel in FP64, reference operation order, no FMA */
#define TRG_PRECISION_FP32 1   /* hydro in FP32 (compensated E - KE), FP64 for ionisation, dt, sums */

/* Raw run parameters: the values of the Lua Parameters table (cgs where the
 * reference keeps cgs).  Enum values follow src/Torch/Common.hpp. */
typedef struct trg_params {
	double dscale, pscale, tscale;
	int spatial_order, temporal_order;
	double tmax;
	int radiation_on, cooling_on;
	int nd;
	int ncells[3];
	double side_length;
	int geometry;                /* 0 cartesian, 1 cylindrical, 2 spherical */
	int left_bc[3], right_bc[3]; /* 0 free, 1 reflecting, 2 outflow, 3 inflow, 4 periodic */
	double gamma, dfloor, tfloor;
	int riemann;                 /* 0 HLLC, 1 RotatedHLLC, 2 HLL */
	int limiter;                 /* 0 monotonised_central, 1 superbee, 2 minmod, 3 maxmod, 4 leer, 5 ospre, 6 albada */
	double K1, K2, K3, K4;
	double photoion_xsec, alphaB, tau0, minX, THI, THII, mass_frac_h;
	int rt_scheme;               /* 0 implicit, 1 implicit2, 2 explicit (Radiation.cpp:48-53) */
	int collisions_on;
	int coupling;                /* 0 tti, 1 neq, 2 off */
	double heating_amp, thermo_hii_switch;
	int thermo_subcycling, min_temp_initial_state;
	int star_on;
	int star_pos[3];
	int face_snap[3];
	double photon_energy, photon_rate, mass_loss_rate, wind_velocity, wind_temperature;
	int wind_cell_radius;
	int precision;               /* TRG_PRECISION_* */
	int device;                  /* CUDA device ordinal */
} trg_params;

typedef struct trg_ctx trg_ctx;

/* Component ids and phases for trg_component (ComponentID, src/Torch/Torch.hpp:29). */
#define TRG_COMP_HYDRO 0
#define TRG_COMP_RAD 1
#define TRG_COMP_THERMO 2
#define TRG_COMP_FLUID 3
#define TRG_PHASE_PRE 0         /* Integrator::preTimeStepCalculations */
#define TRG_PHASE_DT 1          /* Integrator::calculateTimeStep (returns dt in *out) */
#define TRG_PHASE_INTEGRATE 2   /* Integrator::integrate(dt) */
#define TRG_PHASE_SOURCES 3     /* Integrator::updateSourceTerms(dt) (accumulates UDOT) */
#define TRG_PHASE_Q_FROM_U 4    /* FLUID: globalQfromU + fixPrimitives */
#define TRG_PHASE_ADVANCE 5     /* FLUID: advSolution(dt) + fixSolution */

/* den..v2: initial primitives in cgs over the interior cells (N each); v1, v2
 * and grav ([3][N], cgs) may be NULL for zero.  ncells/side_length describe
 * the grid (for a text snapshot, side_length = dx * ncells[0] as
 * DataReader::readDataParameters derives it). */
int trg_create(const trg_params* p, const double* den, const double* pre, const double* hii,
               const double* v0, const double* v1, const double* v2, const double* grav,
               trg_ctx** out);
/* The arguments Torch::setUpLua (src/Torch/Torch.cpp:196-228) passes to the
 * Lua setup function initialise(x, y, z, xs, ys, zs) of a run with
 * parameters p: every cell's centre (x, y, z: N each, cgs, flat index
 * i + nx*(j + ny*k), any may be NULL) and the star's position (star_xyz[3],
 * may be NULL), formed as the reference forms them (cell index coordinates
 * times the code-unit grid spacing, converted back to cgs).  Host only: needs
 * no GPU.  The setup function's nine results per cell become trg_create's
 * den, pre, hii, v0, v1, v2 and grav. */
int trg_setup_positions(const trg_params* p, double* x, double* y, double* z, double* star_xyz);
int trg_full_step(trg_ctx* c, double dt_next_checkpoint, double* dt_taken);
int trg_run_steps(trg_ctx* c, int nsteps, double dt_next_checkpoint, double* dts_out);
int trg_component(trg_ctx* c, int comp, int phase, double dt, double* out);
/* Any pointer may be NULL.  U, Q: [7][N]; R: [6][N]; T: [4][N]; Tmin: [N]. */
int trg_get_state(trg_ctx* c, double* U, double* Q, double* R, double* T, double* Tmin);
int trg_set_conserved(trg_ctx* c, const double* U);
int trg_synchronize(trg_ctx* c);
double trg_time(const trg_ctx* c);
double trg_dt_max(const trg_ctx* c);
long trg_ncells(const trg_ctx* c);
/* Kernel launches issued by this context since creation (for accounting). */
long long trg_kernel_launches(const trg_ctx* c);

/* Measurement hooks (no counterpart in the reference, which has no timers):
 *   trg_enqueue_steps  like trg_run_steps but returns right after enqueuing,
 *                      without waiting or checking the device error word
 *                      (call trg_synchronize afterwards);
 *   trg_stream         the context's cudaStream_t, for events recorded by the caller;
 *   trg_profile_enable when on, every kernel launch is bracketed by CUDA events
 *                      on the context's stream;
 *   trg_profile_read   total milliseconds and launch count of the kernels whose
 *                      name contains `name` since profiling was enabled. */
int trg_enqueue_steps(trg_ctx* c, int nsteps, double dt_next_checkpoint);
void* trg_stream(const trg_ctx* c);
int trg_profile_enable(trg_ctx* c, int on);
int trg_profile_read(trg_ctx* c, const char* name, double* total_ms, long long* launches);

/* Solver counters (no counterpart in the reference, which counts nothing):
 * when enabled, the implicit ionisation solve (Radiation::update_HIIfrac,
 * src/Radiation/Radiation.cpp:375-478) and the thermal subcycles
 * (Thermodynamics::integrate, src/Thermodynamics/Thermodynamics.cpp:266-337)
 * accumulate the TRG_STAT_* counters below.  trg_stats copies TRG_NSTATS
 * values out (after synchronising) and zeroes them when reset != 0. */
#define TRG_NSTATS 24
enum {
	TRG_STAT_PICARD_CELLS = 0, /* cells that ran the Picard solve */
	TRG_STAT_PICARD_ITERS = 1, /* Picard iterations, summed over cells */
	TRG_STAT_PICARD_MAX = 2,   /* most iterations in one cell */
	TRG_STAT_PICARD_HIST = 3,  /* 8 bins: 1, 2, 3-4, 5-8, 9-16, 17-64, 65-1024, >1024 iterations */
	TRG_STAT_LEARNED_CELLS = 11,    /* cells that started from the learned iterate */
	TRG_STAT_LEARNED_ACCEPTED = 12, /* ... whose first iteration met the convergence test */
	TRG_STAT_LEARNED_ITERS = 13,    /* Picard iterations of the learned-start cells */
	TRG_STAT_THERMO_CELLS = 14,     /* cells that subcycled */
	TRG_STAT_THERMO_SUBCYCLES = 15, /* subcycles, summed over cells */
	TRG_STAT_THERMO_MAX = 16,       /* most subcycles in one cell */
	TRG_STAT_SWEEPS = 17,           /* radiation sweeps counted */
	TRG_STAT_FRONT_CELLS = 18,      /* front cells (tau < 20, x_HII < 0.99): the learned start's domain */
	TRG_STAT_FRONT_ITERS = 19,      /* Picard iterations of the front cells */
	TRG_STAT_FP64_CELLS = 20        /* FP32 form: hydro cell updates done in FP64 (pressure contrast) */
};
/* FP32 form with radiation or cooling (no counterpart in the reference): a
 * hydro cell update is done in FP64 instead of FP32 where the pressures of
 * its stencil (two cells either side along each axis) differ by more than
 * the factor `contrast` (default 1e3; 0 turns the fallback off), i.e. around
 * strong shocks, where FP32 flux differences keep too few digits.  The count
 * of such updates is the TRG_STAT_FP64_CELLS counter. */
int trg_fp32_contrast(trg_ctx* c, double contrast);
/* FP32 form with radiation or cooling (no counterpart in the reference): the
 * fused hydro pass stages each plane of a CTA whose haloed box lies inside
 * the grid with one tiled TMA copy (on, the default) or, off, with per-cell
 * asynchronous copies like the CTAs at the grid's edges.  Bitwise the same
 * results either way. */
int trg_fp32_tma(trg_ctx* c, int on);

/* Thermal sub-cycles through a work queue (no counterpart in the reference,
 * whose Thermodynamics::integrate, src/Integrators/Thermodynamics.cpp:266-337,
 * loops over the cells): with min_subcycles > 0, cells whose closed-form
 * sub-cycle count (:304-310) is at least min_subcycles leave the in-place pass
 * for a queue, binned by the bit length of their count, heaviest first, which
 * a persistent kernel drains (each warp takes 32 cells of similar count).
 * Results are bitwise those of the in-place pass; a cell with more than 2^26
 * sub-cycles is reported as TRG_ERR_SUBCYCLE.  0 (the default) switches the
 * queue off.  Single grids only (batches run the sub-cycles in place). */
int trg_thermo_queue(trg_ctx* c, int min_subcycles);

/* Global FP64 conservation sums (no counterpart in the reference): total
 * mass sum(rho V) and total energy sum(E V) over the grid's cells (code
 * units; V the cell volume of Grid::computeCellVolume,
 * src/Fluid/Grid.cpp:876-905).  Every product is formed exactly and the sum
 * is carried in double-double in a fixed order, so the result is
 * deterministic and is the exact sum rounded once.  trg_conservation_sums
 * returns the sums of the current state (either pointer may be NULL).  With
 * trg_conservation_enable(c, 1) every full step also records the sums of the
 * state it starts from (in the FP64 forms as a side product of the time-step
 * reduction, Torch::calculateTimeStep); trg_conservation_history copies up
 * to max_entries records [n][2] (mass, energy), record k being the state
 * after k steps, and sets *n_entries to the number of steps recorded so far
 * (NaN for steps run while recording was off). */
int trg_conservation_sums(trg_ctx* c, double* mass, double* energy);
int trg_conservation_enable(trg_ctx* c, int on);
int trg_conservation_history(trg_ctx* c, double* out, long long max_entries, long long* n_entries);

/* Heating and cooling diagnostics (Thermodynamics::fillHeatingArrays,
 * src/Integrators/Thermodynamics.cpp:419-461, as printed by
 * DataPrinter::printHeating at every checkpoint of Torch::run): with
 * trg_heating_enable(c, 1) the step keeps the terms it produces (EUV heating
 * and recombination cooling of the radiation module, the total rate of the
 * thermal sub-cycles); trg_heating then runs the column-density sweep and the
 * remaining terms and copies the 11 fields [11][N] (code units, in the order
 * IMLC NMLC RHII CEHI CIEC NMC EUVH FUVH IRH CRH TOT) to H. */
#define TRG_NHEAT 11
int trg_heating_enable(trg_ctx* c, int on);
int trg_heating(trg_ctx* c, double* H);

/* Checkpoint / restart (the reference restarts from its text snapshots,
 * src/IO/DataReader.cpp:18-125, which hold the primitives only): the whole
 * step state - U, Q, R (radiation), T (thermodynamics), T_min, the FP32
 * state, time, time step and the split's counters - as one binary blob of
 * trg_checkpoint_bytes(c) bytes.  trg_checkpoint_load restores it into a
 * context created with the same parameters and grid; stepping on is
 * bit-identical to the run that was saved.  The blob holds the device layout
 * of R and T and a format version (2); a blob of another version is rejected
 * with TRG_ERR_ARG.  The FP64 form and the FP32 form of a radiation or
 * cooling run keep the same FP64 state, so either form continues the other's
 * blob (switching precision mid-run); the hydro-only FP32 form's state is
 * FP32 and its blobs restore only into that form. */
long long trg_checkpoint_bytes(const trg_ctx* c);
int trg_checkpoint_save(trg_ctx* c, void* buf, long long bytes);
int trg_checkpoint_load(trg_ctx* c, const void* buf, long long bytes);

/* Tile autotuner (no counterpart in the reference): for the FP32 form, times
 * the fused hydro stage kernel on this grid for a range of CTA tile depths
 * (z planes marched by one CTA) and keeps the fastest; the trials write only
 * scratch and leave the state and time step untouched.  zchunk_out / ms_out
 * (may be NULL) receive the choice and its time per launch; the FP64 form has
 * nothing to tune (0). */
int trg_autotune(trg_ctx* c, int* zchunk_out, double* ms_out);
/* Sets the FP32 form's CTA tile depth directly (1..nz; results do not depend
 * on it), in place of the autotuner's choice; returns the depth in effect. */
int trg_fp32_tile(trg_ctx* c, int zchunk);

int trg_stats_enable(trg_ctx* c, int on);
int trg_stats(trg_ctx* c, unsigned long long* out, int reset);

/* Learned starting iterate of the implicit ionisation solve (no counterpart
 * in the reference, whose update_HIIfrac, src/Radiation/Radiation.cpp:375-478,
 * always starts from the cell's current x_HII).
 *
 * Model: a 5 -> 64 -> 64 -> 3 perceptron with ReLU hidden layers, BF16
 * weights and activations and FP32 accumulation on the tensor cores
 * (tcgen05).  Inputs: log10 n_H, log10 T, x_HII, log10 of the optically thin
 * photoionisation rate (photon rate e^-tau sigma ds / shell volume), log10 dt.
 * Outputs: the change of logit10 from the start-of-step x_HII to the
 * converged time-averaged fraction <x> and to the end-of-step x, and log2 of
 * the plain solve's iteration count (logit10 p = log10(p / (1 - p)), p
 * clipped to [1e-9, 1 - 1e-9]).  Parameters
 * are a flat float vector of TRG_MLP_NPARAMS values: W1[5][64] b1[64]
 * W2[64][64] b2[64] W3[64][3] b3[3], then the input mean[5] and 1/std[5] and
 * the output mean[3] and 1/std[3] of the normalisation (x - mean) * scale.
 *
 * Training set records are 8 floats: the 5 inputs then the 3 targets, as the
 * plain solve records them with trg_harvest.  trg_mlp_train sets the
 * normalisation from the training set, then runs `epochs` passes of Adam
 * (beta 0.9/0.999, eps 1e-8) over seeded shuffles in batches of `batch`, on
 * the weighted squared error with per-output weights out_weight[3];
 * loss_history[e] = mean weighted squared error of epoch e (may be null).
 * trg_mlp_gradient returns the summed gradient and loss of one pass over the
 * records without updating, for gradient checks.
 *
 * trg_learned_start(ctx, m) makes the front cells (tau < 20, x_HII < 0.99)
 * of ctx's radiation sweeps that m predicts to need more than two plain
 * iterations try m's predicted <x> beside their plain first Picard iteration:
 * the prediction's iteration is accepted when it passes the solver's own
 * convergence test (its residual is below the solver tolerance) and the
 * plain one does not; otherwise the plain iteration goes on unchanged.
 * m = NULL restores the plain solve.  m must live on ctx's device; its
 * parameters are copied, so later training does not change ctx until the
 * next call.
 * trg_harvest(ctx, capacity) makes the plain solve record front cells (at
 * most `capacity` records; 0 stops and frees); trg_harvest_read copies up to
 * `max` records out and returns how many were recorded in total. */
#define TRG_MLP_NPARAMS 4755
#define TRG_MLP_NTRAIN 4739
typedef struct trg_mlp trg_mlp;
int trg_mlp_create(const float* params, int device, trg_mlp** out);
int trg_mlp_get_params(trg_mlp* m, float* params);
int trg_mlp_set_params(trg_mlp* m, const float* params);
int trg_mlp_forward(trg_mlp* m, const float* x, long n, float* y);
int trg_mlp_gradient(trg_mlp* m, const float* records, long n, const float* out_weight, float* grad, double* loss);
int trg_mlp_train(trg_mlp* m, const float* records, long n, int epochs, int batch, float lr, unsigned seed,
                  const float* out_weight, float* loss_history);
const char* trg_mlp_last_error(const trg_mlp* m);
void trg_mlp_destroy(trg_mlp* m);
int trg_learned_start(trg_ctx* c, const trg_mlp* m);
int trg_harvest(trg_ctx* c, long capacity);
long trg_harvest_read(trg_ctx* c, float* out, long max);
const char* trg_last_error(const trg_ctx* c);
void trg_destroy(trg_ctx* c);

/* Batches (no counterpart in the reference, which runs one grid per job):
 * many independent grids advance together, one kernel launch per stage for
 * all of them (one per shell for the radiation and column-density sweeps).
 * trg_batch_create takes up to 512 contexts made by trg_create in the FP64
 * form on one device, not yet stepped, with the same physics flags, solver
 * and integrator components (sizes, geometry of the star, photon rate and
 * initial state may differ), each of at most 4194304 cells.  While the batch
 * exists the grids are stepped only through it; their states are read with
 * trg_get_state after trg_batch_synchronize.  trg_batch_destroy hands the
 * step count back to the grids, which stay owned by the caller.  Every grid
 * takes its own time step (the step's minimum with dt_next_checkpoint). */
typedef struct trg_batch trg_batch;
int trg_batch_create(trg_ctx* const* grids, int ngrids, trg_batch** out);
int trg_batch_run_steps(trg_batch* b, int nsteps, double dt_next_checkpoint);
int trg_batch_enqueue_steps(trg_batch* b, int nsteps, double dt_next_checkpoint);
/* One captured CUDA graph per timestep (default on): the steps of a batch
 * after its first are replayed from graphs captured once per position of the
 * operator split's rotating component order (bitwise the same results as the
 * launches themselves, which `on` = 0 restores). */
int trg_batch_step_graphs(trg_batch* b, int on);
/* The learned starting iterate (trg_learned_start) for every grid of a batch
 * of radiation grids (implicit scheme): before each radiation sweep one
 * launch lists the candidate front cells of all grids and one runs the
 * network over them; m = NULL restores the plain solve.  A batch with the
 * network steps every grid as trg_learned_start steps it alone. */
int trg_batch_learned_start(trg_batch* b, const trg_mlp* m);
/* The conserved state U [7][N_g] of grid g of the batch, copied in or out on
 * the batch's stream, ordered with its steps (asynchronous with respect to
 * the host: pinned host buffers, and trg_batch_synchronize before reading a
 * result).  A state copied in is the start of the next step, as
 * trg_set_conserved is for a single grid. */
int trg_batch_set_conserved(trg_batch* b, int g, const double* U);
int trg_batch_get_conserved(trg_batch* b, int g, double* U);
int trg_batch_synchronize(trg_batch* b);
void* trg_batch_stream(const trg_batch* b);
long long trg_batch_kernel_launches(const trg_batch* b);
long long trg_batch_cells(const trg_batch* b);
int trg_batch_profile_enable(trg_batch* b, int on);
int trg_batch_profile_read(trg_batch* b, const char* name, double* total_ms, long long* launches);
const char* trg_batch_last_error(const trg_batch* b);
void trg_batch_destroy(trg_batch* b);

/* No counterpart in the reference.  One FP32 RK2 hydro step - the two fused
 * stage kernels of the FP32 form - from U_in to U_out, both caller-owned
 * device arrays of [7][N] doubles in code units (the layout of trg_get_state;
 * U_in == U_out is allowed), for time step dt (positive and finite), on
 * `stream` (a cudaStream_t, NULL for the default stream), using the
 * parameters of context c.  Hydrodynamics only: a context with radiation or
 * cooling on is rejected with TRG_ERR_ARG.  If dt_next is not NULL it
 * receives the time step the next call may take: the CFL limit of the new
 * state (Hydrodynamics::calculateTimeStep), at most dt_max - the caller
 * chooses dt, and this is the stable choice.  It allocates no device memory:
 * for callers that may not allocate once they run (their device memory is
 * reserved up front by their own allocator, or cudaMalloc's implicit
 * synchronisation is not allowed on their stepping path).  Its intermediate
 * state lives in a static device array of at most TRG_NOALLOC_MAX_CELLS
 * cells (about 14 MiB, held by every GPU that loads the library until exit);
 * larger grids are rejected with TRG_ERR_ARG.  All calls share that array:
 * calls that overlap on the GPU race.  The call switches to the context's
 * device and restores the caller's current device before it returns; it
 * waits for its stream (it reads the error status back), so it must not be
 * made while a stream is being captured. */
#define TRG_NOALLOC_MAX_CELLS 262144
int trg_hydro_step_fp32_noalloc(trg_ctx* c, const double* U_in, double* U_out, double dt, double* dt_next,
                                void* stream);

/* x-slab decomposition, one slab per GPU, as the reference splits its grid over MPI ranks
 * (Grid::initialise, src/Fluid/Grid.cpp:446-459; the halo exchange of
 * Grid::applyBCs PARTITION, :804-833; the minimum time step over ranks,
 * src/Torch/Torch.cpp:323-335).  trg_create_slab takes the whole grid's
 * parameters p and the cells of one slab - global x from x0 to x0 + nx - 1,
 * nx >= 2, every y and z, flat index i + nx*(j + ny*k) - and, for the FP32
 * form, the whole grid's reference density and pressure f32_scale[2] in
 * code units (NULL: the slab's own medians; give the same values to every
 * slab for results equal to the undecomposed run's).  An x face that borders
 * another slab (or the other end of a periodic grid) takes its ghost layers
 * from the neighbour (trg_slab_partitions: bit 1 the low x face, bit 2 the
 * high one).  trg_f32_scales gives the whole grid's f32_scale from its
 * initial fields (host only).  Before stepping, trg_slab_exchange registers
 * the host's hook, two device buffers of trg_slab_halo_bytes(c) bytes each,
 * [side 2][layer 2][field 7][ny*nz] (layer 0 next to the face; doubles, or
 * floats in the hydro-only FP32 form), and a device buffer dt_buf of three
 * unsigned 64-bit integers.  The library calls
 *   fn(user, TRG_EXCHANGE_HALO, stream): halo_send holds this slab's layers,
 *     packed on `stream`; the hook must make halo_recv hold the neighbours'
 *     (recv[left] = left neighbour's send[right], recv[right] = right
 *     neighbour's send[left]) in `stream` order before it returns (e.g. NCCL
 *     send/recv enqueued on `stream`), and must not let a neighbour's next
 *     pack overwrite its send buffer before the copy has read it;
 *   fn(user, TRG_EXCHANGE_DT, stream): dt_buf holds this slab's three
 *     time-step minima (bit patterns of positive doubles: an integer minimum
 *     is the minimum of the values); each must become its minimum over all
 *     slabs, in `stream` order (e.g. an NCCL all-reduce MIN on `stream`);
 * and a nonzero return makes the step return TRG_ERR_ARG.  Every slab calls
 * the hook the same number of times in the same order. */
#define TRG_EXCHANGE_HALO 0
#define TRG_EXCHANGE_DT 1
/* Slabs of a run with a star (radiation and/or cooling, FP64 form, no stellar
 * wind) also sweep slab after slab outwards from the slab that holds the star
 * (trg_slab_star_side: 0 this slab holds it, 1 it lies at lower x, 2 at
 * higher x), as the reference's ranks pass their boundary optical depths and
 * column densities on (Radiation::transferRadiation, src/Integrators/
 * Radiation.cpp:573-636; Thermodynamics::rayTrace, Thermodynamics.cpp:365-417).
 * Before stepping, trg_slab_sweep_exchange registers two more device buffers
 * of trg_slab_sweep_bytes(c) bytes each, [side 2][ny*nz][4] doubles, and the
 * library calls, around every causal sweep,
 *   fn(user, TRG_EXCHANGE_SWEEP_IN, stream): before the sweep; sweep_recv
 *     must hold, in `stream` order, the star-side neighbour's sweep_send of
 *     its side facing this slab (nothing for the star's own slab), and this
 *     slab's sweep_send must be free to be overwritten (every neighbour away
 *     from the star has read its previous contents);
 *   fn(user, TRG_EXCHANGE_SWEEP_OUT, stream): after the sweep; sweep_send
 *     holds this slab's boundary layers, packed on `stream`, for the
 *     neighbours away from the star (the low-x side unless the star lies at
 *     lower x or this is the first slab, the high-x side unless it lies at
 *     higher x or this is the last).
 * Each slab's first causal non-wind cell takes the radiation time step's
 * one-off form, as each rank's does in the reference (Radiation.cpp:300-316).
 * The column-density sweep of the Torch::run prologue, which trg_create runs
 * for a whole grid, runs at the start of a slab's first step (the hook is not
 * registered yet when the slab is created); trg_heating is a collective call
 * for slabs, since its ray trace goes through the sweep exchange. */
#define TRG_EXCHANGE_SWEEP_IN 2
#define TRG_EXCHANGE_SWEEP_OUT 3
typedef int (*trg_exchange_fn)(void* user, int what, void* stream);
int trg_create_slab(const trg_params* p, int x0, int nx, const double* f32_scale, const double* den,
                    const double* pre, const double* hii, const double* v0, const double* v1, const double* v2,
                    const double* grav, trg_ctx** out);
int trg_slab_exchange(trg_ctx* c, trg_exchange_fn fn, void* user, void* halo_send, const void* halo_recv,
                      void* dt_buf);
long long trg_slab_halo_bytes(const trg_ctx* c);
int trg_slab_partitions(const trg_ctx* c);
int trg_slab_sweep_exchange(trg_ctx* c, void* sweep_send, const void* sweep_recv);
long long trg_slab_sweep_bytes(const trg_ctx* c);
int trg_slab_star_side(const trg_ctx* c);
int trg_f32_scales(const trg_params* p, const double* den, const double* pre, const double* hii, const double* v0,
                   const double* v1, const double* v2, double* f32_scale);

#ifdef __cplusplus
}
#endif
#endif
