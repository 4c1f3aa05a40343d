// Kernel entry points shared between the kernel translation units and the
// orchestration in capi.cu.
#pragma once
#include "trg_device.cuh"

// kernels_fp64.cu, built three times: exact (plain-FP64 form, rounds like the
// reference), fast (FP32 form; FMA and CUDA libm) and fastb (fast, with the
// batch dispatch, for FP32-form batches)
#define TRG_FP64_KERNELS \
	__global__ void k_faces_fp64(Params P, State S, int dim); \
	__global__ void k_hydro_update_fp64(Params P, State S, double h, int sel_base, int sel_out, int mode); \
	__global__ void k_q_from_u_fp64(Params P, State S, int sel_src, int fix); \
	__global__ void k_advance_fp64(Params P, State S, double dt); \
	__global__ void k_rad_wind_reset(Params P, State S, const int* cells, int count); \
	__global__ void k_rad_shell_fp64(Params P, State S, const int* cells, int count, double h); \
	__global__ void k_learned_infer(Params P, State S, const int* cells, double h); \
	__global__ void k_rad_shell_sw_diag(Params P, State S, const int* cells, int count, double h, long long off); \
	__global__ void k_rad_shell_sw_ls(Params P, State S, const int* cells, int count, double h, long long off); \
	__global__ void k_rad_shell_fp64_ls(Params P, State S, const int* cells, int count, double h); \
	__global__ void k_batch_learned_prep(Params Pv, State Sv); \
	__global__ void k_batch_learned_infer(Params Pv, State Sv, double h); \
	__global__ void k_rad_shell_diag(Params P, State S, const int* cells, int count, double h); \
	__global__ void k_rad_no_star_fp64(Params P, State S, double h); \
	__global__ void k_rad_tau_shell(Params P, State S, const int* cells, int count); \
	__global__ void k_rad_solve2(Params P, State S, const int* cells, int count, double h); \
	__global__ void k_rad_heating_fp64(Params P, State S); \
	__global__ void k_rad_update_fp64(Params P, State S, double h, int mode); \
	__global__ void k_colden_shell_fp64(Params P, State S, const int* cells, int count); \
	__global__ void k_colden_shell_sw(Params P, State S, const int* cells, int count, long long off); \
	__global__ void k_colden_sweep_prep(Params P, State S, const int* cells, int n, int init); \
	__global__ void k_rad_shell_sw(Params P, State S, const int* cells, int count, double h, long long off); \
	__global__ void k_rad_sweep_prep(Params P, State S, const int* cells, int n, int init); \
	__global__ void k_thermo_rates_fp64(Params P, State S); \
	__global__ void k_thermo_integrate_fp64(Params P, State S, double h); \
	__global__ void k_thq_layout(State S); \
	__global__ void k_thq_scatter(State S); \
	__global__ void k_thq_drain(Params P, State S, double h); \
	__global__ void k_thermo_update_fp64(Params P, State S, double h, int mode); \
	__global__ void k_heating_arrays_fp64(Params P, State S); \
	__global__ void k_fb_flags(Params P, State S, double contrast); \
	__global__ void k_fb_faces(Params P, State S); \
	__global__ void k_fb_update(Params P, State S, double h); \
	__global__ void k_dt_reduce_fp64(Params P, State S, long long first_cell); \
	__global__ void k_dt_finalize(Params P, State S, double dt_next, int first_time, int step); \
	__global__ void k_time_advance(Params P, State S); \
	__global__ void k_dt_reset(Params P, State S);

namespace trg {
namespace exact {
TRG_FP64_KERNELS
}
namespace fast {
TRG_FP64_KERNELS
}
namespace fastb {  // the fast build with the batch dispatch (FP32-form batches)
TRG_FP64_KERNELS
}
// FP32 form of the hydro pass (kernels_fp32.cu)
void launch_hydro_stage_fp32(int stage, const Params& P, const State& S, const float* Uq, const float* Ubase,
                             float* Uout, int zchunk, cudaStream_t stream);
size_t hydro_stage_fp32_smem();
void launch_hydro_substep_fp32(const Params& P, const State& S, const double* U, double* Uout, double h, int zchunk,
                               cudaStream_t stream);
__global__ void k_f64_to_f32(Params P, const double* a, float* b);
// x-slab decomposition: pack the layers next to the partition faces into dst
// (kernels_fp32.cu); src is [7][N] doubles, or floats when f32
void launch_halo_pack(const Params& P, const void* src, void* dst, bool f32, cudaStream_t stream);
// ... and with a star, the boundary x layer of R's optical depths (colden =
// false) or T's column densities into dst [side 2][ny * nz][4] after a sweep
void launch_sweep_pack(const Params& P, const double* src, bool colden, double* dst, cudaStream_t stream);
// FP32 form of a batch of 2-D grids: the hydro sub-step of every grid (U -> U1,
// then U1 copied back to U)
void launch_hydro_substep_fp32_batch(const Params& Pv, const BatchTable* B, int ntiles, double h, cudaStream_t stream);
// global FP64 mass and energy sums (conservation.cu): block partials of a
// state, and the fold of the partials (also those of k_dt_reduce_fp64) into
// out[0] = sum(rho V), out[1] = sum(E V)
long long cons_nparts(const Params& P);
void launch_cons_cells_f64(const Params& P, const double* U, double* part, cudaStream_t st);
void launch_cons_cells_f32(const Params& P, const float* U, double* part, cudaStream_t st);
void launch_cons_finalize(const Params& P, const double* part, double* out, cudaStream_t st);
}  // namespace trg
// network image of a trained model (mlp.cu) and the device it lives on
const unsigned char* mlp_device_image(const trg_mlp* m, int* device);
namespace trg {
__global__ void k_f32_to_f64(Params P, const float* a, double* b);
}  // namespace trg
