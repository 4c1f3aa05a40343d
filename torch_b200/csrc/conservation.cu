// Global FP64 mass and energy sums of a context's state, sum(rho V) and
// sum(E V) over the cells (no counterpart in the reference, whose step keeps no
// such check).
//
// Two passes: per 256-cell block a double-double partial (the time-step
// reduction of the FP64 forms forms the same partials as a side product,
// kernels_fp64.cu), then one block that folds the partials in a fixed order and
// writes the rounded pair (mass, energy).  The result is deterministic and is
// the exact sum of the exact products rho V and E V, rounded once (up to about
// 2^-100 relative before that rounding).
#include <cuda_runtime.h>

#include "trg_kernels.h"

namespace trg {

// Partials of a state held as FP64 code units (scale 1) or as the FP32 form's
// scaled units (the stored value times the field's reference value rho0 or
// p0, formed exactly as a double-double before the volume product).
template <typename TS>
__global__ void __launch_bounds__(256) k_cons_cells(Params P, const TS* __restrict__ U, double sden, double spre,
                                                    double* __restrict__ part) {
	const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	DD m = {0.0, 0.0}, e = {0.0, 0.0};
	if (id < P.N) {
		int ijk[3];
		double xc[3];
		cell_ijk(P, id, ijk);
		cell_xc(P, ijk, xc);
		const double vol = cell_volume_rn(P, xc[0]);
		const double d = (double)U[DEN * P.N + id], E = (double)U[PRE * P.N + id];
		if (sizeof(TS) == sizeof(double)) {
			m = dd_prod(d, vol);
			e = dd_prod(E, vol);
		} else {
			const DD md = dd_prod(d, sden), ed = dd_prod(E, spre);
			m = dd_prod(md.hi, vol);
			m = dd_add(m, DD{__dmul_rn(md.lo, vol), 0.0});
			e = dd_prod(ed.hi, vol);
			e = dd_add(e, DD{__dmul_rn(ed.lo, vol), 0.0});
		}
	}
	block_cons_partial(m, e, part, blockIdx.x);
}

// Folds nparts block partials in a fixed order (thread t takes t, t + 512, ...;
// then a fixed tree) and writes (mass, energy) to out[0], out[1].
__global__ void __launch_bounds__(512) k_cons_finalize(const double* __restrict__ part, long long nparts,
                                                       double* __restrict__ out) {
	__shared__ double red[512][4];
	DD m = {0.0, 0.0}, e = {0.0, 0.0};
	for (long long k = threadIdx.x; k < nparts; k += blockDim.x) {
		m = dd_add(m, DD{part[4 * k + 0], part[4 * k + 1]});
		e = dd_add(e, DD{part[4 * k + 2], part[4 * k + 3]});
	}
	red[threadIdx.x][0] = m.hi;
	red[threadIdx.x][1] = m.lo;
	red[threadIdx.x][2] = e.hi;
	red[threadIdx.x][3] = e.lo;
	__syncthreads();
	for (int w = blockDim.x / 2; w > 0; w >>= 1) {
		if ((int)threadIdx.x < w) {
			const int o = threadIdx.x + w;
			const DD a = dd_add(DD{red[threadIdx.x][0], red[threadIdx.x][1]}, DD{red[o][0], red[o][1]});
			const DD b = dd_add(DD{red[threadIdx.x][2], red[threadIdx.x][3]}, DD{red[o][2], red[o][3]});
			red[threadIdx.x][0] = a.hi;
			red[threadIdx.x][1] = a.lo;
			red[threadIdx.x][2] = b.hi;
			red[threadIdx.x][3] = b.lo;
		}
		__syncthreads();
	}
	if (threadIdx.x == 0) {
		out[0] = __dadd_rn(red[0][0], red[0][1]);
		out[1] = __dadd_rn(red[0][2], red[0][3]);
	}
}

long long cons_nparts(const Params& P) { return (P.N + 255) / 256; }

void launch_cons_cells_f64(const Params& P, const double* U, double* part, cudaStream_t st) {
	k_cons_cells<double><<<(unsigned)cons_nparts(P), 256, 0, st>>>(P, U, 1.0, 1.0, part);
}
void launch_cons_cells_f32(const Params& P, const float* U, double* part, cudaStream_t st) {
	k_cons_cells<float><<<(unsigned)cons_nparts(P), 256, 0, st>>>(P, U, P.f32_rho0, P.f32_p0, part);
}
void launch_cons_finalize(const Params& P, const double* part, double* out, cudaStream_t st) {
	k_cons_finalize<<<1, 512, 0, st>>>(part, cons_nparts(P), out);
}

}  // namespace trg
