// One FP32 RK2 hydro step on caller-owned device buffers that allocates no
// device memory.
//
// Who needs it: callers that may not allocate device memory once they are
// running - a host application that reserves its whole device-memory budget up
// front through its own allocator, or a stepping loop on which cudaMalloc's
// implicit device-wide synchronisation is not acceptable.  The regular path
// (trg_full_step on an FP32 context) keeps its RK2 intermediate state in memory
// the context allocated; this entry point keeps it, and its few scalars, in the
// file-scope array below instead.
//
// Limits and sharing:
//   * at most TRG_NOALLOC_MAX_CELLS cells (larger grids are rejected with
//     TRG_ERR_ARG); the array takes about 14 MiB on every GPU that loads the
//     library, until the process exits;
//   * every call uses the same array and leaves its contents behind; what must
//     start at zero (the error word, the time-step minima) is cleared by each
//     call, and calls that overlap on the GPU race on the array;
//   * the first call on a device looks the array's device address up
//     (cudaGetSymbolAddress, with that device current);
//   * every call waits for its stream (it reads the error word and the next
//     time-step limit back), so it must not be made while a stream is being
//     captured;
//   * hydrodynamics only: contexts with radiation or cooling are rejected.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "../../include/torch_b200.h"
#include "ctx_access.h"
#include "trg_kernels.h"

namespace trg {
namespace {

constexpr long long kMaxCells = TRG_NOALLOC_MAX_CELLS;
constexpr long long kHeaderFloats = 64;  // 256 bytes: 8 doubles (dt, time, minima) + the error word
constexpr long long kScratchFloats = kHeaderFloats + 2LL * 7 * kMaxCells;

// The scratch: [header | U (7 x kMaxCells) | U* (7 x kMaxCells)] in FP32.
// In host code `g_noalloc_scratch` is only a handle for cudaGetSymbolAddress.
static __device__ __align__(256) float g_noalloc_scratch[kScratchFloats];

constexpr int kMaxDevices = 64;
float* g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mutex;

// Device address of the scratch array on the current device (looked up once per device).
cudaError_t scratch_address(int device, float** out) {
	if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
	std::lock_guard<std::mutex> lock(g_scratch_mutex);
	if (!g_scratch_ptr[device]) {
		void* p = nullptr;
		cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		if (e != cudaSuccess) return e;
		g_scratch_ptr[device] = static_cast<float*>(p);
	}
	*out = g_scratch_ptr[device];
	return cudaSuccess;
}

// Stages dt and clears what must start at zero: the error word and the CFL minima.
__global__ void k_noalloc_begin(double* scal, unsigned* err, double dt, double dt_max) {
	scal[0] = dt;
	scal[1] = 0.0;
	unsigned long long big = (unsigned long long)__double_as_longlong(dt_max);
	unsigned long long* slots = reinterpret_cast<unsigned long long*>(scal + 2);
	slots[0] = big;
	slots[1] = big;
	slots[2] = big;
	*err = 0u;
}

}  // namespace
}  // namespace trg

using namespace trg;

namespace {
// Restores the calling thread's current device on every return path.
struct DeviceGuard {
	int prev = -1;
	DeviceGuard() {
		if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
	}
	~DeviceGuard() {
		if (prev >= 0) cudaSetDevice(prev);
	}
};
}  // namespace

extern "C" int trg_hydro_step_fp32_noalloc(trg_ctx* c, const double* U_in, double* U_out, double dt,
                                           double* dt_next, void* stream) {
	if (!c || !U_in || !U_out) return TRG_ERR_ARG;
	const Params& P = ctx_params(c);
	if (P.N > kMaxCells)
		return ctx_fail(c, TRG_ERR_ARG,
		                "trg_hydro_step_fp32_noalloc: grid of " + std::to_string(P.N) +
		                    " cells exceeds the limit of " + std::to_string(kMaxCells) + " cells");
	if (P.nd < 2)
		return ctx_fail(c, TRG_ERR_ARG, "trg_hydro_step_fp32_noalloc: needs a 2-D or 3-D grid");
	if (P.radiation_on || P.cooling_on)
		return ctx_fail(c, TRG_ERR_ARG,
		                "trg_hydro_step_fp32_noalloc: advances hydrodynamics only; the context has radiation or "
		                "cooling on");
	if (!(dt > 0) || !(dt <= 1.0e308))
		return ctx_fail(c, TRG_ERR_ARG, "trg_hydro_step_fp32_noalloc: dt must be positive and finite");
	if (P.lbc[0] == BC_PARTITION || P.rbc[0] == BC_PARTITION)
		return ctx_fail(c, TRG_ERR_ARG, "trg_hydro_step_fp32_noalloc: takes whole grids, not slabs");
	DeviceGuard guard;
	cudaError_t e = cudaSetDevice(ctx_device(c));
	float* base = nullptr;
	if (e == cudaSuccess) e = scratch_address(ctx_device(c), &base);
	if (e != cudaSuccess)
		return ctx_fail(c, TRG_ERR_CUDA, std::string("trg_hydro_step_fp32_noalloc: ") + cudaGetErrorString(e));
	cudaStream_t st = static_cast<cudaStream_t>(stream);
	double* scal = reinterpret_cast<double*>(base);
	unsigned* err = reinterpret_cast<unsigned*>(base + 16);
	float* U0 = base + kHeaderFloats;
	float* Us = U0 + 7 * kMaxCells;
	State S = ctx_state(c);  // geometry / gravity inputs of the context, read only
	S.scal = scal;
	S.err = err;
	S.dt_hist = nullptr;
	const long long N = P.N;
	k_noalloc_begin<<<1, 1, 0, st>>>(scal, err, dt, P.dt_max);
	k_f64_to_f32<<<(unsigned)((7 * N + 255) / 256), 256, 0, st>>>(P, U_in, U0);
	int zchunk = ctx_fp32_zchunk(c);
	launch_hydro_stage_fp32(1, P, S, U0, U0, Us, zchunk, st);
	launch_hydro_stage_fp32(2, P, S, Us, U0, U0, zchunk, st);
	k_f32_to_f64<<<(unsigned)((7 * N + 255) / 256), 256, 0, st>>>(P, U0, U_out);
	// header bytes 16..67: the CFL minimum (scal[2], bits of a positive double)
	// up to the error word (float 16 = byte 64), read back in one copy
	unsigned char hdr[52];
	e = cudaGetLastError();
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(hdr, reinterpret_cast<unsigned char*>(base) + 16, sizeof hdr, cudaMemcpyDeviceToHost, st);
	if (e == cudaSuccess) e = cudaStreamSynchronize(st);
	if (e != cudaSuccess)
		return ctx_fail(c, TRG_ERR_CUDA, std::string("trg_hydro_step_fp32_noalloc: ") + cudaGetErrorString(e));
	unsigned h_err = 0;
	double cfl = 0;
	memcpy(&cfl, hdr, sizeof cfl);
	memcpy(&h_err, hdr + 48, sizeof h_err);
	if (h_err & ERRB_NAN) return ctx_fail(c, TRG_ERR_NAN, "checkValues/fixSolution: invalid cell state");
	if (dt_next) *dt_next = cfl < P.dt_max ? cfl : P.dt_max;
	return TRG_OK;
}
