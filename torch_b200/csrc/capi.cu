// C ABI and step orchestration (Torch::fullStep / subStep / hydroStep,
// src/Torch/Torch.cpp:352-418) for torch_b200.
//
// All device memory belongs to the context; all work is enqueued on the
// context's stream.  Time-step values stay on the device between kernels
// (the dt reduction writes them, the integrators read them), so a sequence of
// steps needs no host round trip.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "../../include/torch_b200.h"
#include "ctx_access.h"
#include "setup.h"
#include "trg_kernels.h"
#include "tc_mlp.cuh"

using namespace trg;

namespace {
constexpr int COMP_HYDRO = 0, COMP_RAD = 1, COMP_THERMO = 2;
}

inline bool colden_overlap_default() {
	const char* v = std::getenv("TRG_COLDEN_OVERLAP");
	return !(v && v[0] == '0');
}
inline bool shell_overlap_default() {
	const char* v = std::getenv("TRG_SHELL_OVERLAP");
	return !(v && v[0] == '0');
}

struct trg_ctx {
	trg_params raw;
	HostSetup hs;
	Params P;
	State S;
	cudaStream_t stream = nullptr;
	Tables* d_tables = nullptr;
	int* d_sweep_all = nullptr;
	int* d_sweep_nonwind = nullptr;
	int* d_wind = nullptr;
	// FP32 form: conserved state U0/U1 and the RK2 intermediate U* (hydro-only runs);
	// with radiation/cooling (`mixed`) the state stays FP64 and the hydro
	// sub-steps run through the FP32 kernel
	bool fp32 = false;
	bool mixed = false;
	// x-slab decomposition: the host's exchange hook and whether it failed
	trg_exchange_fn xfn = nullptr;
	void* xuser = nullptr;
	unsigned long long* xdt = nullptr;  // the host's device buffer of the three time-step minima
	bool xfail = false;
	// ... with a star: the boundary layer packed after each causal sweep for
	// the neighbour away from the star (the received one is S.sweep_recv)
	double* sweep_send = nullptr;
	// ... and the Torch::run prologue's column-density sweep, deferred to the
	// slab's first step
	bool prologue_colden = false;
	// FP32 form (either kind): the FP64 kernels come from the fast build
	int fastk = 0;  // kernel build: 0 exact, 1 fast, 2 fast with the batch dispatch
	// FP32 form with radiation/cooling: Q already holds the primitives of the
	// current U (written by the FP32 hydro sub-step), so the next
	// globalQfromU + fixPrimitives pass can be skipped
	bool q_fresh = false;
	// the column densities of the thermodynamics depend on the density alone,
	// which only hydro sub-steps change: a second sweep with no hydro sub-step
	// since the last one would recompute the same values and is skipped
	bool colden_valid = false;
	// pressure ratio above which a hydro cell update of the FP32 form falls
	// back to FP64 (0: never)
	double fb_contrast = 1.0e3;
	// side stream: the radiation heating pass runs beside the column-density
	// sweep at the start of a step (they touch disjoint fields)
	cudaStream_t side = nullptr;
	cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
	// in a split step whose radiation sub-step comes after a hydro sub-step and
	// before the next thermal one, the column-density sweep that thermal
	// sub-step needs runs on the side stream beside the radiation sweep (the
	// density it reads is the hydro sub-step's, which radiation does not
	// change); TRG_COLDEN_OVERLAP=0 keeps it in the thermal sub-step
	bool colden_overlap = colden_overlap_default();
	bool colden_join_pending = false;
	cudaEvent_t ev_cfork = nullptr, ev_cjoin = nullptr;
	// CUDA graphs of the shell sweeps (all shells of one sweep, launched as one)
	cudaGraphExec_t g_colden = nullptr;
	cudaGraphExec_t g_rad[2] = {nullptr, nullptr};
	cudaGraphExec_t g_tau = nullptr;
	long long g_tau_nodes = 0;
	long long g_colden_nodes = 0, g_rad_nodes[2] = {0, 0};
	bool use_graphs = true;
	// shells after the first of a sweep start while the previous one runs
	// (programmatic dependent launch); TRG_SHELL_OVERLAP=0 serialises them
	bool shell_overlap = shell_overlap_default();
	// per-grid scalar kernels (dt, time) run on this many threads: 1, or the
	// number of grids of a batch
	int nscalar = 1;
	int batch_tiles = 0;  // batch context, FP32 form: CTA tiles of the hydro pass
	float* U32 = nullptr;
	float* U32s = nullptr;
	unsigned char* mlp_img = nullptr;
	int* lcand_buf = nullptr;
	unsigned* lcand_n_buf = nullptr;
	double* d_heat = nullptr;
	int zchunk = 64;
	std::vector<void*> allocs;
	int first_time = 1;
	int rad_once_pending = 1;
	int stepCounter = 0;
	long long steps = 0;
	long long launches = 0;
	int dt_hist_cap = 0;
	// global FP64 mass and energy sums: on-demand result (2 doubles), block
	// partials, and (when on) the per-step record [cap][2] of the state each
	// step starts from
	// thermal sub-cycle work queue (allocated when first switched on)
	int* thq_buf = nullptr;
	int* thq_sorted_buf = nullptr;
	unsigned char* thq_bin_buf = nullptr;
	unsigned* thq_ctl_buf = nullptr;
	double* cons_out = nullptr;
	double* cons_part = nullptr;
	double* cons_hist = nullptr;
	long long cons_cap = 0;
	bool cons_on = false;
	std::string err;
	// optional per-launch CUDA-event timing
	bool profiling = false;
	struct Rec { const char* name; cudaEvent_t a, b; };
	std::vector<Rec> recs;
	std::vector<cudaEvent_t> event_pool;
	std::vector<std::pair<std::string, std::pair<double, long long>>> prof_totals;
};

namespace {

int set_error(trg_ctx* c, int code, const std::string& msg) {
	if (c) c->err = msg;
	return code;
}

#define CUDA_TRY(call)                                                                                  \
	do {                                                                                                \
		cudaError_t e_ = (call);                                                                        \
		if (e_ != cudaSuccess)                                                                          \
			return set_error(c, e_ == cudaErrorMemoryAllocation ? TRG_ERR_OOM : TRG_ERR_CUDA,         \
			                 std::string(#call) + ": " + cudaGetErrorString(e_));                         \
	} while (0)

template <typename T>
int dalloc(trg_ctx* c, T** p, size_t count) {
	void* v = nullptr;
	CUDA_TRY(cudaMalloc(&v, count * sizeof(T) + 16));
	c->allocs.push_back(v);
	*p = static_cast<T*>(v);
	return 0;
}

inline unsigned grid_for(long long n, int block) { return (unsigned)((n + block - 1) / block); }

cudaEvent_t pool_event(trg_ctx* c) {
	if (!c->event_pool.empty()) {
		cudaEvent_t e = c->event_pool.back();
		c->event_pool.pop_back();
		return e;
	}
	cudaEvent_t e = nullptr;
	cudaEventCreate(&e);
	return e;
}

// Folds completed event pairs into per-kernel totals (the stream must be idle).
void profile_collect(trg_ctx* c) {
	for (auto& r : c->recs) {
		float ms = 0;
		cudaEventElapsedTime(&ms, r.a, r.b);
		bool found = false;
		for (auto& t : c->prof_totals)
			if (t.first == r.name) { t.second.first += ms; t.second.second += 1; found = true; break; }
		if (!found) c->prof_totals.push_back({r.name, {(double)ms, 1LL}});
		c->event_pool.push_back(r.a);
		c->event_pool.push_back(r.b);
	}
	c->recs.clear();
}

// the exact or the fast build of a kernels_fp64.cu kernel, by the context's form
#define KF(name) (c->fastk == 1 ? trg::fast::name : (c->fastk == 2 ? trg::fastb::name : trg::exact::name))

#define LAUNCH(kernel, n, block, ...)                                                        \
	do {                                                                                     \
		if ((n) > 0) {                                                                       \
			cudaEvent_t ea_ = nullptr, eb_ = nullptr;                                        \
			if (c->profiling) { ea_ = pool_event(c); eb_ = pool_event(c);                    \
			                    cudaEventRecord(ea_, c->stream); }                           \
			kernel<<<grid_for((n), (block)), (block), 0, c->stream>>>(__VA_ARGS__);          \
			if (c->profiling) { cudaEventRecord(eb_, c->stream);                             \
			                    c->recs.push_back({#kernel, ea_, eb_}); }                    \
			c->launches++;                                                                   \
		}                                                                                    \
	} while (0)

// A shell of a causal sweep.  Every shell after the first of a sweep is
// launched with programmatic stream serialisation: its CTAs may start while
// the previous shell runs and wait for it inside the kernel (sweep_wait).
template <typename... KArgs, typename... Args>
void launch_shell(trg_ctx* c, void (*kernel)(KArgs...), int n, int block, bool overlap, Args... args) {
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3(grid_for(n, block));
	cfg.blockDim = dim3(block);
	cfg.dynamicSmemBytes = 0;
	cfg.stream = c->stream;
	cudaLaunchAttribute attr[1];
	attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
	attr[0].val.programmaticStreamSerializationAllowed = 1;
	cfg.attrs = attr;
	cfg.numAttrs = overlap && c->shell_overlap ? 1 : 0;
	cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}
#define LAUNCH_SHELL(kernel, n, block, overlap, ...)                                          \
	do {                                                                                     \
		if ((n) > 0) {                                                                       \
			cudaEvent_t ea_ = nullptr, eb_ = nullptr;                                        \
			if (c->profiling) { ea_ = pool_event(c); eb_ = pool_event(c);                    \
			                    cudaEventRecord(ea_, c->stream); }                           \
			launch_shell(c, kernel, (n), (block), (overlap), __VA_ARGS__);                   \
			if (c->profiling) { cudaEventRecord(eb_, c->stream);                             \
			                    c->recs.push_back({#kernel, ea_, eb_}); }                    \
			c->launches++;                                                                   \
		}                                                                                    \
	} while (0)

// sel: 0 = S.U, 1 = S.U1
#define LAUNCH_SCALAR(kernel, ...) LAUNCH(kernel, c->nscalar, c->nscalar > 1 ? 64 : 1, __VA_ARGS__)

// R and T between the C ABI's field-after-field order (soa) and the device
// layout (trg_types.h); U1, free between calls, stages the other side.
__global__ void k_layout_rt(long long N, int nf, const double* __restrict__ src, double* __restrict__ dst,
                            int to_device) {
	const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (i >= nf * N) return;
	const int f = (int)(i / N);
	const long long id = i - f * N;
	const long long d = nf == 6 ? r_index(N, f, id) : t_index(N, f, id);
	if (to_device) dst[d] = src[i];
	else dst[i] = src[d];
}
int upload_rt(trg_ctx* c, double* dev, const double* host, int nf) {
	const long long N = c->P.N;
	CUDA_TRY(cudaMemcpyAsync(c->S.U1, host, nf * N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
	k_layout_rt<<<grid_for(nf * N, 256), 256, 0, c->stream>>>(N, nf, c->S.U1, dev, 1);
	return TRG_OK;
}
int download_rt(trg_ctx* c, double* host, const double* dev, int nf) {
	const long long N = c->P.N;
	k_layout_rt<<<grid_for(nf * N, 256), 256, 0, c->stream>>>(N, nf, dev, c->S.U1, 0);
	CUDA_TRY(cudaMemcpyAsync(host, c->S.U1, nf * N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
	return TRG_OK;
}

void q_from_u(trg_ctx* c, int sel, int fix) { LAUNCH(KF(k_q_from_u_fp64), c->P.N, 256, c->P, c->S, sel, fix); }

// x-slab decomposition: before a flux computation, the layers next to the
// partition faces of `src` (the state it reads) are packed into the halo send
// buffer and the host's hook fills the receive buffer from the neighbours
// (Grid::applyBCs PARTITION, Grid.cpp:804-833), all on the context's stream.
void halo_exchange(trg_ctx* c, const void* src, bool f32) {
	if (!c->S.halo_send) return;
	launch_halo_pack(c->P, src, c->S.halo_send, f32, c->stream);
	c->launches++;
	if (c->xfn(c->xuser, TRG_EXCHANGE_HALO, c->stream) != 0) c->xfail = true;
}
// ... and before the time step is taken from the per-component minima, their
// minimum over all slabs (Torch::calculateTimeStep's MPI minimum, Torch.cpp:323-335).
void dt_exchange(trg_ctx* c) {
	if (!c->xfn) return;
	const size_t b = 3 * sizeof(unsigned long long);
	cudaMemcpyAsync(c->xdt, c->S.scal + 2, b, cudaMemcpyDeviceToDevice, c->stream);
	if (c->xfn(c->xuser, TRG_EXCHANGE_DT, c->stream) != 0) c->xfail = true;
	cudaMemcpyAsync(c->S.scal + 2, c->xdt, b, cudaMemcpyDeviceToDevice, c->stream);
}

// x-slab decomposition with a star: the causal sweeps run slab after slab
// outwards from the star's slab, as the reference's ranks do
// (Radiation.cpp:573-636, Thermodynamics.cpp:365-417).  Before a sweep the
// hook makes S.sweep_recv hold the star-side neighbour's boundary layer of
// the fields that sweep reads (and frees this slab's send buffer); after it,
// this slab's boundary layers are packed and the hook hands them on.
void sweep_in(trg_ctx* c) {
	if (!c->sweep_send) return;
	if (c->xfn(c->xuser, TRG_EXCHANGE_SWEEP_IN, c->stream) != 0) c->xfail = true;
}
void sweep_out(trg_ctx* c, bool colden) {
	if (!c->sweep_send) return;
	launch_sweep_pack(c->P, colden ? c->S.T : c->S.R, colden, c->sweep_send, c->stream);
	c->launches++;
	if (c->xfn(c->xuser, TRG_EXCHANGE_SWEEP_OUT, c->stream) != 0) c->xfail = true;
}

void colden_sweep_direct(trg_ctx* c) {
	const auto& off = c->hs.off_all;
	const bool sw = c->S.sw_col != nullptr;
	if (sw) LAUNCH(KF(k_colden_sweep_prep), c->S.sw_col_n, 256, c->P, c->S, c->d_sweep_all, (int)c->S.sw_col_n, 0);
	for (size_t s = 0; s + 1 < off.size(); ++s) {
		int count = (int)(off[s + 1] - off[s]);
		if (sw)
			LAUNCH_SHELL(KF(k_colden_shell_sw), count, 128, s > 0, c->P, c->S, c->d_sweep_all + off[s], count,
			             (long long)off[s]);
		else
			LAUNCH_SHELL(KF(k_colden_shell_fp64), count, 128, s > 0, c->P, c->S, c->d_sweep_all + off[s], count);
	}
}

// Captures `body` (kernel launches on c->stream) into an executable graph.
template <typename F>
cudaGraphExec_t capture_graph(trg_ctx* c, F body, long long& nodes) {
	bool prof = c->profiling;
	c->profiling = false;
	long long before = c->launches;
	cudaGraph_t g = nullptr;
	cudaGraphExec_t ge = nullptr;
	if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
		body();
		if (cudaStreamEndCapture(c->stream, &g) == cudaSuccess && g) {
			if (cudaGraphInstantiate(&ge, g, 0) != cudaSuccess) ge = nullptr;
			cudaGraphDestroy(g);
		}
	}
	nodes = c->launches - before;
	c->launches = before;
	c->profiling = prof;
	cudaGetLastError();
	return ge;
}

void launch_graph(trg_ctx* c, cudaGraphExec_t ge, long long nodes, const char* name) {
	cudaEvent_t ea = nullptr, eb = nullptr;
	if (c->profiling) { ea = pool_event(c); eb = pool_event(c); cudaEventRecord(ea, c->stream); }
	cudaGraphLaunch(ge, c->stream);
	if (c->profiling) { cudaEventRecord(eb, c->stream); c->recs.push_back({name, ea, eb}); }
	c->launches += nodes;
}

void colden_sweep(trg_ctx* c) {
	if (c->use_graphs && !c->g_colden)
		c->g_colden = capture_graph(c, [&] { colden_sweep_direct(c); }, c->g_colden_nodes);
	sweep_in(c);
	if (c->use_graphs && c->g_colden) launch_graph(c, c->g_colden, c->g_colden_nodes, "graph_colden_sweep");
	else colden_sweep_direct(c);
	sweep_out(c, true);
}

void thermo_pre(trg_ctx* c) {
	// Thermodynamics::preTimeStepCalculations: column densities, then rates.
	if (c->colden_join_pending) {  // the sweep ran on the side stream
		cudaStreamWaitEvent(c->stream, c->ev_cjoin, 0);
		c->colden_join_pending = false;
	}
	if (c->P.star_on && !c->colden_valid) {
		colden_sweep(c);
		c->colden_valid = true;
	}
	LAUNCH(KF(k_thermo_rates_fp64), c->P.N, 256, c->P, c->S);
}

void rad_pre(trg_ctx* c) { LAUNCH(KF(k_rad_heating_fp64), c->P.N, 256, c->P, c->S); }

void comp_pre(trg_ctx* c, int comp) {
	if (comp == COMP_RAD) rad_pre(c);
	else if (comp == COMP_THERMO) thermo_pre(c);
}

void hydro_fluxes(trg_ctx* c) {
	halo_exchange(c, c->S.Q, false);
	for (int d = 0; d < c->P.nd; ++d) LAUNCH(KF(k_faces_fp64), c->S.nfaces[d], 128, c->P, c->S, d);
}

// Single grids: the shells read their cells' own inputs in sweep order
// (S.sw_rad, refreshed by k_rad_sweep_prep at the start of the sweep).
void rad_shell_launch(trg_ctx* c, const int* cells, int count, double h, bool overlap, long long off) {
	if (c->S.sw_rad) {
		if (c->P.stats_on || c->S.harvest)
			LAUNCH_SHELL(KF(k_rad_shell_sw_diag), count, 128, overlap, c->P, c->S, cells, count, h, off);
		else if (c->S.mlp_img)
			LAUNCH_SHELL(KF(k_rad_shell_sw_ls), count, 128, overlap, c->P, c->S, cells, count, h, off);
		else
			LAUNCH_SHELL(KF(k_rad_shell_sw), count, 128, overlap, c->P, c->S, cells, count, h, off);
		return;
	}
	if (c->P.stats_on || c->S.harvest)
		LAUNCH_SHELL(KF(k_rad_shell_diag), count, 128, overlap, c->P, c->S, cells, count, h);
	else if (c->P.batch && c->S.mlp_img)
		LAUNCH_SHELL(KF(k_rad_shell_fp64_ls), count, 128, overlap, c->P, c->S, cells, count, h);
	else
		LAUNCH_SHELL(KF(k_rad_shell_fp64), count, 128, overlap, c->P, c->S, cells, count, h);
}

void rad_sweep_direct(trg_ctx* c, double h) {
	int nw = (int)c->hs.wind_cells.size();
	LAUNCH(KF(k_rad_wind_reset), nw, 128, c->P, c->S, c->d_wind, nw);
	if (c->S.sw_rad) {
		if (c->S.lstart) cudaMemsetAsync(c->S.lcand_n, 0, sizeof(unsigned), c->stream);
		LAUNCH(KF(k_rad_sweep_prep), c->S.sw_rad_n, 256, c->P, c->S, c->d_sweep_nonwind, (int)c->S.sw_rad_n, 0);
		if (c->S.lstart) {
			// learned starting iterates of the listed candidates (one tcgen05 tile per CTA)
			cudaEvent_t ea = nullptr, eb = nullptr;
			if (c->profiling) { ea = pool_event(c); eb = pool_event(c); cudaEventRecord(ea, c->stream); }
			KF(k_learned_infer)<<<INFER_CTAS, 128, mlp::INFER_SMEM, c->stream>>>(c->P, c->S,
			                                                                          c->d_sweep_nonwind, h);
			if (c->profiling) { cudaEventRecord(eb, c->stream); c->recs.push_back({"k_learned_infer", ea, eb}); }
			c->launches++;
		}
	} else if (c->P.batch && c->S.mlp_img) {
		// a batch with a network: candidates of every grid, then the network over them
		cudaMemsetAsync(c->S.lcand_n, 0, sizeof(unsigned), c->stream);
		LAUNCH(KF(k_batch_learned_prep), c->P.N, 256, c->P, c->S);
		KF(k_batch_learned_infer)<<<INFER_CTAS, 128, mlp::INFER_SMEM, c->stream>>>(c->P, c->S, h);
		c->launches++;
	}
	const auto& off = c->hs.off_nonwind;
	for (size_t s = 0; s + 1 < off.size(); ++s) {
		int count = (int)(off[s + 1] - off[s]);
		rad_shell_launch(c, c->d_sweep_nonwind + off[s], count, h, s > 0, (long long)off[s]);
	}
}

// Radiation::transferRadiation2 (Radiation.cpp:508-567): the tau-only sweep
// (one graph, like the other sweeps), then one launch over all non-wind cells.
void tau_sweep_direct(trg_ctx* c) {
	int nw = (int)c->hs.wind_cells.size();
	LAUNCH(KF(k_rad_wind_reset), nw, 128, c->P, c->S, c->d_wind, nw);
	const auto& off = c->hs.off_nonwind;
	for (size_t s = 0; s + 1 < off.size(); ++s) {
		int count = (int)(off[s + 1] - off[s]);
		LAUNCH_SHELL(KF(k_rad_tau_shell), count, 128, s > 0, c->P, c->S, c->d_sweep_nonwind + off[s], count);
	}
}

void rad_integrate2(trg_ctx* c, double h) {
	if (c->use_graphs && !c->g_tau) c->g_tau = capture_graph(c, [&] { tau_sweep_direct(c); }, c->g_tau_nodes);
	sweep_in(c);
	if (c->use_graphs && c->g_tau) launch_graph(c, c->g_tau, c->g_tau_nodes, "graph_tau_sweep");
	else tau_sweep_direct(c);
	sweep_out(c, false);
	int n = (int)c->hs.sweep_nonwind.size();
	LAUNCH(KF(k_rad_solve2), n, 128, c->P, c->S, c->d_sweep_nonwind, n, h);
}

void rad_integrate(trg_ctx* c, double h) {
	// Radiation::integrate (Radiation.cpp:58-63): transferRadiation for the
	// implicit scheme (:569-651), transferRadiation2 for the others
	if (c->P.star_on && c->P.rt_scheme != 0) {
		rad_integrate2(c, h);
		return;
	}
	if (c->P.star_on && (h == 0.5 || h == 1.0) && c->use_graphs) {
		int gi = h == 0.5 ? 0 : 1;
		if (!c->g_rad[gi]) c->g_rad[gi] = capture_graph(c, [&] { rad_sweep_direct(c, h); }, c->g_rad_nodes[gi]);
		if (c->g_rad[gi]) {
			sweep_in(c);
			launch_graph(c, c->g_rad[gi], c->g_rad_nodes[gi], "graph_rad_sweep");
			sweep_out(c, false);
			return;
		}
	}
	if (c->P.star_on) {
		sweep_in(c);
		rad_sweep_direct(c, h);
		sweep_out(c, false);
	} else {
		LAUNCH(KF(k_rad_no_star_fp64), c->P.N, 256, c->P, c->S, h);
	}
}

// Thermodynamics::integrate: every cell's sub-cycles in place, or with the
// work queue on, the cells with many sub-cycles drained by a persistent
// kernel after the in-place pass.
void thermo_integrate(trg_ctx* c, double h) {
	if (c->S.thq) cudaMemsetAsync(c->S.thq_ctl, 0, THQ_CTL * sizeof(unsigned), c->stream);
	LAUNCH(KF(k_thermo_integrate_fp64), c->P.N, 256, c->P, c->S, h);
	if (!c->S.thq) return;
	KF(k_thq_layout)<<<1, 32, 0, c->stream>>>(c->S);
	KF(k_thq_scatter)<<<148 * 4, 256, 0, c->stream>>>(c->S);
	KF(k_thq_drain)<<<148 * 8, 128, 0, c->stream>>>(c->P, c->S, h);
	c->launches += 3;
}

void sub_step(trg_ctx* c, double h, bool hasCalculatedHeatFlux, int comp, bool colden_ahead = false) {
	// Torch::subStep, Torch.cpp:352-364
	if (!hasCalculatedHeatFlux) {
		if (!c->q_fresh) q_from_u(c, 0, 1);
		c->q_fresh = false;
		comp_pre(c, comp);
	}
	switch (comp) {
	case COMP_HYDRO:
		if (c->mixed && c->P.batch) {
			// FP32 hydro pass over every grid of the batch, U into U1, then back
			cudaEvent_t ea = nullptr, eb = nullptr;
			if (c->profiling) { ea = pool_event(c); eb = pool_event(c); cudaEventRecord(ea, c->stream); }
			launch_hydro_substep_fp32_batch(c->P, c->P.batch, c->batch_tiles, h, c->stream);
			if (c->profiling) { cudaEventRecord(eb, c->stream); c->recs.push_back({"k_hydro_stage_fp32", ea, eb}); }
			c->launches += 2;
			c->q_fresh = true;
			c->colden_valid = false;
			break;
		}
		if (c->mixed) {
			// FP32 hydro pass on the FP64 state, into U1, then swap
			cudaEvent_t ea = nullptr, eb = nullptr;
			const bool fb = c->fb_contrast > 0 && c->S.fb_flag;
			if (fb) {
				// FP64 fallback, part 1: list the high-contrast cells and compute
				// their faces in FP64 from this sub-step's primitives
				cudaMemsetAsync(c->S.fb_count, 0, sizeof(unsigned), c->stream);
				{
					cudaEvent_t fa = nullptr, fbv = nullptr;
					if (c->profiling) { fa = pool_event(c); fbv = pool_event(c); cudaEventRecord(fa, c->stream); }
					const dim3 g((c->P.nx + 31) / 32, (c->P.ny + 7) / 8, (c->P.nz + FB_ZCHUNK - 1) / FB_ZCHUNK);
					KF(k_fb_flags)<<<g, 256, 0, c->stream>>>(c->P, c->S, c->fb_contrast);
					if (c->profiling) { cudaEventRecord(fbv, c->stream); c->recs.push_back({"k_fb_flags", fa, fbv}); }
					c->launches++;
				}
				LAUNCH(KF(k_fb_faces), 148LL * 8 * 128, 128, c->P, c->S);
			}
			if (c->profiling) { ea = pool_event(c); eb = pool_event(c); cudaEventRecord(ea, c->stream); }
			launch_hydro_substep_fp32(c->P, c->S, c->S.U, c->S.U1, h, c->zchunk, c->stream);
			if (c->profiling) { cudaEventRecord(eb, c->stream); c->recs.push_back({"k_hydro_stage_fp32", ea, eb}); }
			c->launches++;
			// part 2: their FP64 update overwrites the FP32 result
			if (fb) LAUNCH(KF(k_fb_update), 148LL * 8 * 256, 256, c->P, c->S, h);
			std::swap(c->S.U, c->S.U1);
			c->q_fresh = true;
			c->colden_valid = false;
			break;
		}
		hydro_fluxes(c);
		LAUNCH(KF(k_hydro_update_fp64), c->P.N, 256, c->P, c->S, h, 0, 0, 0);
		c->colden_valid = false;
		break;
	case COMP_RAD:
		if (colden_ahead) {
			// the next thermal sub-step's column densities, beside this sub-step
			cudaEventRecord(c->ev_cfork, c->stream);
			cudaStreamWaitEvent(c->side, c->ev_cfork, 0);
			std::swap(c->stream, c->side);
			colden_sweep(c);
			std::swap(c->stream, c->side);
			cudaEventRecord(c->ev_cjoin, c->side);
			c->colden_valid = true;
			c->colden_join_pending = true;
		}
		rad_integrate(c, h);
		// mode 2 (FP32 form): the update also leaves Q of the new state
		LAUNCH(KF(k_rad_update_fp64), c->P.N, 256, c->P, c->S, h, c->mixed ? 2 : 0);
		c->q_fresh = c->mixed;
		break;
	default:
		thermo_integrate(c, h);
		LAUNCH(KF(k_thermo_update_fp64), c->P.N, 256, c->P, c->S, h, c->mixed ? 2 : 0);
		c->q_fresh = c->mixed;
		break;
	}
}

void hydro_step(trg_ctx* c) {
	// Torch::hydroStep (hasCalculatedHeatFlux = true), Torch.cpp:366-387: the
	// saved state W is the untouched U; the predictor writes U1.
	c->colden_valid = false;
	hydro_fluxes(c);
	LAUNCH(KF(k_hydro_update_fp64), c->P.N, 256, c->P, c->S, 0.5, 0, 1, 0);
	q_from_u(c, 1, 0);
	hydro_fluxes(c);
	LAUNCH(KF(k_hydro_update_fp64), c->P.N, 256, c->P, c->S, 1.0, 0, 0, 0);
}

// Global FP64 mass and energy sums of the state the current step starts from
// into the per-step record: the partials come from the time-step reduction
// (fused) or, where none ran, from a pass of their own.
void cons_record(trg_ctx* c, bool fused) {
	if (!fused) {
		if (c->fp32) launch_cons_cells_f32(c->P, c->U32, c->cons_part, c->stream);
		else launch_cons_cells_f64(c->P, c->S.U, c->cons_part, c->stream);
		c->launches++;
	}
	if (c->steps < c->cons_cap) {
		launch_cons_finalize(c->P, c->cons_part, c->cons_hist + 2 * c->steps, c->stream);
		c->launches++;
	}
}

void time_step(trg_ctx* c, double dt_next) {
	// Torch::calculateTimeStep and the min with dt_next_checkpoint (Torch.cpp:304-339, :394)
	int step = c->steps < c->dt_hist_cap ? (int)c->steps : -1;
	if (c->first_time) {
		if (c->cons_on) cons_record(c, false);
		LAUNCH_SCALAR(KF(k_dt_finalize), c->P, c->S, dt_next, 1, step);
		c->first_time = 0;
		return;
	}
	long long first_cell = -1;
	if (c->P.radiation_on && c->P.star_on && c->P.K1 != 0.0 && c->rad_once_pending) {
		first_cell = c->hs.first_nonwind_cell;
		c->rad_once_pending = 0;
	}
	LAUNCH_SCALAR(KF(k_dt_reset), c->P, c->S);
	LAUNCH(KF(k_dt_reduce_fp64), c->P.N, 256, c->P, c->S, first_cell);
	if (c->cons_on) cons_record(c, true);
	dt_exchange(c);
	LAUNCH_SCALAR(KF(k_dt_finalize), c->P, c->S, dt_next, 0, step);
}

void enqueue_full_step_fp32(trg_ctx* c, double dt_next) {
	// Hydro-only Torch::fullStep in the FP32 form: dt comes from the CFL minimum
	// the previous corrector reduced (FP64), the two RK2 stages are one fused
	// kernel each.
	int step = c->steps < c->dt_hist_cap ? (int)c->steps : -1;
	if (c->cons_on) cons_record(c, false);
	if (!c->first_time) dt_exchange(c);
	LAUNCH_SCALAR(KF(k_dt_finalize), c->P, c->S, dt_next, c->first_time, step);
	c->first_time = 0;
	LAUNCH_SCALAR(KF(k_dt_reset), c->P, c->S);
	auto stage = [&](int st, const float* Uq, const float* Ub, float* Uo) {
		halo_exchange(c, Uq, true);
		cudaEvent_t ea = nullptr, eb = nullptr;
		if (c->profiling) { ea = pool_event(c); eb = pool_event(c); cudaEventRecord(ea, c->stream); }
		launch_hydro_stage_fp32(st, c->P, c->S, Uq, Ub, Uo, c->zchunk, c->stream);
		if (c->profiling) { cudaEventRecord(eb, c->stream); c->recs.push_back({"k_hydro_stage_fp32", ea, eb}); }
		c->launches++;
	};
	stage(1, c->U32, c->U32, c->U32s);
	stage(2, c->U32s, c->U32, c->U32);
	LAUNCH_SCALAR(KF(k_time_advance), c->P, c->S);
	c->steps++;
}

void enqueue_full_step(trg_ctx* c, double dt_next) {
	if (c->fp32) {
		enqueue_full_step_fp32(c, dt_next);
		return;
	}
	// Torch::fullStep, Torch.cpp:389-418
	if (!c->q_fresh) q_from_u(c, 0, 1);
	c->q_fresh = false;
	if (c->prologue_colden) {  // a slab's deferred prologue sweep (of this Q: no second sweep below)
		colden_sweep(c);
		c->prologue_colden = false;
		c->colden_valid = true;
	}
	if (c->P.cooling_on && c->P.radiation_on && c->P.star_on && c->side) {
		// Radiation::preTimeStepCalculations (heating rates, reads Q, R) beside
		// Thermodynamics::preTimeStepCalculations (column densities and rates,
		// writes T): the sweep leaves most of the GPU idle
		cudaEventRecord(c->ev_fork, c->stream);
		cudaStreamWaitEvent(c->side, c->ev_fork, 0);
		std::swap(c->stream, c->side);
		rad_pre(c);
		std::swap(c->stream, c->side);
		cudaEventRecord(c->ev_join, c->side);
		thermo_pre(c);
		cudaStreamWaitEvent(c->stream, c->ev_join, 0);
	} else {
		if (c->P.cooling_on) thermo_pre(c);
		if (c->P.radiation_on) rad_pre(c);
	}
	time_step(c, dt_next);
	const int ncomps = c->hs.nactive;
	if (ncomps == 1) {
		hydro_step(c);
	} else {
		c->stepCounter = (c->stepCounter + 1) % ncomps;
		// the symmetric split: components in the rotated order, then back
		int seq[5];
		double hs[5];
		int ns = 0;
		for (int i = 0; i < ncomps; ++i) {
			seq[ns] = c->hs.active[(i + c->stepCounter) % ncomps];
			hs[ns++] = (i == ncomps - 1) ? 1.0 : 0.5;
		}
		for (int i = ncomps - 2; i >= 0; --i) {
			seq[ns] = c->hs.active[(i + c->stepCounter) % ncomps];
			hs[ns++] = 0.5;
		}
		const bool can_overlap = c->colden_overlap && c->side && c->P.star_on && c->P.cooling_on;
		for (int k = 0; k < ns; ++k) {
			bool ahead = false;
			if (can_overlap && seq[k] == COMP_RAD && !c->colden_valid) {
				// the first thermal or hydro sub-step after this one: a thermal
				// one needs the column densities of the current density
				for (int j = k + 1; j < ns; ++j) {
					if (seq[j] == COMP_HYDRO) break;
					if (seq[j] == COMP_THERMO) {
						ahead = true;
						break;
					}
				}
			}
			sub_step(c, hs[k], k == 0, seq[k], ahead);
		}
	}
	LAUNCH_SCALAR(KF(k_time_advance), c->P, c->S);
	c->steps++;
}

int check_device_error(trg_ctx* c) {
	CUDA_TRY(cudaGetLastError());
	unsigned e = 0;
	CUDA_TRY(cudaMemcpyAsync(&e, c->S.err, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
	CUDA_TRY(cudaStreamSynchronize(c->stream));
	// checkValues runs before every integrator in the reference, so an invalid
	// state is reported ahead of the failures it causes downstream.
	if (e & ERRB_NAN) return set_error(c, TRG_ERR_NAN, "checkValues/fixSolution: invalid cell state");
	if (e & ERRB_FLUX) return set_error(c, TRG_ERR_FLUX, "Riemann solver: HII flux is NaN");
	if (e & ERRB_PICARD) return set_error(c, TRG_ERR_PICARD, "update_HIIfrac: implicit method not converging");
	if (e & ERRB_DT) return set_error(c, TRG_ERR_DT, "Radiation::calculateTimeStep: invalid timestep");
	if (e & ERRB_TC) return set_error(c, TRG_ERR_TC, "learned start: tensor-core wait expired");
	if (e & ERRB_ASYNC) return set_error(c, TRG_ERR_CUDA, "hydro pass: a TMA plane copy did not complete in time");
	if (e & ERRB_SLAB)
		return set_error(c, TRG_ERR_ARG, "slab sweep: a partition-face neighbour was read before any boundary layer "
		                                 "was exchanged");
	if (e & ERRB_SUBCYCLE)
		return set_error(c, TRG_ERR_SUBCYCLE, "Thermodynamics::integrate: a cell needs more thermal sub-cycles than "
		                                      "the work queue runs (2^26)");
	if (c->xfail) {
		c->xfail = false;
		return set_error(c, TRG_ERR_ARG, "slab exchange: the host's exchange hook reported a failure");
	}
	return TRG_OK;
}

int ensure_cons_hist(trg_ctx* c, long long needed) {
	if (!c->cons_on || needed <= c->cons_cap) return 0;
	long long cap = std::max<long long>(needed, 2LL * c->cons_cap + 1024);
	double* nh = nullptr;
	if (dalloc(c, &nh, 2 * cap)) return TRG_ERR_OOM;
	CUDA_TRY(cudaMemsetAsync(nh, 0xff, sizeof(double) * 2 * cap, c->stream));  // NaN: step not recorded
	if (c->cons_hist && c->steps > 0)
		CUDA_TRY(cudaMemcpyAsync(nh, c->cons_hist, sizeof(double) * 2 * std::min<long long>(c->steps, c->cons_cap),
		                         cudaMemcpyDeviceToDevice, c->stream));
	c->cons_hist = nh;
	c->cons_cap = cap;
	return 0;
}

int ensure_dt_hist(trg_ctx* c, long long needed) {
	if (int rc = ensure_cons_hist(c, needed)) return rc;
	if (needed <= c->dt_hist_cap) return 0;
	int cap = (int)std::max<long long>(needed, 2LL * c->dt_hist_cap + 1024);
	double* nh = nullptr;
	if (dalloc(c, &nh, cap)) return TRG_ERR_OOM;
	if (c->S.dt_hist && c->steps > 0)
		CUDA_TRY(cudaMemcpyAsync(nh, c->S.dt_hist, sizeof(double) * std::min<long long>(c->steps, c->dt_hist_cap),
		                         cudaMemcpyDeviceToDevice, c->stream));
	c->S.dt_hist = nh;
	c->dt_hist_cap = cap;
	return 0;
}

}  // namespace

namespace trg {
const Params& ctx_params(const trg_ctx* c) { return c->P; }
State ctx_state(const trg_ctx* c) { return c->S; }
int ctx_device(const trg_ctx* c) { return c->raw.device; }
int ctx_fp32_zchunk(const trg_ctx* c) {
	int sms = 148;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->raw.device);
	long long tiles = (long long)((c->P.nx + 31) / 32) * ((c->P.ny + 7) / 8);
	long long nchunks = (4LL * 2 * sms + tiles - 1) / tiles;
	if (nchunks < 1) nchunks = 1;
	int zc = (int)((c->P.nz + nchunks - 1) / nchunks);
	return zc < 16 ? 16 : zc;
}
int ctx_fail(trg_ctx* c, int code, const std::string& msg) { return set_error(c, code, msg); }
// a slab with partition faces and no exchange hook yet
// (with a star, also the buffers of the sweep exchange)
bool slab_unhooked(const trg_ctx* c) {
	const bool part = c->P.lbc[0] == BC_PARTITION || c->P.rbc[0] == BC_PARTITION;
	return part && (!c->xfn || (c->P.star_on && !c->sweep_send));
}
}  // namespace trg

extern "C" {

namespace {
int create_impl(const trg_params* p, const SlabSpec* slab, const double* den, const double* pre, const double* hii,
                const double* v0, const double* v1, const double* v2, const double* grav, trg_ctx** out) {
	if (!p || !out) return TRG_ERR_ARG;
	*out = nullptr;
	trg_ctx* c = new trg_ctx();
	c->raw = *p;
	if (p->precision != TRG_PRECISION_FP64 && p->precision != TRG_PRECISION_FP32) {
		c->err = "unknown precision";
		*out = c;
		return TRG_ERR_ARG;
	}
	std::string why = host_setup(*p, den, pre, hii, v0, v1, v2, grav, c->hs, slab);
	if (!why.empty()) {
		c->err = why;
		*out = c;
		return TRG_ERR_ARG;
	}
	*out = c;
	c->P = c->hs.P;
	// slabs with a star call the sweep hooks on the context's own stream only
	if (slab && c->P.star_on) c->colden_overlap = false;
	const long long N = c->P.N;
	CUDA_TRY(cudaSetDevice(p->device));
	CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
	CUDA_TRY(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
	CUDA_TRY(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
	CUDA_TRY(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
	CUDA_TRY(cudaEventCreateWithFlags(&c->ev_cfork, cudaEventDisableTiming));
	CUDA_TRY(cudaEventCreateWithFlags(&c->ev_cjoin, cudaEventDisableTiming));
	State& S = c->S;
	std::memset(&S, 0, sizeof(S));
	int rc = 0;
	rc |= dalloc(c, &S.U, 7 * N);
	rc |= dalloc(c, &S.Q, 7 * N);
	rc |= dalloc(c, &S.U1, 7 * N);
	rc |= dalloc(c, &S.UDOT, 7 * N);
	rc |= dalloc(c, &S.R, 6 * N);
	rc |= dalloc(c, &S.T, 4 * N);
	rc |= dalloc(c, &S.Tmin, N);
	rc |= dalloc(c, &S.ds, N);
	rc |= dalloc(c, &S.shellVol, N);
	rc |= dalloc(c, &S.err, 1);
	rc |= dalloc(c, &S.stats, TRG_NSTATS);
	rc |= dalloc(c, &S.scal, 8);
	if (c->hs.has_grav) rc |= dalloc(c, &S.grav, 3 * N);
	for (int d = 0; d < 3; ++d) {
		int n = d == 0 ? c->P.nx : (d == 1 ? c->P.ny : c->P.nz);
		S.nfaces[d] = (N / n) * (n + 1);
		if (d < c->P.nd) rc |= dalloc(c, &S.F[d], 7 * S.nfaces[d]);
	}
	rc |= dalloc(c, &c->d_tables, 1);
	rc |= dalloc(c, &c->d_sweep_all, c->hs.sweep_all.size() + 1);
	rc |= dalloc(c, &c->d_sweep_nonwind, c->hs.sweep_nonwind.size() + 1);
	rc |= dalloc(c, &c->d_wind, c->hs.wind_cells.size() + 1);
	if (rc) return rc;
	S.tables = c->d_tables;
	cudaStream_t st = c->stream;
	CUDA_TRY(cudaMemcpyAsync(S.U, c->hs.U.data(), 7 * N * sizeof(double), cudaMemcpyHostToDevice, st));
	CUDA_TRY(cudaMemcpyAsync(S.Q, c->hs.Q.data(), 7 * N * sizeof(double), cudaMemcpyHostToDevice, st));
	if ((rc = upload_rt(c, S.R, c->hs.R.data(), 6)) || (rc = upload_rt(c, S.T, c->hs.T.data(), 4))) return rc;
	CUDA_TRY(cudaMemcpyAsync(S.Tmin, c->hs.Tmin.data(), N * sizeof(double), cudaMemcpyHostToDevice, st));
	CUDA_TRY(cudaMemcpyAsync(S.ds, c->hs.ds.data(), N * sizeof(double), cudaMemcpyHostToDevice, st));
	CUDA_TRY(cudaMemcpyAsync(S.shellVol, c->hs.shellVol.data(), N * sizeof(double), cudaMemcpyHostToDevice, st));
	if (c->hs.has_grav)
		CUDA_TRY(cudaMemcpyAsync(S.grav, c->hs.grav.data(), 3 * N * sizeof(double), cudaMemcpyHostToDevice, st));
	CUDA_TRY(cudaMemsetAsync(S.UDOT, 0, 7 * N * sizeof(double), st));
	CUDA_TRY(cudaMemsetAsync(S.U1, 0, 7 * N * sizeof(double), st));
	CUDA_TRY(cudaMemsetAsync(S.err, 0, sizeof(unsigned), st));
	CUDA_TRY(cudaMemsetAsync(S.stats, 0, TRG_NSTATS * sizeof(unsigned long long), st));
	CUDA_TRY(cudaMemsetAsync(S.scal, 0, 8 * sizeof(double), st));
	CUDA_TRY(cudaMemcpyAsync(c->d_tables, &c->hs.tables, sizeof(Tables), cudaMemcpyHostToDevice, st));
	if (!c->hs.sweep_all.empty())
		CUDA_TRY(cudaMemcpyAsync(c->d_sweep_all, c->hs.sweep_all.data(), c->hs.sweep_all.size() * sizeof(int),
		                         cudaMemcpyHostToDevice, st));
	if (!c->hs.sweep_nonwind.empty())
		CUDA_TRY(cudaMemcpyAsync(c->d_sweep_nonwind, c->hs.sweep_nonwind.data(),
		                         c->hs.sweep_nonwind.size() * sizeof(int), cudaMemcpyHostToDevice, st));
	if (!c->hs.wind_cells.empty())
		CUDA_TRY(cudaMemcpyAsync(c->d_wind, c->hs.wind_cells.data(), c->hs.wind_cells.size() * sizeof(int),
		                         cudaMemcpyHostToDevice, st));
	if ((rc = ensure_dt_hist(c, 1024))) return rc;
	if (c->P.star_on) {
		// sweep-ordered own-cell inputs of the causal sweeps, with their fixed parts
		S.sw_col_n = (long long)c->hs.sweep_all.size();
		S.sw_rad_n = (long long)c->hs.sweep_nonwind.size();
		if ((rc = dalloc(c, &S.sw_col, 2 * S.sw_col_n)) || (rc = dalloc(c, &S.sw_rad, SW_RAD_ROWS * S.sw_rad_n)))
			return rc;
		LAUNCH(trg::exact::k_colden_sweep_prep, S.sw_col_n, 256, c->P, c->S, c->d_sweep_all, (int)S.sw_col_n, 1);
		LAUNCH(trg::exact::k_rad_sweep_prep, S.sw_rad_n, 256, c->P, c->S, c->d_sweep_nonwind, (int)S.sw_rad_n, 1);
	}
	if (p->precision == TRG_PRECISION_FP32 && c->hs.nactive > 1) {
		if (c->P.nd < 2) return set_error(c, TRG_ERR_ARG, "the FP32 form needs a 2-D or 3-D grid");
		c->mixed = true;
		c->fastk = 1;
		c->zchunk = ctx_fp32_zchunk(c);
		if ((rc = dalloc(c, &c->S.fb_flag, N)) || (rc = dalloc(c, &c->S.fb_list, N)) ||
		    (rc = dalloc(c, &c->S.fb_count, 1)))
			return rc;
	} else if (p->precision == TRG_PRECISION_FP32) {
		if (c->P.nd < 2) return set_error(c, TRG_ERR_ARG, "the FP32 form needs a 2-D or 3-D grid");
		c->fp32 = true;
		c->fastk = 1;
		// z chunk per CTA: about four waves of two 256-thread CTAs per SM
		c->zchunk = ctx_fp32_zchunk(c);
		if ((rc = dalloc(c, &c->U32, 7 * N)) || (rc = dalloc(c, &c->U32s, 7 * N))) return rc;
		LAUNCH(k_f64_to_f32, 7 * N, 256, c->P, S.U, c->U32);
		CUDA_TRY(cudaMemsetAsync(c->U32s, 0, 7 * N * sizeof(float), st));
	}
	// TRG_FP64_KERNELS=exact|fast, read when a context is created: the build of
	// the FP64 kernels (radiation, cooling and time step; the FP64 form's
	// hydrodynamics too) in place of the form's own (exact for the FP64 form,
	// fast for the FP32 form), to measure what each build contributes to the
	// difference between the forms
	if (const char* kb = std::getenv("TRG_FP64_KERNELS")) {
		if (!std::strcmp(kb, "exact")) c->fastk = 0;
		else if (!std::strcmp(kb, "fast")) c->fastk = 1;
	}
	// Torch::run prologue (Torch.cpp:245-264): Q from U with floors, and the
	// column-density ray trace of fillHeatingArrays (Thermodynamics.cpp:420-421).
	// A slab's sweep needs its neighbours' boundary layers, which the host's
	// hook can move only once every slab is registered: a slab runs this
	// prologue sweep at the start of its first step instead (on the same Q).
	q_from_u(c, 0, 1);
	if (c->P.star_on) {
		if (slab && (c->P.lbc[0] == BC_PARTITION || c->P.rbc[0] == BC_PARTITION)) c->prologue_colden = true;
		else colden_sweep(c);
	}
	// the host copies of the initial fields are no longer needed
	std::vector<double>().swap(c->hs.U);
	std::vector<double>().swap(c->hs.Q);
	std::vector<double>().swap(c->hs.R);
	std::vector<double>().swap(c->hs.T);
	std::vector<double>().swap(c->hs.grav);
	return check_device_error(c);
}
}  // namespace

int trg_create(const trg_params* p, const double* den, const double* pre, const double* hii, const double* v0,
               const double* v1, const double* v2, const double* grav, trg_ctx** out) {
	return create_impl(p, nullptr, den, pre, hii, v0, v1, v2, grav, out);
}

int trg_create_slab(const trg_params* p, int x0, int nx, const double* f32_scale, const double* den,
                    const double* pre, const double* hii, const double* v0, const double* v1, const double* v2,
                    const double* grav, trg_ctx** out) {
	SlabSpec sl;
	sl.x0 = x0;
	sl.nx = nx;
	if (f32_scale) {
		sl.f32_rho0 = f32_scale[0];
		sl.f32_p0 = f32_scale[1];
	}
	return create_impl(p, &sl, den, pre, hii, v0, v1, v2, grav, out);
}

int trg_slab_exchange(trg_ctx* c, trg_exchange_fn fn, void* user, void* halo_send, const void* halo_recv,
                      void* dt_buf) {
	if (!c) return TRG_ERR_ARG;
	const bool part = c->P.lbc[0] == BC_PARTITION || c->P.rbc[0] == BC_PARTITION;
	if (fn && (!dt_buf || (part && (!halo_send || !halo_recv))))
		return set_error(c, TRG_ERR_ARG, "trg_slab_exchange: the hook needs the time-step buffer and, for a slab "
		                                 "with partition faces, both halos");
	CUDA_TRY(cudaStreamSynchronize(c->stream));
	c->xfn = fn;
	c->xuser = user;
	c->xdt = static_cast<unsigned long long*>(dt_buf);
	c->S.halo_send = fn && part ? halo_send : nullptr;
	c->S.halo_recv = fn && part ? halo_recv : nullptr;
	return TRG_OK;
}

static void drop_graphs(trg_ctx* c);
int trg_slab_sweep_exchange(trg_ctx* c, void* sweep_send, const void* sweep_recv) {
	if (!c) return TRG_ERR_ARG;
	const bool part = c->P.lbc[0] == BC_PARTITION || c->P.rbc[0] == BC_PARTITION;
	if (!part || !c->P.star_on)
		return set_error(c, TRG_ERR_ARG, "trg_slab_sweep_exchange: only slabs of a run with a star exchange sweeps");
	if (!sweep_send || !sweep_recv)
		return set_error(c, TRG_ERR_ARG, "trg_slab_sweep_exchange: needs both sweep buffers");
	CUDA_TRY(cudaStreamSynchronize(c->stream));
	c->sweep_send = static_cast<double*>(sweep_send);
	c->S.sweep_recv = static_cast<const double*>(sweep_recv);
	drop_graphs(c);  // the captured sweeps hold the state by value
	return TRG_OK;
}

long long trg_slab_sweep_bytes(const trg_ctx* c) {
	if (!c) return 0;
	return 2LL * 4 * c->P.ny * c->P.nz * (long long)sizeof(double);
}

int trg_slab_star_side(const trg_ctx* c) {
	if (!c || !c->P.star_on) return 0;
	const int sx = c->raw.star_pos[0];
	return sx < c->P.x0 ? 1 : (sx > c->P.x0 + c->P.nx - 1 ? 2 : 0);
}

long long trg_slab_halo_bytes(const trg_ctx* c) {
	if (!c) return 0;
	return 4LL * 7 * c->P.ny * c->P.nz * (long long)(c->fp32 ? sizeof(float) : sizeof(double));
}

int trg_slab_partitions(const trg_ctx* c) {
	if (!c) return 0;
	return (c->P.lbc[0] == BC_PARTITION ? 1 : 0) | (c->P.rbc[0] == BC_PARTITION ? 2 : 0);
}

int trg_f32_scales(const trg_params* p, const double* den, const double* pre, const double* hii, const double* v0,
                   const double* v1, const double* v2, double* scales) {
	if (!p || !scales) return TRG_ERR_ARG;
	HostSetup hs;
	std::string why = host_setup(*p, den, pre, hii, v0, v1, v2, nullptr, hs);
	if (!why.empty()) return TRG_ERR_ARG;
	scales[0] = hs.P.f32_rho0;
	scales[1] = hs.P.f32_p0;
	return TRG_OK;
}

int trg_full_step(trg_ctx* c, double dt_next_checkpoint, double* dt_taken) {
	if (!c) return TRG_ERR_ARG;
	if (slab_unhooked(c)) return set_error(c, TRG_ERR_ARG, "a slab steps only after trg_slab_exchange (with a star, also trg_slab_sweep_exchange)");
	int rc = ensure_dt_hist(c, c->steps + 1);
	if (rc) return rc;
	enqueue_full_step(c, dt_next_checkpoint);
	if ((rc = check_device_error(c))) return rc;
	if (dt_taken) {
		CUDA_TRY(cudaMemcpy(dt_taken, c->S.scal, sizeof(double), cudaMemcpyDeviceToHost));
	}
	return TRG_OK;
}

int trg_run_steps(trg_ctx* c, int nsteps, double dt_next_checkpoint, double* dts_out) {
	if (!c || nsteps < 0) return TRG_ERR_ARG;
	if (slab_unhooked(c)) return set_error(c, TRG_ERR_ARG, "a slab steps only after trg_slab_exchange (with a star, also trg_slab_sweep_exchange)");
	long long first = c->steps;
	int rc = ensure_dt_hist(c, c->steps + nsteps);
	if (rc) return rc;
	for (int s = 0; s < nsteps; ++s) enqueue_full_step(c, dt_next_checkpoint);
	if ((rc = check_device_error(c))) return rc;
	if (dts_out && nsteps > 0)
		CUDA_TRY(cudaMemcpy(dts_out, c->S.dt_hist + first, sizeof(double) * nsteps, cudaMemcpyDeviceToHost));
	return TRG_OK;
}

int trg_enqueue_steps(trg_ctx* c, int nsteps, double dt_next_checkpoint) {
	if (!c || nsteps < 0) return TRG_ERR_ARG;
	if (slab_unhooked(c)) return set_error(c, TRG_ERR_ARG, "a slab steps only after trg_slab_exchange (with a star, also trg_slab_sweep_exchange)");
	int rc = ensure_dt_hist(c, c->steps + nsteps);
	if (rc) return rc;
	for (int s = 0; s < nsteps; ++s) enqueue_full_step(c, dt_next_checkpoint);
	CUDA_TRY(cudaGetLastError());
	return TRG_OK;
}

void* trg_stream(const trg_ctx* c) { return c ? (void*)c->stream : nullptr; }

int trg_profile_enable(trg_ctx* c, int on) {
	if (!c) return TRG_ERR_ARG;
	CUDA_TRY(cudaStreamSynchronize(c->stream));
	profile_collect(c);
	if (on && !c->profiling) c->prof_totals.clear();
	c->profiling = on != 0;
	return TRG_OK;
}

int trg_profile_read(trg_ctx* c, const char* name, double* total_ms, long long* launches) {
	if (!c || !name) return TRG_ERR_ARG;
	CUDA_TRY(cudaStreamSynchronize(c->stream));
	profile_collect(c);
	double ms = 0;
	long long n = 0;
	for (auto& t : c->prof_totals)
		if (t.first.find(name) != std::string::npos) { ms += t.second.first; n += t.second.second; }
	if (total_ms) *total_ms = ms;
	if (launches) *launches = n;
	return TRG_OK;
}

int trg_component(trg_ctx* c, int comp, int phase, double dt, double* out) {
	if (c) c->q_fresh = c->colden_valid = false;
	if (!c) return TRG_ERR_ARG;
	if (c->fp32 || c->mixed) return set_error(c, TRG_ERR_ARG, "per-component phases are provided by the FP64 form");
	if (slab_unhooked(c)) return set_error(c, TRG_ERR_ARG, "a slab steps only after trg_slab_exchange (with a star, also trg_slab_sweep_exchange)");
	if (c->prologue_colden) {  // a slab's deferred prologue sweep
		colden_sweep(c);
		c->prologue_colden = false;
	}
	// The phase kernels read dt from the device scalar: stage the caller's dt.
	CUDA_TRY(cudaMemcpyAsync(c->S.scal, &dt, sizeof(double), cudaMemcpyHostToDevice, c->stream));
	switch (phase) {
	case TRG_PHASE_PRE:
		if (comp == TRG_COMP_THERMO) thermo_pre(c);
		else if (comp == TRG_COMP_RAD) rad_pre(c);
		break;
	case TRG_PHASE_DT: {
		LAUNCH_SCALAR(KF(k_dt_reset), c->P, c->S);
		long long first_cell = -1;
		if (comp == TRG_COMP_RAD && c->P.radiation_on && c->P.star_on && c->P.K1 != 0.0 && c->rad_once_pending) {
			first_cell = c->hs.first_nonwind_cell;
			c->rad_once_pending = 0;
		}
		LAUNCH(KF(k_dt_reduce_fp64), c->P.N, 256, c->P, c->S, first_cell);
		double mins[3];
		CUDA_TRY(cudaMemcpyAsync(mins, c->S.scal + 2, sizeof(mins), cudaMemcpyDeviceToHost, c->stream));
		CUDA_TRY(cudaStreamSynchronize(c->stream));
		double v = c->P.dt_max;
		if (comp == TRG_COMP_HYDRO) v = mins[0] < v ? mins[0] : v;
		else if (comp == TRG_COMP_RAD) v = (c->P.star_on && mins[1] < v) ? mins[1] : v;
		else if (comp == TRG_COMP_THERMO) v = mins[2] < v ? mins[2] : v;
		if (out) *out = v;
		break;
	}
	case TRG_PHASE_INTEGRATE:
		if (comp == TRG_COMP_HYDRO) hydro_fluxes(c);
		else if (comp == TRG_COMP_RAD) rad_integrate(c, 1.0);
		else if (comp == TRG_COMP_THERMO) thermo_integrate(c, 1.0);
		break;
	case TRG_PHASE_SOURCES:
		if (comp == TRG_COMP_HYDRO)
			LAUNCH(KF(k_hydro_update_fp64), c->P.N, 256, c->P, c->S, 1.0, 0, 0, 1);
		else if (comp == TRG_COMP_RAD) LAUNCH(KF(k_rad_update_fp64), c->P.N, 256, c->P, c->S, 1.0, 1);
		else if (comp == TRG_COMP_THERMO) LAUNCH(KF(k_thermo_update_fp64), c->P.N, 256, c->P, c->S, 1.0, 1);
		break;
	case TRG_PHASE_Q_FROM_U:
		q_from_u(c, 0, 1);
		break;
	case TRG_PHASE_ADVANCE:
		LAUNCH(KF(k_advance_fp64), c->P.N, 256, c->P, c->S, dt);
		break;
	default:
		return set_error(c, TRG_ERR_ARG, "unknown phase");
	}
	return check_device_error(c);
}

int trg_get_state(trg_ctx* c, double* U, double* Q, double* R, double* T, double* Tmin) {
	if (!c) return TRG_ERR_ARG;
	const long long N = c->P.N;
	cudaStream_t st = c->stream;
	if (c->fp32) {
		// expose the FP32 state as FP64 (Q = QfromU without floors)
		LAUNCH(k_f32_to_f64, 7 * N, 256, c->P, c->U32, c->S.U);
		q_from_u(c, 0, 0);
	}
	if (U) CUDA_TRY(cudaMemcpyAsync(U, c->S.U, 7 * N * sizeof(double), cudaMemcpyDeviceToHost, st));
	if (Q) CUDA_TRY(cudaMemcpyAsync(Q, c->S.Q, 7 * N * sizeof(double), cudaMemcpyDeviceToHost, st));
	int rc = 0;
	if (R && (rc = download_rt(c, R, c->S.R, 6))) return rc;
	if (T && (rc = download_rt(c, T, c->S.T, 4))) return rc;
	if (Tmin) CUDA_TRY(cudaMemcpyAsync(Tmin, c->S.Tmin, N * sizeof(double), cudaMemcpyDeviceToHost, st));
	CUDA_TRY(cudaStreamSynchronize(st));
	return TRG_OK;
}

int trg_set_conserved(trg_ctx* c, const double* U) {
	if (!c || !U) return TRG_ERR_ARG;
	c->q_fresh = false;
	c->colden_valid = false;
	CUDA_TRY(cudaMemcpyAsync(c->S.U, U, 7 * c->P.N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
	if (c->fp32) LAUNCH(k_f64_to_f32, 7 * c->P.N, 256, c->P, c->S.U, c->U32);
	return TRG_OK;
}

// ---------------------------------------------------------- checkpoints
namespace {
struct CkptHeader {
	char magic[8];
	// version 2: R and T in the grouped device layout (trg_types.h)
	int version, form;  // form: 0 FP64, 1 FP32 hydro-only, 2 FP32 with radiation/cooling
	long long N;
	int nx, ny, nz, nd;
	long long steps;
	int first_time, rad_once_pending, stepCounter, q_fresh;
	double scal[8];
};
int ckpt_form(const trg_ctx* c) { return c->fp32 ? 1 : (c->mixed ? 2 : 0); }
}  // namespace

long long trg_checkpoint_bytes(const trg_ctx* c) {
	if (!c) return 0;
	const long long N = c->P.N;
	return (long long)sizeof(CkptHeader) + (7 + 7 + 6 + 4 + 1) * N * (long long)sizeof(double) +
	       (c->fp32 ? 7 * N * (long long)sizeof(float) : 0);
}

int trg_checkpoint_save(trg_ctx* c, void* buf, long long bytes) {
	if (!c || !buf || bytes < trg_checkpoint_bytes(c)) return TRG_ERR_ARG;
	CUDA_TRY(cudaStreamSynchronize(c->stream));
	CkptHeader h{};
	memcpy(h.magic, "TRGCKPT1", 8);
	h.version = 2;
	h.form = ckpt_form(c);
	h.N = c->P.N;
	h.nx = c->P.nx;
	h.ny = c->P.ny;
	h.nz = c->P.nz;
	h.nd = c->P.nd;
	h.steps = c->steps;
	h.first_time = c->first_time;
	h.rad_once_pending = c->rad_once_pending;
	h.stepCounter = c->stepCounter;
	h.q_fresh = c->q_fresh ? 1 : 0;
	CUDA_TRY(cudaMemcpy(h.scal, c->S.scal, sizeof(h.scal), cudaMemcpyDeviceToHost));
	char* p = static_cast<char*>(buf);
	memcpy(p, &h, sizeof(h));
	p += sizeof(h);
	const long long N = c->P.N;
	const std::pair<const double*, long long> arrs[] = {
	    {c->S.U, 7 * N}, {c->S.Q, 7 * N}, {c->S.R, 6 * N}, {c->S.T, 4 * N}, {c->S.Tmin, N}};
	for (auto& a : arrs) {
		CUDA_TRY(cudaMemcpy(p, a.first, a.second * sizeof(double), cudaMemcpyDeviceToHost));
		p += a.second * sizeof(double);
	}
	if (c->fp32) CUDA_TRY(cudaMemcpy(p, c->U32, 7 * N * sizeof(float), cudaMemcpyDeviceToHost));
	return TRG_OK;
}

int trg_checkpoint_load(trg_ctx* c, const void* buf, long long bytes) {
	if (!c || !buf || bytes < (long long)sizeof(CkptHeader)) return TRG_ERR_ARG;
	CkptHeader h;
	memcpy(&h, buf, sizeof(h));
	if (memcmp(h.magic, "TRGCKPT1", 8) != 0 || h.version != 2)
		return set_error(c, TRG_ERR_ARG, "trg_checkpoint_load: not a checkpoint of this library");
	// the FP64 form (0) and the FP32 form on the FP64 state (2) keep the same
	// state arrays, so either continues the other's checkpoint; the FP32
	// state of the hydro-only FP32 form (1) is its own
	const bool same_state = h.form == ckpt_form(c) || (h.form != 1 && ckpt_form(c) != 1);
	if (!same_state || h.N != c->P.N || h.nx != c->P.nx || h.ny != c->P.ny || h.nz != c->P.nz ||
	    h.nd != c->P.nd || bytes < trg_checkpoint_bytes(c))
		return set_error(c, TRG_ERR_ARG, "trg_checkpoint_load: the checkpoint is of another grid or form");
	CUDA_TRY(cudaStreamSynchronize(c->stream));
	const char* p = static_cast<const char*>(buf) + sizeof(h);
	const long long N = c->P.N;
	const std::pair<double*, long long> arrs[] = {
	    {c->S.U, 7 * N}, {c->S.Q, 7 * N}, {c->S.R, 6 * N}, {c->S.T, 4 * N}, {c->S.Tmin, N}};
	for (auto& a : arrs) {
		CUDA_TRY(cudaMemcpy(a.first, p, a.second * sizeof(double), cudaMemcpyHostToDevice));
		p += a.second * sizeof(double);
	}
	if (c->fp32) CUDA_TRY(cudaMemcpy(c->U32, p, 7 * N * sizeof(float), cudaMemcpyHostToDevice));
	CUDA_TRY(cudaMemcpy(c->S.scal, h.scal, sizeof(h.scal), cudaMemcpyHostToDevice));
	CUDA_TRY(cudaMemset(c->S.UDOT, 0, 7 * N * sizeof(double)));
	c->q_fresh = h.q_fresh != 0;
	c->colden_valid = false;
	c->prologue_colden = false;  // the restored T is the saved run's
	c->steps = h.steps;
	c->first_time = h.first_time;
	c->rad_once_pending = h.rad_once_pending;
	c->stepCounter = h.stepCounter;
	int rc = ensure_dt_hist(c, c->steps + 1);
	if (rc) return rc;
	// the sweep-ordered copy of the optical depths (the learned start's
	// candidate test) from the restored state
	if (c->S.sw_rad) {
		if (c->S.lstart) CUDA_TRY(cudaMemsetAsync(c->S.lcand_n, 0, sizeof(unsigned), c->stream));
		LAUNCH(KF(k_rad_sweep_prep), c->S.sw_rad_n, 256, c->P, c->S, c->d_sweep_nonwind, (int)c->S.sw_rad_n, 1);
	}
	CUDA_TRY(cudaDeviceSynchronize());  // the copies above went through the default stream
	return TRG_OK;
}

int trg_synchronize(trg_ctx* c) {
	if (!c) return TRG_ERR_ARG;
	CUDA_TRY(cudaStreamSynchronize(c->stream));
	return check_device_error(c);
}

double trg_time(const trg_ctx* c) {
	if (!c || !c->S.scal) return 0;
	double t = 0;
	cudaStreamSynchronize(c->stream);
	cudaMemcpy(&t, c->S.scal + 1, sizeof(double), cudaMemcpyDeviceToHost);
	return t;
}

int trg_setup_positions(const trg_params* p, double* x, double* y, double* z, double* star_xyz) {
	if (!p) return TRG_ERR_ARG;
	return setup_positions(*p, x, y, z, star_xyz).empty() ? TRG_OK : TRG_ERR_ARG;
}

double trg_dt_max(const trg_ctx* c) { return c ? c->hs.dt_max : 0; }
long trg_ncells(const trg_ctx* c) { return c ? (long)c->P.N : 0; }
static void drop_graphs(trg_ctx* c) {
	// the sweep graphs hold the kernel arguments (Params, State) by value
	if (c->g_colden) cudaGraphExecDestroy(c->g_colden);
	c->g_colden = nullptr;
	if (c->g_tau) cudaGraphExecDestroy(c->g_tau);
	c->g_tau = nullptr;
	for (auto& g : c->g_rad) {
		if (g) cudaGraphExecDestroy(g);
		g = nullptr;
	}
}

int trg_stats_enable(trg_ctx* c, int on) {
	if (!c) return TRG_ERR_ARG;
	CUDA_TRY(cudaStreamSynchronize(c->stream));
	if ((c->P.stats_on != 0) != (on != 0)) drop_graphs(c);
	c->P.stats_on = on ? 1 : 0;
	return TRG_OK;
}

int trg_stats(trg_ctx* c, unsigned long long* out, int reset) {
	if (!c || !out) return TRG_ERR_ARG;
	CUDA_TRY(cudaMemcpyAsync(out, c->S.stats, TRG_NSTATS * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
	                         c->stream));
	CUDA_TRY(cudaStreamSynchronize(c->stream));
	if (reset) {
		CUDA_TRY(cudaMemsetAsync(c->S.stats, 0, TRG_NSTATS * sizeof(unsigned long long), c->stream));
		CUDA_TRY(cudaStreamSynchronize(c->stream));
	}
	return TRG_OK;
}

int trg_fp32_tma(trg_ctx* c, int on) {
	if (!c) return TRG_ERR_ARG;
	CUDA_TRY(cudaStreamSynchronize(c->stream));
	c->P.hydro_tma = on ? 1 : 0;
	return TRG_OK;
}

int trg_thermo_queue(trg_ctx* c, int min_subcycles) {
	if (!c || min_subcycles < 0) return TRG_ERR_ARG;
	CUDA_TRY(cudaStreamSynchronize(c->stream));
	if (min_subcycles == 0) {
		c->S.thq = nullptr;
		return TRG_OK;
	}
	if (!c->thq_buf) {
		const long long N = c->P.N;
		if (dalloc(c, &c->thq_buf, N) || dalloc(c, &c->thq_sorted_buf, N) || dalloc(c, &c->thq_bin_buf, N) ||
		    dalloc(c, &c->thq_ctl_buf, THQ_CTL))
			return TRG_ERR_OOM;
	}
	c->S.thq = c->thq_buf;
	c->S.thq_sorted = c->thq_sorted_buf;
	c->S.thq_binof = c->thq_bin_buf;
	c->S.thq_ctl = c->thq_ctl_buf;
	c->S.thq_min = min_subcycles;
	return TRG_OK;
}

int trg_fp32_contrast(trg_ctx* c, double contrast) {
	if (!c || !(contrast >= 0)) return TRG_ERR_ARG;
	c->fb_contrast = contrast;
	return TRG_OK;
}

static int cons_buffers(trg_ctx* c) {
	if (!c->cons_part && dalloc(c, &c->cons_part, 4 * cons_nparts(c->P))) return TRG_ERR_OOM;
	if (!c->cons_out && dalloc(c, &c->cons_out, 2)) return TRG_ERR_OOM;
	return TRG_OK;
}

int trg_conservation_sums(trg_ctx* c, double* mass, double* energy) {
	if (!c) return TRG_ERR_ARG;
	if (int rc = cons_buffers(c)) return rc;
	if (c->fp32) launch_cons_cells_f32(c->P, c->U32, c->cons_part, c->stream);
	else launch_cons_cells_f64(c->P, c->S.U, c->cons_part, c->stream);
	launch_cons_finalize(c->P, c->cons_part, c->cons_out, c->stream);
	double h[2] = {0, 0};
	CUDA_TRY(cudaMemcpyAsync(h, c->cons_out, sizeof h, cudaMemcpyDeviceToHost, c->stream));
	CUDA_TRY(cudaStreamSynchronize(c->stream));
	CUDA_TRY(cudaGetLastError());
	if (mass) *mass = h[0];
	if (energy) *energy = h[1];
	return TRG_OK;
}

int trg_conservation_enable(trg_ctx* c, int on) {
	if (!c) return TRG_ERR_ARG;
	CUDA_TRY(cudaStreamSynchronize(c->stream));
	if (on) {
		if (int rc = cons_buffers(c)) return rc;
		c->cons_on = true;
		c->S.cons_part = c->cons_part;
		if (int rc = ensure_cons_hist(c, c->steps + 1024)) return rc;
	} else {
		c->cons_on = false;
		c->S.cons_part = nullptr;
	}
	return TRG_OK;
}

int trg_conservation_history(trg_ctx* c, double* out, long long max_entries, long long* n_entries) {
	if (!c || (max_entries > 0 && !out)) return TRG_ERR_ARG;
	const long long n = std::min<long long>(c->steps, c->cons_cap);
	const long long k = std::min<long long>(n, std::max<long long>(max_entries, 0));
	if (k > 0) CUDA_TRY(cudaMemcpyAsync(out, c->cons_hist, sizeof(double) * 2 * k, cudaMemcpyDeviceToHost, c->stream));
	CUDA_TRY(cudaStreamSynchronize(c->stream));
	if (n_entries) *n_entries = n;
	return TRG_OK;
}

int trg_heating_enable(trg_ctx* c, int on) {
	if (!c) return TRG_ERR_ARG;
	if (c->fp32) return set_error(c, TRG_ERR_ARG, "trg_heating_enable: hydro-only FP32 runs have no heating terms");
	CUDA_TRY(cudaStreamSynchronize(c->stream));
	if (on && !c->S.H) {
		if (!c->d_heat && dalloc(c, &c->d_heat, (size_t)NH * c->P.N)) return TRG_ERR_OOM;
		CUDA_TRY(cudaMemset(c->d_heat, 0, (size_t)NH * c->P.N * sizeof(double)));
		c->S.H = c->d_heat;
	} else if (!on) {
		c->S.H = nullptr;
	}
	drop_graphs(c);
	return TRG_OK;
}

int trg_heating(trg_ctx* c, double* H) {
	if (!c || !H) return TRG_ERR_ARG;
	if (!c->S.H) return set_error(c, TRG_ERR_ARG, "trg_heating: call trg_heating_enable before stepping");
	// (slabs: a collective call, its ray trace runs through the sweep exchange)
	if (slab_unhooked(c)) return set_error(c, TRG_ERR_ARG, "a slab steps only after trg_slab_exchange (with a star, also trg_slab_sweep_exchange)");
	// Thermodynamics::fillHeatingArrays: rayTrace, then the per-cell terms
	if (c->P.star_on) colden_sweep(c);
	LAUNCH(KF(k_heating_arrays_fp64), c->P.N, 256, c->P, c->S);
	int rc = check_device_error(c);
	if (rc) return rc;
	CUDA_TRY(cudaMemcpy(H, c->S.H, (size_t)NH * c->P.N * sizeof(double), cudaMemcpyDeviceToHost));
	return TRG_OK;
}

int trg_learned_start(trg_ctx* c, const trg_mlp* m) {
	if (!c) return TRG_ERR_ARG;
	CUDA_TRY(cudaStreamSynchronize(c->stream));
	if (!m) {
		c->S.mlp_img = nullptr;
		c->S.lstart = nullptr;
		drop_graphs(c);
		return TRG_OK;
	}
	int dev = -1;
	const unsigned char* src = mlp_device_image(m, &dev);
	if (dev != c->raw.device) return set_error(c, TRG_ERR_ARG, "trg_learned_start: network on another device");
	if (!c->mlp_img && dalloc(c, &c->mlp_img, mlp::IMG_INFER_BYTES)) return TRG_ERR_OOM;
	if (!c->S.sw_rad) return set_error(c, TRG_ERR_ARG, "trg_learned_start: the run has no radiation sweep");
	if (!c->lcand_buf && (dalloc(c, &c->lcand_buf, c->S.sw_rad_n) || dalloc(c, &c->lcand_n_buf, 1)))
		return TRG_ERR_OOM;
	CUDA_TRY(cudaMemcpy(c->mlp_img, src, mlp::IMG_INFER_BYTES, cudaMemcpyDeviceToDevice));
	c->S.mlp_img = c->mlp_img;
	c->S.lstart = c->S.sw_rad + SW_LSTART * c->S.sw_rad_n;
	c->S.lcand = c->lcand_buf;
	c->S.lcand_n = c->lcand_n_buf;
	drop_graphs(c);
	return TRG_OK;
}

int trg_harvest(trg_ctx* c, long capacity) {
	if (!c || capacity < 0) return TRG_ERR_ARG;
	CUDA_TRY(cudaStreamSynchronize(c->stream));
	if (c->S.harvest) {
		cudaFree(c->S.harvest);
		cudaFree(c->S.harvest_n);
	}
	c->S.harvest = nullptr;
	c->S.harvest_n = nullptr;
	c->S.harvest_cap = 0;
	if (capacity > 0) {
		CUDA_TRY(cudaMalloc(&c->S.harvest, (size_t)capacity * 8 * sizeof(float)));
		CUDA_TRY(cudaMalloc(&c->S.harvest_n, sizeof(unsigned long long)));
		CUDA_TRY(cudaMemset(c->S.harvest_n, 0, sizeof(unsigned long long)));
		c->S.harvest_cap = capacity;
	}
	drop_graphs(c);
	return TRG_OK;
}

long trg_harvest_read(trg_ctx* c, float* out, long max) {
	if (!c || !c->S.harvest) return 0;
	if (cudaStreamSynchronize(c->stream) != cudaSuccess) return -TRG_ERR_CUDA;
	unsigned long long n = 0;
	if (cudaMemcpy(&n, c->S.harvest_n, sizeof(n), cudaMemcpyDeviceToHost) != cudaSuccess) return -TRG_ERR_CUDA;
	long avail = (long)std::min<unsigned long long>(n, (unsigned long long)c->S.harvest_cap);
	long k = std::min(avail, max);
	if (out && k > 0 &&
	    cudaMemcpy(out, c->S.harvest, (size_t)k * 8 * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
		return -TRG_ERR_CUDA;
	return (long)n;
}

int trg_autotune(trg_ctx* c, int* zchunk_out, double* ms_out) {
	if (!c) return TRG_ERR_ARG;
	if (zchunk_out) *zchunk_out = 0;
	if (ms_out) *ms_out = 0;
	if (!(c->fp32 || c->mixed)) return TRG_OK;
	// The timed launches only write scratch (U32s, or U1 of the mixed form),
	// but they fold their CFL minimum into the time-step slots: save and
	// restore those and the error word around the trials.
	double scal[8];
	unsigned err = 0;
	CUDA_TRY(cudaStreamSynchronize(c->stream));
	CUDA_TRY(cudaMemcpy(scal, c->S.scal, sizeof(scal), cudaMemcpyDeviceToHost));
	CUDA_TRY(cudaMemcpy(&err, c->S.err, sizeof(err), cudaMemcpyDeviceToHost));
	std::vector<int> cand;
	const int nz = c->P.nz;
	for (int z : {4, 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256})
		if (z < nz) cand.push_back(z);
	cand.push_back(nz);
	cand.push_back(std::min(nz, ctx_fp32_zchunk(c)));
	std::sort(cand.begin(), cand.end());
	cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
	cudaEvent_t e0, e1;
	CUDA_TRY(cudaEventCreate(&e0));
	CUDA_TRY(cudaEventCreate(&e1));
	auto trial = [&](int zc) {
		if (c->fp32) launch_hydro_stage_fp32(1, c->P, c->S, c->U32, c->U32, c->U32s, zc, c->stream);
		else launch_hydro_substep_fp32(c->P, c->S, c->S.U, c->S.U1, 0.5, zc, c->stream);
	};
	// Launches before the timed ones bring the SM clock up from idle (the
	// first candidates would otherwise be timed at a lower clock than the
	// last), and every candidate is timed in two rounds, keeping its faster.
	for (int r = 0; r < 8; ++r) trial(cand.back());
	std::vector<float> cand_ms(cand.size(), 1e30f);
	for (int round = 0; round < 2; ++round)
		for (size_t i = 0; i < cand.size(); ++i) {
			trial(cand[i]);
			cudaEventRecord(e0, c->stream);
			for (int r = 0; r < 3; ++r) trial(cand[i]);
			cudaEventRecord(e1, c->stream);
			CUDA_TRY(cudaEventSynchronize(e1));
			float ms = 0;
			cudaEventElapsedTime(&ms, e0, e1);
			cand_ms[i] = std::min(cand_ms[i], ms);
		}
	int best = c->zchunk;
	float best_ms = 1e30f;
	for (size_t i = 0; i < cand.size(); ++i)
		if (cand_ms[i] < best_ms) {
			best_ms = cand_ms[i];
			best = cand[i];
		}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	CUDA_TRY(cudaMemcpy(c->S.scal, scal, sizeof(scal), cudaMemcpyHostToDevice));
	CUDA_TRY(cudaMemcpy(c->S.err, &err, sizeof(err), cudaMemcpyHostToDevice));
	CUDA_TRY(cudaGetLastError());
	c->zchunk = best;
	if (zchunk_out) *zchunk_out = best;
	if (ms_out) *ms_out = best_ms / 3.0;
	return TRG_OK;
}

int trg_fp32_tile(trg_ctx* c, int zchunk) {
	if (!c) return 0;
	if (zchunk > 0) c->zchunk = std::min(zchunk, c->P.nz);
	return c->zchunk;
}

long long trg_kernel_launches(const trg_ctx* c) { return c ? c->launches : 0; }
const char* trg_last_error(const trg_ctx* c) { return c ? c->err.c_str() : "null context"; }

void trg_destroy(trg_ctx* c) {
	if (!c) return;
	if (c->stream) cudaStreamSynchronize(c->stream);
	profile_collect(c);
	for (cudaEvent_t e : c->event_pool) cudaEventDestroy(e);
	drop_graphs(c);
	if (c->S.harvest) cudaFree(c->S.harvest);
	if (c->S.harvest_n) cudaFree(c->S.harvest_n);
	for (void* p : c->allocs) cudaFree(p);
	if (c->side) cudaStreamSynchronize(c->side);
	if (c->ev_fork) cudaEventDestroy(c->ev_fork);
	if (c->ev_join) cudaEventDestroy(c->ev_join);
	if (c->ev_cfork) cudaEventDestroy(c->ev_cfork);
	if (c->ev_cjoin) cudaEventDestroy(c->ev_cjoin);
	if (c->side) cudaStreamDestroy(c->side);
	if (c->stream) cudaStreamDestroy(c->stream);
	delete c;
}

}  // extern "C"

// ------------------------------------------------------------------ batches
struct trg_batch {
	int G = 0;
	std::vector<trg_ctx*> grids;
	trg_ctx* v = nullptr;  // the batch's own context: flags of grid 0, tables of all grids
	// One captured CUDA graph per timestep: the operator split visits the
	// components in an order that rotates with the step counter, so a step is
	// one of `ncomps` fixed launch sequences (after the first step and the
	// radiation time step's one-off first call), given whether Q and the
	// column densities are up to date when it starts.  Each is captured the
	// first time it is needed and replayed after.
	struct StepGraph {
		cudaGraphExec_t exec = nullptr;
		long long nodes = 0;
		double dt_next = 0;
		bool q_fresh1 = false, colden_valid1 = false;  // host-side state the step ends with
	};
	StepGraph step_graph[3][2][2];  // [position][Q up to date][column densities up to date]
	bool step_graphs = true;
	int ntiles = 0;  // FP32 form: CTA tiles of the batch's hydro pass
	std::vector<State> Ss;          // the grids' State copies (host), uploaded to dS
	State* dS = nullptr;
	std::vector<long long> cell_off;  // padded cell offsets of the grids
	double* lpred = nullptr;          // learned start: one prediction slot per (padded) cell
};

namespace {

template <typename T>
int upload(trg_ctx* v, T** dst, const std::vector<T>& src) {
	int rc = dalloc(v, dst, src.size() + 1);
	if (rc) return rc;
	if (!src.empty()) {
		trg_ctx* c = v;
		CUDA_TRY(cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
	}
	return TRG_OK;
}

long long round_up(long long n, long long m) { return (n + m - 1) / m * m; }

// Concatenates shell `s` of every grid (lists `lists`, offsets `offs`) into
// one batched sweep with (grid << BATCH_CELL_BITS) | cell entries.
void concat_shells(const std::vector<trg_ctx*>& grids, bool nonwind, std::vector<int>& cells,
                   std::vector<long long>& off) {
	size_t nshell = 0;
	for (auto* g : grids) nshell = std::max(nshell, (nonwind ? g->hs.off_nonwind : g->hs.off_all).size() - 1);
	off.assign(1, 0);
	for (size_t s = 0; s < nshell; ++s) {
		for (size_t gi = 0; gi < grids.size(); ++gi) {
			const auto& o = nonwind ? grids[gi]->hs.off_nonwind : grids[gi]->hs.off_all;
			const auto& l = nonwind ? grids[gi]->hs.sweep_nonwind : grids[gi]->hs.sweep_all;
			if (s + 1 >= o.size()) continue;
			for (long long k = o[s]; k < o[s + 1]; ++k) cells.push_back(((int)gi << BATCH_CELL_BITS) | l[k]);
		}
		off.push_back((long long)cells.size());
	}
}

bool same_flags(const trg_ctx* a, const trg_ctx* b) {
	const Params &p = a->P, &q = b->P;
	return p.nd == q.nd && p.geometry == q.geometry && p.order == q.order && p.riemann == q.riemann &&
	       p.limiter == q.limiter && p.radiation_on == q.radiation_on && p.cooling_on == q.cooling_on &&
	       p.star_on == q.star_on && p.collisions_on == q.collisions_on && p.coupling == q.coupling &&
	       p.thermo_subcycling == q.thermo_subcycling && (p.K1 != 0.0) == (q.K1 != 0.0) &&
	       a->hs.nactive == b->hs.nactive && a->hs.active[0] == b->hs.active[0] &&
	       a->hs.active[1] == b->hs.active[1] && a->hs.active[2] == b->hs.active[2] && a->raw.device == b->raw.device;
}

}  // namespace

extern "C" {

int trg_batch_create(trg_ctx* const* grids, int G, trg_batch** out) {
	if (!grids || !out || G < 1 || G > BATCH_MAX_GRIDS) return TRG_ERR_ARG;
	*out = nullptr;
	for (int g = 0; g < G; ++g) {
		trg_ctx* c = grids[g];
		if (!c) return TRG_ERR_ARG;
		if (c->fp32)
			return set_error(c, TRG_ERR_ARG, "trg_batch_create: batches run radiation-hydro grids (FP64 or FP32 form)");
		if (c->mixed != grids[0]->mixed)
			return set_error(c, TRG_ERR_ARG, "trg_batch_create: grids of a batch share one precision form");
		if (c->mixed && c->P.nd != 2)
			return set_error(c, TRG_ERR_ARG, "trg_batch_create: FP32-form batches take 2-D grids");
		if (c->P.N > (long long)BATCH_CELL_MASK + 1)
			return set_error(c, TRG_ERR_ARG, "trg_batch_create: a batched grid holds at most 4194304 cells");
		if (c->steps != 0 || !c->first_time)
			return set_error(c, TRG_ERR_ARG, "trg_batch_create: grids join a batch before their first step");
		if (!same_flags(grids[0], c))
			return set_error(c, TRG_ERR_ARG, "trg_batch_create: grids differ in physics flags, solver or device");
		if (c->S.mlp_img || c->S.harvest)
			return set_error(c, TRG_ERR_ARG, "trg_batch_create: no learned start or harvest in a batch");
		if (c->P.x0 != 0 || c->P.lbc[0] == BC_PARTITION || c->P.rbc[0] == BC_PARTITION)
			return set_error(c, TRG_ERR_ARG, "trg_batch_create: slabs of a decomposed grid are not batched");
	}
	trg_batch* b = new trg_batch();
	b->G = G;
	b->grids.assign(grids, grids + G);
	trg_ctx* v = new trg_ctx();
	b->v = v;
	auto bail = [&](int rc) {
		trg_batch_destroy(b);
		return rc;
	};
	trg_ctx* c = v;  // for CUDA_TRY
	v->raw = grids[0]->raw;
	CUDA_TRY(cudaSetDevice(v->raw.device));
	if (cudaStreamCreateWithFlags(&v->stream, cudaStreamNonBlocking) != cudaSuccess ||
	    cudaStreamCreateWithFlags(&v->side, cudaStreamNonBlocking) != cudaSuccess ||
	    cudaEventCreateWithFlags(&v->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
	    cudaEventCreateWithFlags(&v->ev_join, cudaEventDisableTiming) != cudaSuccess ||
	    cudaEventCreateWithFlags(&v->ev_cfork, cudaEventDisableTiming) != cudaSuccess ||
	    cudaEventCreateWithFlags(&v->ev_cjoin, cudaEventDisableTiming) != cudaSuccess)
		return bail(TRG_ERR_CUDA);
	v->P = grids[0]->P;
	v->S = grids[0]->S;
	v->hs.nactive = grids[0]->hs.nactive;
	for (int i = 0; i < 3; ++i) v->hs.active[i] = grids[0]->hs.active[i];
	v->nscalar = G;
	// batches run a build with the batch dispatch: the exact one (FP64 form)
	// or the fast one with the dispatch (FP32 form)
	v->fastk = grids[0]->mixed ? 2 : 0;
	v->mixed = grids[0]->mixed;
	v->dt_hist_cap = 0;
	// offsets of the padded cell and face ranges
	std::vector<long long> cell_off(G + 1, 0), face_off[3], first_cell(G, -1);
	for (int d = 0; d < 3; ++d) face_off[d].assign(G + 1, 0);
	v->hs.first_nonwind_cell = -1;
	for (int g = 0; g < G; ++g) {
		cell_off[g + 1] = cell_off[g] + round_up(grids[g]->P.N, 256);
		for (int d = 0; d < 3; ++d) face_off[d][g + 1] = face_off[d][g] + round_up(grids[g]->S.nfaces[d], 256);
		first_cell[g] = grids[g]->hs.first_nonwind_cell;
		if (first_cell[g] >= 0) v->hs.first_nonwind_cell = 0;
	}
	// per-grid copies; one error word and one counter block for the batch
	if (dalloc(v, &v->S.err, 1) || dalloc(v, &v->S.stats, TRG_NSTATS)) return bail(TRG_ERR_OOM);
	CUDA_TRY(cudaMemset(v->S.err, 0, sizeof(unsigned)));
	CUDA_TRY(cudaMemset(v->S.stats, 0, TRG_NSTATS * sizeof(unsigned long long)));
	std::vector<Params> Ps(G);
	std::vector<State> Ss(G);
	for (int g = 0; g < G; ++g) {
		Ps[g] = grids[g]->P;
		Ps[g].batch = nullptr;
		Ps[g].stats_on = 0;
		Ss[g] = grids[g]->S;
		Ss[g].err = v->S.err;
		Ss[g].stats = v->S.stats;
		Ss[g].cons_part = nullptr;
		Ss[g].fb_flag = nullptr;  // FP32-form batches have no FP64 fallback pass
		Ss[g].thq = nullptr;  // batches run the sub-cycles in place
	}
	// batched sweeps and wind list
	std::vector<int> wind;
	for (int g = 0; g < G; ++g)
		for (int w : grids[g]->hs.wind_cells) wind.push_back((g << BATCH_CELL_BITS) | w);
	concat_shells(b->grids, false, v->hs.sweep_all, v->hs.off_all);
	concat_shells(b->grids, true, v->hs.sweep_nonwind, v->hs.off_nonwind);
	v->hs.wind_cells = wind;
	Params* dP = nullptr;
	State* dS = nullptr;
	long long *dcell = nullptr, *dface[3] = {nullptr, nullptr, nullptr}, *dfirst = nullptr;
	BatchTable* dtab = nullptr;
	int rc = 0;
	if ((rc = upload(v, &dP, Ps)) || (rc = upload(v, &dS, Ss)) || (rc = upload(v, &dcell, cell_off)) ||
	    (rc = upload(v, &dface[0], face_off[0])) || (rc = upload(v, &dface[1], face_off[1])) ||
	    (rc = upload(v, &dface[2], face_off[2])) || (rc = upload(v, &dfirst, first_cell)) ||
	    (rc = upload(v, &v->d_sweep_all, v->hs.sweep_all)) ||
	    (rc = upload(v, &v->d_sweep_nonwind, v->hs.sweep_nonwind)) || (rc = upload(v, &v->d_wind, wind)))
		return bail(rc);
	BatchTable tab;
	tab.G = G;
	tab.P = dP;
	tab.S = dS;
	tab.cell_off = dcell;
	for (int d = 0; d < 3; ++d) tab.face_off[d] = dface[d];
	tab.first_cell = dfirst;
	tab.tiles = nullptr;
	tab.ntiles = 0;
	if (v->mixed) {
		std::vector<BatchTile> tiles;
		for (int g = 0; g < G; ++g)
			for (int ty = 0; ty < (grids[g]->P.ny + 7) / 8; ++ty)
				for (int tx = 0; tx < (grids[g]->P.nx + 31) / 32; ++tx) tiles.push_back({g, tx, ty, 0});
		BatchTile* dtiles = nullptr;
		if ((rc = upload(v, &dtiles, tiles))) return bail(rc);
		tab.tiles = dtiles;
		tab.ntiles = (int)tiles.size();
		b->ntiles = tab.ntiles;
		v->batch_tiles = tab.ntiles;
	}
	if ((rc = upload(v, &dtab, std::vector<BatchTable>(1, tab)))) return bail(rc);
	b->Ss = Ss;
	b->dS = dS;
	b->cell_off = cell_off;
	v->P.batch = dtab;
	v->P.N = cell_off[G];
	v->P.stats_on = 0;
	for (int d = 0; d < 3; ++d) v->S.nfaces[d] = face_off[d][G];
	v->S.mlp_img = nullptr;
	v->S.lstart = nullptr;
	v->S.harvest = nullptr;
	v->S.harvest_n = nullptr;
	v->S.dt_hist = nullptr;
	v->S.cons_part = nullptr;
	v->S.sw_rad = v->S.sw_col = nullptr;  // batches read each grid's cells in place
	v->S.thq = nullptr;
	v->S.sw_rad_n = v->S.sw_col_n = 0;
	*out = b;
	return TRG_OK;
}

namespace {
void batch_drop_step_graphs(trg_batch* b) {
	for (auto& a : b->step_graph)
		for (auto& bb : a)
			for (auto& g : bb) {
				if (g.exec) cudaGraphExecDestroy(g.exec);
				g = trg_batch::StepGraph();
			}
}

// One timestep of a batch: the step's captured graph when it can be replayed,
// else the launches themselves (capturing them first when the step has a
// fixed launch sequence).
void batch_step(trg_batch* b, double dt_next) {
	trg_ctx* v = b->v;
	const bool rad_once = v->P.radiation_on && v->P.star_on && v->P.K1 != 0.0 && v->rad_once_pending;
	if (!b->step_graphs || v->first_time || rad_once || v->profiling) {
		enqueue_full_step(v, dt_next);
		return;
	}
	const int n = v->hs.nactive;
	const int phase = n > 1 ? (v->stepCounter + 1) % n : 0;
	trg_batch::StepGraph& g = b->step_graph[phase][v->q_fresh ? 1 : 0][v->colden_valid ? 1 : 0];
	if (g.exec && g.dt_next == dt_next) {
		cudaGraphLaunch(g.exec, v->stream);
		if (n > 1) v->stepCounter = phase;
		v->steps++;
		v->q_fresh = g.q_fresh1;
		v->colden_valid = g.colden_valid1;
		v->launches += g.nodes;
		return;
	}
	if (g.exec) cudaGraphExecDestroy(g.exec);
	g = trg_batch::StepGraph();
	g.dt_next = dt_next;
	const bool q_fresh0 = v->q_fresh, colden_valid0 = v->colden_valid;
	// the sweeps go into the step's graph directly (not as graphs of their own)
	const bool use_graphs = v->use_graphs;
	v->use_graphs = false;
	const long long before = v->launches;
	cudaGraph_t graph = nullptr;
	bool captured = false;
	if (cudaStreamBeginCapture(v->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
		enqueue_full_step(v, dt_next);
		captured = cudaStreamEndCapture(v->stream, &graph) == cudaSuccess && graph;
	}
	v->use_graphs = use_graphs;
	if (captured && cudaGraphInstantiate(&g.exec, graph, 0) != cudaSuccess) g.exec = nullptr;
	if (graph) cudaGraphDestroy(graph);
	cudaGetLastError();
	g.nodes = v->launches - before;
	g.q_fresh1 = v->q_fresh;
	g.colden_valid1 = v->colden_valid;
	if (g.exec) {
		cudaGraphLaunch(g.exec, v->stream);  // the capture recorded the step without running it
		return;
	}
	// capture failed: run this step's launches directly; the host state the
	// capture advanced is rewound first
	g = trg_batch::StepGraph();
	b->step_graphs = false;
	v->steps--;
	v->launches = before;
	if (n > 1) v->stepCounter = (v->stepCounter + n - 1) % n;
	v->q_fresh = q_fresh0;
	v->colden_valid = colden_valid0;
	enqueue_full_step(v, dt_next);
}
}  // namespace

int trg_batch_learned_start(trg_batch* b, const trg_mlp* m) {
	if (!b) return TRG_ERR_ARG;
	trg_ctx* v = b->v;
	trg_ctx* c = v;  // for CUDA_TRY
	CUDA_TRY(cudaStreamSynchronize(v->stream));
	if (m) {
		if (!v->P.radiation_on || !v->P.star_on || v->P.rt_scheme != 0)
			return set_error(v, TRG_ERR_ARG, "trg_batch_learned_start: the grids have no implicit radiation sweep");
		int dev = -1;
		const unsigned char* src = mlp_device_image(m, &dev);
		if (dev != v->raw.device)
			return set_error(v, TRG_ERR_ARG, "trg_batch_learned_start: network on another device");
		if (!v->mlp_img && dalloc(v, &v->mlp_img, mlp::IMG_INFER_BYTES)) return TRG_ERR_OOM;
		if (!b->lpred && dalloc(v, &b->lpred, v->P.N)) return TRG_ERR_OOM;
		if (!v->lcand_buf && (dalloc(v, &v->lcand_buf, v->P.N) || dalloc(v, &v->lcand_n_buf, 1))) return TRG_ERR_OOM;
		CUDA_TRY(cudaMemcpy(v->mlp_img, src, mlp::IMG_INFER_BYTES, cudaMemcpyDeviceToDevice));
	}
	for (int g = 0; g < b->G; ++g) {
		b->Ss[g].mlp_img = m ? v->mlp_img : nullptr;
		b->Ss[g].lstart = m ? b->lpred + b->cell_off[g] : nullptr;
		b->Ss[g].lcand = m ? v->lcand_buf : nullptr;  // the batch's candidate list and count
		b->Ss[g].lcand_n = m ? v->lcand_n_buf : nullptr;
	}
	CUDA_TRY(cudaMemcpy(b->dS, b->Ss.data(), b->Ss.size() * sizeof(State), cudaMemcpyHostToDevice));
	v->S.mlp_img = m ? v->mlp_img : nullptr;
	v->S.lstart = m ? b->lpred : nullptr;
	v->S.lcand = m ? v->lcand_buf : nullptr;
	v->S.lcand_n = m ? v->lcand_n_buf : nullptr;
	batch_drop_step_graphs(b);
	drop_graphs(v);
	return TRG_OK;
}

int trg_batch_enqueue_steps(trg_batch* b, int nsteps, double dt_next_checkpoint) {
	if (!b || nsteps < 0) return TRG_ERR_ARG;
	for (int s = 0; s < nsteps; ++s) batch_step(b, dt_next_checkpoint);
	trg_ctx* c = b->v;
	CUDA_TRY(cudaGetLastError());
	return TRG_OK;
}

int trg_batch_set_conserved(trg_batch* b, int g, const double* U) {
	if (!b || g < 0 || g >= b->G || !U) return TRG_ERR_ARG;
	trg_ctx* c = b->v;
	trg_ctx* grid = b->grids[g];
	CUDA_TRY(cudaMemcpyAsync(grid->S.U, U, 7 * grid->P.N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
	c->q_fresh = false;  // the next step rebuilds Q, and the column densities, from the new state
	c->colden_valid = false;
	return TRG_OK;
}

int trg_batch_get_conserved(trg_batch* b, int g, double* U) {
	if (!b || g < 0 || g >= b->G || !U) return TRG_ERR_ARG;
	trg_ctx* c = b->v;
	trg_ctx* grid = b->grids[g];
	CUDA_TRY(cudaMemcpyAsync(U, grid->S.U, 7 * grid->P.N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
	return TRG_OK;
}

int trg_batch_step_graphs(trg_batch* b, int on) {
	if (!b) return TRG_ERR_ARG;
	trg_ctx* c = b->v;
	CUDA_TRY(cudaStreamSynchronize(c->stream));
	batch_drop_step_graphs(b);
	b->step_graphs = on != 0;
	return TRG_OK;
}

int trg_batch_run_steps(trg_batch* b, int nsteps, double dt_next_checkpoint) {
	int rc = trg_batch_enqueue_steps(b, nsteps, dt_next_checkpoint);
	if (rc) return rc;
	return check_device_error(b->v);
}

int trg_batch_synchronize(trg_batch* b) {
	if (!b) return TRG_ERR_ARG;
	return check_device_error(b->v);
}

void* trg_batch_stream(const trg_batch* b) { return b ? (void*)b->v->stream : nullptr; }
long long trg_batch_kernel_launches(const trg_batch* b) { return b ? b->v->launches : 0; }
long long trg_batch_cells(const trg_batch* b) {
	long long n = 0;
	if (b)
		for (auto* g : b->grids) n += g->P.N;
	return n;
}
const char* trg_batch_last_error(const trg_batch* b) { return b ? b->v->err.c_str() : "null batch"; }

int trg_batch_profile_enable(trg_batch* b, int on) { return b ? trg_profile_enable(b->v, on) : TRG_ERR_ARG; }
int trg_batch_profile_read(trg_batch* b, const char* name, double* total_ms, long long* launches) {
	return b ? trg_profile_read(b->v, name, total_ms, launches) : TRG_ERR_ARG;
}

void trg_batch_destroy(trg_batch* b) {
	if (!b) return;
	trg_ctx* v = b->v;
	if (v) {
		if (v->stream) cudaStreamSynchronize(v->stream);
		batch_drop_step_graphs(b);
		// the grids continue on their own from where the batch left them
		for (auto* g : b->grids) {
			g->steps = v->steps;
			g->first_time = v->first_time;
			g->rad_once_pending = v->rad_once_pending;
			g->stepCounter = v->stepCounter;
		}
		trg_destroy(v);
	}
	delete b;
}

}  // extern "C"
