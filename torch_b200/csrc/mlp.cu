// Training and stand-alone inference of the learned starting iterate's
// network on the tensor cores (tcgen05), and its C ABI.
//
// A training step is three launches: k_mlp_grad (forward, loss and backward
// of 128-sample tiles, one CTA each), k_mlp_adam (the optimizer on the FP32
// master parameters) and k_mlp_pack (BF16 operand images for the next step).
//
// Per tile, with X the normalised inputs rounded to BF16 and every activation
// rounded to BF16 where it becomes a tensor-core operand:
//   Z1 = X W1 + b1, H1 = relu(Z1)                 tcgen05 M=128 N=64 K=16
//   Z2 = H1 W2 + b2, H2 = relu(Z2)                tcgen05 M=128 N=64 K=64
//   Y  = H2 W3 + b3                               tcgen05 M=128 N=16 K=64
//   dY = w (Y - T)                                (loss 1/2 sum w (Y - T)^2)
//   dZ2 = (dY W3^T) * [H2 > 0]                    tcgen05 M=128 N=64 K=16
//   dZ1 = (dZ2 W2^T) * [H1 > 0]                   tcgen05 M=128 N=64 K=64
//   [dW2 ; dW3] = [H1^T ; H2^T] [dZ2 | dY]        tcgen05 M=128 N=80 K=128
//   dW1 = X^T dZ1, db = column sums                warp reductions
// The stacked weight-gradient product puts dW2 in rows 0-63, columns 0-63 and
// dW3 in rows 64-127, columns 64-66 of one 128 x 80 accumulator.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "../../include/torch_b200.h"
#include "tc_mlp.cuh"
#include "trg_types.h"

using namespace trg;
using namespace trg::mlp;

static_assert(P_TOTAL == TRG_MLP_NPARAMS && P_NTRAIN == TRG_MLP_NTRAIN, "parameter layout");

namespace {

// ---------------------------------------------------------------- kernels
__global__ void k_mlp_pack(const float* __restrict__ P, unsigned char* __restrict__ img) {
	for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < HID * HID; i += blockDim.x * gridDim.x) {
		const int n = i / HID, k = i % HID;
		st_bf16(img + IMG_W2T, kmajor_off(n, k, HID), P[P_W2 + k * HID + n]);  // (j, i) = W2[i][j]
		st_bf16(img + IMG_W2, kmajor_off(n, k, HID), P[P_W2 + n * HID + k]);   // (i, j) = W2[i][j]
		if (i < HID * K1) {
			const int n1 = i / K1, k1 = i % K1;
			st_bf16(img + IMG_W1T, kmajor_off(n1, k1, K1), k1 < IN ? P[P_W1 + k1 * HID + n1] : 0.0f);
			st_bf16(img + IMG_W3, kmajor_off(n1, k1, K1), k1 < OUT ? P[P_W3 + n1 * OUT + k1] : 0.0f);
		}
		if (i < N3 * HID) {
			const int n3 = i / HID, k3 = i % HID;
			st_bf16(img + IMG_W3T, kmajor_off(n3, k3, HID), n3 < OUT ? P[P_W3 + k3 * OUT + n3] : 0.0f);
		}
		if (i < F_COUNT) {
			float v = 0;
			if (i < 64) v = P[P_B1 + i];
			else if (i < 128) v = P[P_B2 + i - 64];
			else if (i < 128 + OUT) v = P[P_B3 + i - 128];
			else if (i >= F_IN_MEAN && i < F_IN_MEAN + IN) v = P[P_IN_MEAN + i - F_IN_MEAN];
			else if (i >= F_IN_SCALE && i < F_IN_SCALE + IN) v = P[P_IN_SCALE + i - F_IN_SCALE];
			else if (i >= F_OUT_MEAN && i < F_OUT_MEAN + OUT) v = P[P_OUT_MEAN + i - F_OUT_MEAN];
			else if (i >= F_OUT_SCALE && i < F_OUT_SCALE + OUT) v = P[P_OUT_SCALE + i - F_OUT_SCALE];
			reinterpret_cast<float*>(img + IMG_F32)[i] = v;
		}
	}
}

__global__ void __launch_bounds__(128) k_mlp_forward(const uint4* __restrict__ img, const float* __restrict__ X,
                                                     float* __restrict__ Y, long long n, unsigned* err) {
	extern __shared__ __align__(128) unsigned char sm[];
	const long long row = (long long)blockIdx.x * 128 + threadIdx.x;
	float x[IN] = {0, 0, 0, 0, 0}, y[OUT];
	if (row < n)
		for (int f = 0; f < IN; ++f) x[f] = X[row * IN + f];
	if (!infer_tile(sm, img, x, y)) {
		if (threadIdx.x == 0) atomicOr(err, ERRB_TC);
	}
	if (row < n)
		for (int k = 0; k < OUT; ++k) Y[row * OUT + k] = y[k];
}

// shared-memory plan of k_mlp_grad (bytes)
constexpr int G_X = 0;                       // X   [128][K1]
constexpr int G_H1 = G_X + 128 * K1 * 2;     // H1  [128][64]
constexpr int G_H2 = G_H1 + 128 * HID * 2;   // H2  [128][64]
constexpr int G_DY = G_H2 + 128 * HID * 2;   // dY  [128][16]
constexpr int G_DZ2 = G_DY + 128 * N3 * 2;   // dZ2 [128][64]
constexpr int G_AT = G_DZ2 + 128 * HID * 2;  // [H1^T ; H2^T] [128][128]
constexpr int G_GB = G_AT + 128 * 128 * 2;   // [dZ2^T ; dY^T ; 0] [80][128]
constexpr int G_W = G_GB + 80 * 128 * 2;     // operand images
constexpr int G_BAR = G_W + ((IMG_BYTES + 127) / 128) * 128;
constexpr int G_SMEM = G_BAR + 16;
// TMEM columns: Z1 and dH2 at 0, Z2 and dH1 at 64, Y at 128, [dW2 ; dW3] at 144
constexpr int T_A = 0, T_B = 64, T_Y = 128, T_G = 144, T_COLS = 256;

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}
__device__ __forceinline__ float bf16r(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }
__device__ __forceinline__ float ld_bf16(const unsigned char* base, uint32_t off) {
	return __bfloat162float(__ushort_as_bfloat16(*reinterpret_cast<const uint16_t*>(base + off)));
}

__global__ void __launch_bounds__(128, 1)
    k_mlp_grad(const uint4* __restrict__ img, const float* __restrict__ rec, const int* __restrict__ order, int count,
               const float* __restrict__ ow, float* __restrict__ grad, double* __restrict__ loss, unsigned* err) {
	extern __shared__ __align__(128) unsigned char sm[];
	const int t = threadIdx.x, lane = t & 31;
	const int row = blockIdx.x * 128 + t;
	const bool valid = row < count;
	unsigned char* W = sm + G_W;
	for (int i = t; i < IMG_BYTES / 16; i += 128) reinterpret_cast<uint4*>(W)[i] = img[i];
	const float* Fg = reinterpret_cast<const float*>(reinterpret_cast<const unsigned char*>(img) + IMG_F32);
	float x[8] = {0, 0, 0, 0, 0, 0, 0, 0}, tg[OUT] = {0, 0, 0}, zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
	if (valid) {
		const float* r = rec + (long long)order[row] * 8;
#pragma unroll
		for (int f = 0; f < IN; ++f) x[f] = bf16r((r[f] - Fg[F_IN_MEAN + f]) * Fg[F_IN_SCALE + f]);
#pragma unroll
		for (int k = 0; k < OUT; ++k) tg[k] = (r[IN + k] - Fg[F_OUT_MEAN + k]) * Fg[F_OUT_SCALE + k];
	}
	st_chunk(sm + G_X, t, 0, K1, x);
	st_chunk(sm + G_X, t, 8, K1, zero);
	st_chunk(sm + G_DY, t, 8, N3, zero);
	for (int r = HID + OUT; r < 80; ++r) st_bf16(sm + G_GB, kmajor_off(r, t, 128), 0.0f);
	const uint32_t bar = smem_u32(sm + G_BAR);
	if (t == 0) mbar_init(bar, 1);
	if (t < 32) tmem_alloc(smem_u32(sm + G_BAR + 8), T_COLS);
	sync_tc();
	const uint32_t tm = *reinterpret_cast<volatile uint32_t*>(sm + G_BAR + 8);
	const float* Fs = reinterpret_cast<const float*>(W + IMG_F32);
	bool ok = true;
	uint32_t phase = 0;
	float a[HID];

	// forward, hidden layers
#pragma unroll 1
	for (int layer = 0; layer < 2; ++layer) {
		if (t == 0) {
			if (layer == 0) gemm_tile(tm + T_A, smem_u32(sm + G_X), smem_u32(W + IMG_W1T), HID, K1, 0);
			else gemm_tile(tm + T_B, smem_u32(sm + G_H1), smem_u32(W + IMG_W2T), HID, HID, 0);
			commit(bar);
		}
		ok = mbar_wait(bar, phase) && ok;
		phase ^= 1;
		fence_after();
		const int col = layer == 0 ? T_A : T_B;
#pragma unroll
		for (int c = 0; c < HID / 16; ++c) tmem_ld16(tmem_row_addr(tm, col + 16 * c), a + 16 * c);
		const float* b = Fs + (layer == 0 ? F_B1 : F_B2);
		unsigned char* Hs = sm + (layer == 0 ? G_H1 : G_H2);
#pragma unroll
		for (int j = 0; j < HID; ++j) a[j] = bf16r(fmaxf(a[j] + b[j], 0.0f));
#pragma unroll
		for (int c = 0; c < HID / 8; ++c) st_chunk(Hs, t, 8 * c, HID, a + 8 * c);
#pragma unroll
		for (int j = 0; j < HID; ++j) st_bf16(sm + G_AT, kmajor_off(layer * HID + j, t, 128), a[j]);
		sync_tc();
	}
	// output layer and loss
	if (t == 0) {
		gemm_tile(tm + T_Y, smem_u32(sm + G_H2), smem_u32(W + IMG_W3T), N3, HID, 0);
		commit(bar);
	}
	ok = mbar_wait(bar, phase) && ok;
	phase ^= 1;
	fence_after();
	float o[16], dy[8] = {0, 0, 0, 0, 0, 0, 0, 0};
	tmem_ld16(tmem_row_addr(tm, T_Y), o);
	double l = 0;
#pragma unroll
	for (int k = 0; k < OUT; ++k) {
		float e = (o[k] + Fs[F_B3 + k]) - tg[k];
		dy[k] = valid ? ow[k] * e : 0.0f;
		l += valid ? (double)ow[k] * e * e : 0.0;
	}
	l = warp_sum_d(l);
	if (lane == 0) atomicAdd(loss, l);
#pragma unroll
	for (int k = 0; k < OUT; ++k) {
		float s = warp_sum(dy[k]);
		if (lane == 0) atomicAdd(grad + P_B3 + k, s);
	}
	st_chunk(sm + G_DY, t, 0, N3, dy);
#pragma unroll
	for (int k = 0; k < OUT; ++k) st_bf16(sm + G_GB, kmajor_off(HID + k, t, 128), dy[k]);
	sync_tc();

	// dH2 = dY W3^T, dZ2 = dH2 [H2 > 0]
	if (t == 0) {
		gemm_tile(tm + T_A, smem_u32(sm + G_DY), smem_u32(W + IMG_W3), HID, N3, 0);
		commit(bar);
	}
	ok = mbar_wait(bar, phase) && ok;
	phase ^= 1;
	fence_after();
#pragma unroll
	for (int c = 0; c < HID / 16; ++c) tmem_ld16(tmem_row_addr(tm, T_A + 16 * c), a + 16 * c);
#pragma unroll
	for (int j = 0; j < HID; ++j) {
		a[j] = ld_bf16(sm + G_H2, kmajor_off(t, j, HID)) > 0.0f ? a[j] : 0.0f;
		float s = warp_sum(a[j]);
		if (lane == 0) atomicAdd(grad + P_B2 + j, s);
	}
#pragma unroll
	for (int c = 0; c < HID / 8; ++c) st_chunk(sm + G_DZ2, t, 8 * c, HID, a + 8 * c);
#pragma unroll
	for (int j = 0; j < HID; ++j) st_bf16(sm + G_GB, kmajor_off(j, t, 128), a[j]);
	sync_tc();

	// dH1 = dZ2 W2^T and the stacked weight gradients, one commit
	if (t == 0) {
		gemm_tile(tm + T_B, smem_u32(sm + G_DZ2), smem_u32(W + IMG_W2), HID, HID, 0);
		gemm_tile(tm + T_G, smem_u32(sm + G_AT), smem_u32(sm + G_GB), 80, 128, 0);
		commit(bar);
	}
	ok = mbar_wait(bar, phase) && ok;
	phase ^= 1;
	fence_after();
#pragma unroll
	for (int c = 0; c < HID / 16; ++c) tmem_ld16(tmem_row_addr(tm, T_B + 16 * c), a + 16 * c);
#pragma unroll
	for (int j = 0; j < HID; ++j) {
		float dz1 = ld_bf16(sm + G_H1, kmajor_off(t, j, HID)) > 0.0f ? a[j] : 0.0f;
		float s = warp_sum(dz1);
		if (lane == 0) atomicAdd(grad + P_B1 + j, s);
#pragma unroll
		for (int f = 0; f < IN; ++f) {
			float g = warp_sum(x[f] * dz1);
			if (lane == 0) atomicAdd(grad + P_W1 + f * HID + j, g);
		}
	}
	// row t of [dW2 ; dW3]
#pragma unroll 1
	for (int c = 0; c < 5; ++c) {
		float g[16];
		tmem_ld16(tmem_row_addr(tm, T_G + 16 * c), g);
		if (t < HID) {
			if (c < 4) {
#pragma unroll
				for (int j = 0; j < 16; ++j) atomicAdd(grad + P_W2 + t * HID + 16 * c + j, g[j]);
			}
		} else if (c == 4) {
#pragma unroll
			for (int k = 0; k < OUT; ++k) atomicAdd(grad + P_W3 + (t - HID) * OUT + k, g[k]);
		}
	}
	fence_before();
	__syncthreads();
	if (t < 32) tmem_dealloc(tm, T_COLS);
	if (!ok && t == 0) atomicOr(err, ERRB_TC);
}

__global__ void k_mlp_adam(float* __restrict__ P, float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                           float lr, float gscale, float bc1, float bc2) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= P_NTRAIN) return;
	const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
	float gi = g[i] * gscale;
	g[i] = 0.0f;
	float mi = b1 * m[i] + (1.0f - b1) * gi;
	float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
	m[i] = mi;
	v[i] = vi;
	P[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

}  // namespace

// ------------------------------------------------------------------ host
struct trg_mlp {
	int device = 0;
	cudaStream_t stream = nullptr;
	float* P = nullptr;        // P_TOTAL
	unsigned char* img = nullptr;
	float* grad = nullptr;     // P_NTRAIN
	float* m1 = nullptr;
	float* m2 = nullptr;
	double* loss = nullptr;
	unsigned* err = nullptr;
	int adam_step = 0;
	std::string msg;
};

const unsigned char* mlp_device_image(const trg_mlp* m, int* device) {
	if (device) *device = m->device;
	return m->img;
}

namespace {

int fail(trg_mlp* m, int code, const std::string& s) {
	if (m) m->msg = s;
	return code;
}

#define MLP_TRY(call)                                                                                   \
	do {                                                                                                \
		cudaError_t e_ = (call);                                                                        \
		if (e_ != cudaSuccess)                                                                          \
			return fail(m, e_ == cudaErrorMemoryAllocation ? TRG_ERR_OOM : TRG_ERR_CUDA,               \
			            std::string(#call) + ": " + cudaGetErrorString(e_));                            \
	} while (0)

int pack(trg_mlp* m) {
	k_mlp_pack<<<16, 256, 0, m->stream>>>(m->P, m->img);
	MLP_TRY(cudaGetLastError());
	return TRG_OK;
}

int check_err(trg_mlp* m) {
	unsigned e = 0;
	MLP_TRY(cudaMemcpyAsync(&e, m->err, sizeof(unsigned), cudaMemcpyDeviceToHost, m->stream));
	MLP_TRY(cudaStreamSynchronize(m->stream));
	if (e & ERRB_TC) return fail(m, TRG_ERR_TC, "tensor-core wait expired in the network kernels");
	return TRG_OK;
}

struct DevBuf {
	void* p = nullptr;
	~DevBuf() { if (p) cudaFree(p); }
};

// Summed gradient and loss of records order[0..count) into m->grad / m->loss.
int grad_pass(trg_mlp* m, const float* d_rec, const int* d_order, int count, const float* d_ow) {
	const int blocks = (count + 127) / 128;
	k_mlp_grad<<<blocks, 128, G_SMEM, m->stream>>>(reinterpret_cast<const uint4*>(m->img), d_rec, d_order, count, d_ow,
	                                               m->grad, m->loss, m->err);
	MLP_TRY(cudaGetLastError());
	return TRG_OK;
}

}  // namespace

extern "C" {

int trg_mlp_create(const float* params, int device, trg_mlp** out) {
	if (!params || !out) return TRG_ERR_ARG;
	*out = nullptr;
	trg_mlp* m = new trg_mlp();
	m->device = device;
	auto bail = [&](int rc) { trg_mlp_destroy(m); return rc; };
	if (cudaSetDevice(device) != cudaSuccess) return bail(TRG_ERR_CUDA);
	if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(TRG_ERR_CUDA);
	if (cudaMalloc(&m->P, P_TOTAL * sizeof(float)) != cudaSuccess ||
	    cudaMalloc(&m->img, IMG_BYTES + 256) != cudaSuccess ||
	    cudaMalloc(&m->grad, P_NTRAIN * sizeof(float)) != cudaSuccess ||
	    cudaMalloc(&m->m1, P_NTRAIN * sizeof(float)) != cudaSuccess ||
	    cudaMalloc(&m->m2, P_NTRAIN * sizeof(float)) != cudaSuccess ||
	    cudaMalloc(&m->loss, sizeof(double)) != cudaSuccess || cudaMalloc(&m->err, sizeof(unsigned)) != cudaSuccess)
		return bail(TRG_ERR_OOM);
	if (cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, G_SMEM) != cudaSuccess)
		return bail(TRG_ERR_CUDA);
	cudaMemsetAsync(m->grad, 0, P_NTRAIN * sizeof(float), m->stream);
	cudaMemsetAsync(m->m1, 0, P_NTRAIN * sizeof(float), m->stream);
	cudaMemsetAsync(m->m2, 0, P_NTRAIN * sizeof(float), m->stream);
	cudaMemsetAsync(m->img, 0, IMG_BYTES + 256, m->stream);
	cudaMemsetAsync(m->err, 0, sizeof(unsigned), m->stream);
	int rc = trg_mlp_set_params(m, params);
	if (rc) return bail(rc);
	*out = m;
	return TRG_OK;
}

int trg_mlp_set_params(trg_mlp* m, const float* params) {
	if (!m || !params) return TRG_ERR_ARG;
	MLP_TRY(cudaMemcpyAsync(m->P, params, P_TOTAL * sizeof(float), cudaMemcpyHostToDevice, m->stream));
	int rc = pack(m);
	if (rc) return rc;
	MLP_TRY(cudaStreamSynchronize(m->stream));
	return TRG_OK;
}

int trg_mlp_get_params(trg_mlp* m, float* params) {
	if (!m || !params) return TRG_ERR_ARG;
	MLP_TRY(cudaMemcpyAsync(params, m->P, P_TOTAL * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
	MLP_TRY(cudaStreamSynchronize(m->stream));
	return TRG_OK;
}

int trg_mlp_forward(trg_mlp* m, const float* x, long n, float* y) {
	if (!m || n < 0 || (n > 0 && (!x || !y))) return TRG_ERR_ARG;
	if (n == 0) return TRG_OK;
	DevBuf dx, dy;
	MLP_TRY(cudaMalloc(&dx.p, n * IN * sizeof(float)));
	MLP_TRY(cudaMalloc(&dy.p, n * OUT * sizeof(float)));
	MLP_TRY(cudaMemcpyAsync(dx.p, x, n * IN * sizeof(float), cudaMemcpyHostToDevice, m->stream));
	const long blocks = (n + 127) / 128;
	k_mlp_forward<<<(unsigned)blocks, 128, INFER_SMEM, m->stream>>>(reinterpret_cast<const uint4*>(m->img),
	                                                                 (const float*)dx.p, (float*)dy.p, n, m->err);
	MLP_TRY(cudaGetLastError());
	MLP_TRY(cudaMemcpyAsync(y, dy.p, n * OUT * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
	return check_err(m);
}

int trg_mlp_gradient(trg_mlp* m, const float* records, long n, const float* out_weight, float* grad, double* loss) {
	if (!m || !records || n <= 0 || n > (1L << 30) || !out_weight || !grad) return TRG_ERR_ARG;
	DevBuf drec, dord, dow;
	std::vector<int> order(n);
	std::iota(order.begin(), order.end(), 0);
	MLP_TRY(cudaMalloc(&drec.p, n * 8 * sizeof(float)));
	MLP_TRY(cudaMalloc(&dord.p, n * sizeof(int)));
	MLP_TRY(cudaMalloc(&dow.p, OUT * sizeof(float)));
	MLP_TRY(cudaMemcpyAsync(drec.p, records, n * 8 * sizeof(float), cudaMemcpyHostToDevice, m->stream));
	MLP_TRY(cudaMemcpyAsync(dord.p, order.data(), n * sizeof(int), cudaMemcpyHostToDevice, m->stream));
	MLP_TRY(cudaMemcpyAsync(dow.p, out_weight, OUT * sizeof(float), cudaMemcpyHostToDevice, m->stream));
	MLP_TRY(cudaMemsetAsync(m->grad, 0, P_NTRAIN * sizeof(float), m->stream));
	MLP_TRY(cudaMemsetAsync(m->loss, 0, sizeof(double), m->stream));
	int rc = grad_pass(m, (const float*)drec.p, (const int*)dord.p, (int)n, (const float*)dow.p);
	if (rc) return rc;
	MLP_TRY(cudaMemcpyAsync(grad, m->grad, P_NTRAIN * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
	double l = 0;
	MLP_TRY(cudaMemcpyAsync(&l, m->loss, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
	MLP_TRY(cudaMemsetAsync(m->grad, 0, P_NTRAIN * sizeof(float), m->stream));
	rc = check_err(m);
	if (loss) *loss = 0.5 * l;
	return rc;
}

int trg_mlp_train(trg_mlp* m, const float* records, long n, int epochs, int batch, float lr, unsigned seed,
                  const float* out_weight, float* loss_history) {
	if (!m || !records || n <= 0 || n > (1L << 30) || epochs < 0 || batch <= 0 || !out_weight) return TRG_ERR_ARG;
	// normalisation from the training set: (v - mean) / std, std floored
	std::vector<float> P(P_TOTAL);
	int rc = trg_mlp_get_params(m, P.data());
	if (rc) return rc;
	for (int c = 0; c < IN + OUT; ++c) {
		double s = 0, s2 = 0;
		for (long i = 0; i < n; ++i) s += records[i * 8 + c];
		double mean = s / n;
		for (long i = 0; i < n; ++i) s2 += (records[i * 8 + c] - mean) * (records[i * 8 + c] - mean);
		double sd = std::max(std::sqrt(s2 / n), 1e-3);
		if (c < IN) {
			P[P_IN_MEAN + c] = (float)mean;
			P[P_IN_SCALE + c] = (float)(1.0 / sd);
		} else {
			P[P_OUT_MEAN + c - IN] = (float)mean;
			P[P_OUT_SCALE + c - IN] = (float)(1.0 / sd);
		}
	}
	if ((rc = trg_mlp_set_params(m, P.data()))) return rc;
	DevBuf drec, dord, dow;
	MLP_TRY(cudaMalloc(&drec.p, n * 8 * sizeof(float)));
	MLP_TRY(cudaMalloc(&dord.p, n * sizeof(int)));
	MLP_TRY(cudaMalloc(&dow.p, OUT * sizeof(float)));
	MLP_TRY(cudaMemcpyAsync(drec.p, records, n * 8 * sizeof(float), cudaMemcpyHostToDevice, m->stream));
	MLP_TRY(cudaMemcpyAsync(dow.p, out_weight, OUT * sizeof(float), cudaMemcpyHostToDevice, m->stream));
	std::vector<int> order(n);
	std::iota(order.begin(), order.end(), 0);
	std::mt19937 rng(seed);
	const float wsum = out_weight[0] + out_weight[1] + out_weight[2];
	for (int e = 0; e < epochs; ++e) {
		std::shuffle(order.begin(), order.end(), rng);
		MLP_TRY(cudaMemcpyAsync(dord.p, order.data(), n * sizeof(int), cudaMemcpyHostToDevice, m->stream));
		MLP_TRY(cudaMemsetAsync(m->loss, 0, sizeof(double), m->stream));
		for (long b0 = 0; b0 < n; b0 += batch) {
			const int cnt = (int)std::min<long>(batch, n - b0);
			if ((rc = grad_pass(m, (const float*)drec.p, (const int*)dord.p + b0, cnt, (const float*)dow.p))) return rc;
			++m->adam_step;
			const float bc1 = 1.0f - std::pow(0.9f, (float)m->adam_step);
			const float bc2 = 1.0f - std::pow(0.999f, (float)m->adam_step);
			k_mlp_adam<<<(P_NTRAIN + 255) / 256, 256, 0, m->stream>>>(m->P, m->grad, m->m1, m->m2, lr, 1.0f / cnt, bc1,
			                                                          bc2);
			MLP_TRY(cudaGetLastError());
			if ((rc = pack(m))) return rc;
		}
		if (loss_history) {
			double l = 0;
			MLP_TRY(cudaMemcpyAsync(&l, m->loss, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
			MLP_TRY(cudaStreamSynchronize(m->stream));
			loss_history[e] = (float)(l / ((double)n * wsum));
		}
	}
	return check_err(m);
}

const char* trg_mlp_last_error(const trg_mlp* m) { return m ? m->msg.c_str() : "null network"; }

void trg_mlp_destroy(trg_mlp* m) {
	if (!m) return;
	if (m->stream) cudaStreamSynchronize(m->stream);
	for (void* p : {(void*)m->P, (void*)m->img, (void*)m->grad, (void*)m->m1, (void*)m->m2, (void*)m->loss,
	                (void*)m->err})
		if (p) cudaFree(p);
	if (m->stream) cudaStreamDestroy(m->stream);
	delete m;
}

}  // extern "C"
