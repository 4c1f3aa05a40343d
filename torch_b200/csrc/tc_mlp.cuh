// Tensor-core (tcgen05) building blocks of the learned starting iterate: a
// 5 -> 64 -> 64 -> 3 multilayer perceptron with BF16 weights and activations
// and FP32 accumulation in tensor memory (TMEM).
//
// One CTA of 128 threads owns a tile of 128 samples (thread t = sample row t,
// which is also TMEM lane t of an M = 128 accumulator).  Operands are staged
// by the threads in shared memory in the canonical K-major, no-swizzle layout
// of the tcgen05 shared-memory descriptors: 8-row x 16-byte core matrices,
// the two core matrices of one 16-element K slice LBO = 128 bytes apart and
// consecutive 8-row groups SBO = K * 2 * 8 bytes apart.  One elected thread
// issues tcgen05.mma (kind::f16, BF16 x BF16 -> FP32), commits to an mbarrier,
// and every warp reads its 32 accumulator rows back with tcgen05.ld 32x32b.
// Every wait on the mbarrier is bounded; on expiry the caller's error word gets
// ERRB_TC and the results are garbage but the kernel returns.
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

namespace trg {
namespace mlp {

constexpr int IN = 5, HID = 64, OUT = 3;
constexpr int K1 = 16;   // layer-1 K (5 inputs, zero padded)
constexpr int N3 = 16;   // layer-3 N (3 outputs, zero padded)

// Flat FP32 parameter vector (the host-visible model), offsets in floats.
constexpr int P_W1 = 0;                      // [IN][HID]
constexpr int P_B1 = P_W1 + IN * HID;        // [HID]
constexpr int P_W2 = P_B1 + HID;             // [HID][HID]  (row = input unit)
constexpr int P_B2 = P_W2 + HID * HID;       // [HID]
constexpr int P_W3 = P_B2 + HID;             // [HID][OUT]
constexpr int P_B3 = P_W3 + HID * OUT;       // [OUT]
constexpr int P_NTRAIN = P_B3 + OUT;         // trainable parameters
constexpr int P_IN_MEAN = P_NTRAIN;          // feature normalisation
constexpr int P_IN_SCALE = P_IN_MEAN + IN;
constexpr int P_OUT_MEAN = P_IN_SCALE + IN;  // target normalisation
constexpr int P_OUT_SCALE = P_OUT_MEAN + OUT;
constexpr int P_TOTAL = P_OUT_SCALE + OUT;

// BF16 operand images (bytes), each already in the core-matrix layout:
//   W1T [HID rows n][K1]   B of Z1 = X W1
//   W2T [HID rows n][HID]  B of Z2 = H1 W2
//   W3T [N3 rows n][HID]   B of Y  = H2 W3
//   W3  [HID rows n][N3]   B of dH2 = dY W3^T
//   W2  [HID rows n][HID]  B of dH1 = dZ2 W2^T
constexpr int IMG_W1T = 0;
constexpr int IMG_W2T = IMG_W1T + HID * K1 * 2;
constexpr int IMG_W3T = IMG_W2T + HID * HID * 2;
// FP32 tail: b1[64] b2[64] b3[4] in_mean[5] in_scale[5] out_mean[3] out_scale[3]
// (floats, padded to a 16-byte multiple)
constexpr int IMG_F32 = IMG_W3T + N3 * HID * 2;
constexpr int F_B1 = 0, F_B2 = 64, F_B3 = 128, F_IN_MEAN = 132, F_IN_SCALE = 137, F_OUT_MEAN = 142,
              F_OUT_SCALE = 145, F_COUNT = 148;
constexpr int IMG_INFER_BYTES = IMG_F32 + F_COUNT * 4;  // what inference needs
constexpr int IMG_W3 = IMG_INFER_BYTES;
constexpr int IMG_W2 = IMG_W3 + HID * N3 * 2;
constexpr int IMG_BYTES = IMG_W2 + HID * HID * 2;

// byte offset of element (r, k) of a K-major [rows][K] BF16 operand
__host__ __device__ __forceinline__ uint32_t kmajor_off(int r, int k, int K) {
	return (uint32_t)((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
	return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor (tcgen05): start address, LBO and SBO in
// 16-byte units, descriptor version 1 (bits 46-47), no swizzle.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, int K) {
	uint64_t d = 0;
	d |= (uint64_t)((saddr >> 4) & 0x3FFF);
	d |= (uint64_t)(128 >> 4) << 16;                 // LBO: next 8-element K chunk
	d |= (uint64_t)(((uint32_t)K * 16) >> 4) << 32;  // SBO: next 8-row group
	d |= (uint64_t)1 << 46;
	return d;
}

// Instruction descriptor, kind::f16: FP32 accumulator, BF16 A and B, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
	return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, int accumulate) {
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "setp.ne.b32 p, %4, 0;\n\t"
	    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
	    "}\n" ::"r"(tmem_d),
	    "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

// D[128 x N] (+)= A[128 x K] * B[K x N], A and B K-major in shared memory.
// Issued by one thread.
__device__ __forceinline__ void gemm_tile(uint32_t tmem_d, uint32_t a_saddr, uint32_t b_saddr, int N, int K,
                                          int accumulate) {
	const uint32_t id = idesc_bf16(128, N);
	for (int kk = 0; kk < K / 16; ++kk)
		mma_bf16(tmem_d, sdesc(a_saddr + kk * 256, K), sdesc(b_saddr + kk * 256, K), id, (accumulate || kk) ? 1 : 0);
}

__device__ __forceinline__ void commit(uint32_t bar) {
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t bar, int count) {
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t phase) {
	uint32_t ok;
	asm volatile(
	    "{\n\t.reg .pred P1;\n\t"
	    "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
	    "selp.b32 %0, 1, 0, P1;\n\t}\n"
	    : "=r"(ok)
	    : "r"(bar), "r"(phase)
	    : "memory");
	return ok != 0;
}
// Bounded wait: false after `limit` polls (each poll itself suspends for a
// hardware-defined slice), so a wait that never completes cannot hang the GPU.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase, int limit = 1 << 22) {
	for (int i = 0; i < limit; ++i)
		if (mbar_try(bar, phase)) return true;
	return false;
}

// TMEM allocation by one full warp; the base address lands in *slot.  The
// CTA then gives up its allocation permit: a CTA allocates once in its life
// (a second tcgen05.alloc after the relinquish is not allowed), so every
// kernel here runs at most one allocating tile per CTA.
__device__ __forceinline__ void tmem_alloc(uint32_t slot_saddr, int ncols) {
	asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot_saddr), "r"(ncols)
	             : "memory");
	asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, int ncols) {
	asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 accumulator columns of this thread's row (warp-collective).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
	uint32_t r[16];
	asm volatile(
	    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
	    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
	      "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
	    : "r"(taddr));
	asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
	for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// TMEM address of this warp's lane quarter at column `col`.
__device__ __forceinline__ uint32_t tmem_row_addr(uint32_t base, int col) {
	return base + ((uint32_t)((threadIdx.x >> 5) & 3) * 32u << 16) + (uint32_t)col;
}

__device__ __forceinline__ uint16_t bf16_bits(float f) {
	return __bfloat16_as_ushort(__float2bfloat16_rn(f));
}
__device__ __forceinline__ void st_bf16(unsigned char* base, uint32_t off, float v) {
	*reinterpret_cast<uint16_t*>(base + off) = bf16_bits(v);
}

// Writes one 8-element K chunk (16 bytes) of row r.
__device__ __forceinline__ void st_chunk(unsigned char* base, int r, int k0, int K, const float* v) {
	uint32_t w[4];
#pragma unroll
	for (int i = 0; i < 4; ++i) w[i] = (uint32_t)bf16_bits(v[2 * i]) | ((uint32_t)bf16_bits(v[2 * i + 1]) << 16);
	*reinterpret_cast<uint4*>(base + kmajor_off(r, k0, K)) = make_uint4(w[0], w[1], w[2], w[3]);
}

// Shared-memory footprint of infer_tile (bytes): X tile, H tile, operand
// images, mbarrier and TMEM slot.
constexpr int INFER_SM_X = 0;
constexpr int INFER_SM_H = INFER_SM_X + 128 * K1 * 2;
constexpr int INFER_SM_W = INFER_SM_H + 128 * HID * 2;
constexpr int INFER_SM_BAR = INFER_SM_W + ((IMG_INFER_BYTES + 127) / 128) * 128;
constexpr int INFER_SMEM = INFER_SM_BAR + 16;

__device__ __forceinline__ void sync_tc() {
	fence_async_smem();
	fence_before();
	__syncthreads();
	fence_after();
}

// Forward passes of 128-sample tiles by one CTA (all 128 threads,
// CTA-converged): infer_begin copies the model image (IMG_INFER_BYTES at
// `img`, 16-byte aligned) into shared memory (`sm`, INFER_SMEM bytes, 128-byte
// aligned), initialises the mbarrier and allocates 64 tensor-memory columns
// (once per CTA: the allocation gives up the CTA's allocation permit);
// infer_step runs one tile (x: this thread's 5 raw features, y: its 3 raw
// outputs; `phase` is the mbarrier phase, carried from tile to tile) and
// returns false, the same in every thread, if a tensor-core wait expired (y
// is then garbage and the CTA must stop); infer_end frees the columns.
__device__ __forceinline__ uint32_t infer_begin(unsigned char* sm, const uint4* __restrict__ img) {
	const int t = threadIdx.x;
	unsigned char* W = sm + INFER_SM_W;
	const uint32_t bar = smem_u32(sm + INFER_SM_BAR);
	const uint32_t slot = smem_u32(sm + INFER_SM_BAR + 8);
	for (int i = t; i < IMG_INFER_BYTES / 16; i += blockDim.x) reinterpret_cast<uint4*>(W)[i] = img[i];
	if (t == 0) mbar_init(bar, 1);
	if (t < 32) tmem_alloc(slot, 64);
	sync_tc();
	return *reinterpret_cast<volatile uint32_t*>(sm + INFER_SM_BAR + 8);
}

__device__ __forceinline__ bool infer_step(unsigned char* sm, uint32_t tm, uint32_t& phase, const float* x, float* y) {
	const int t = threadIdx.x;
	unsigned char* X = sm + INFER_SM_X;
	unsigned char* H = sm + INFER_SM_H;
	unsigned char* W = sm + INFER_SM_W;
	const uint32_t bar = smem_u32(sm + INFER_SM_BAR);
	const float* Fs = reinterpret_cast<const float*>(W + IMG_F32);
	float xv[8] = {0, 0, 0, 0, 0, 0, 0, 0}, zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
	for (int f = 0; f < IN; ++f) xv[f] = (x[f] - Fs[F_IN_MEAN + f]) * Fs[F_IN_SCALE + f];
	st_chunk(X, t, 0, K1, xv);
	st_chunk(X, t, 8, K1, zero);
	// the previous tile's reads of the accumulator and of X/H are done
	sync_tc();
	bool ok = true;
	// layer 1 and layer 2: Z = A W, H = relu(Z + b) into the H tile, 16
	// accumulator columns at a time (few live registers)
#pragma unroll 1
	for (int layer = 0; layer < 2; ++layer) {
		if (t == 0) {
			if (layer == 0) gemm_tile(tm, smem_u32(X), smem_u32(W + IMG_W1T), HID, K1, 0);
			else gemm_tile(tm, smem_u32(H), smem_u32(W + IMG_W2T), HID, HID, 0);
			commit(bar);
		}
		ok = mbar_wait(bar, phase) && ok;
		phase ^= 1;
		fence_after();
		const float* b = Fs + (layer == 0 ? F_B1 : F_B2);
#pragma unroll 1
		for (int c = 0; c < HID / 16; ++c) {
			float h[16];
			tmem_ld16(tmem_row_addr(tm, 16 * c), h);
#pragma unroll
			for (int j = 0; j < 16; ++j) h[j] = fmaxf(h[j] + b[16 * c + j], 0.0f);
			st_chunk(H, t, 16 * c, HID, h);
			st_chunk(H, t, 16 * c + 8, HID, h + 8);
		}
		sync_tc();
	}
	if (t == 0) {
		gemm_tile(tm, smem_u32(H), smem_u32(W + IMG_W3T), N3, HID, 0);
		commit(bar);
	}
	ok = mbar_wait(bar, phase) && ok;
	phase ^= 1;
	fence_after();
	float o[16];
	tmem_ld16(tmem_row_addr(tm, 0), o);
#pragma unroll
	for (int k = 0; k < OUT; ++k) y[k] = (o[k] + Fs[F_B3 + k]) / Fs[F_OUT_SCALE + k] + Fs[F_OUT_MEAN + k];
	fence_before();
	return __syncthreads_and(ok) != 0;
}

__device__ __forceinline__ void infer_end(uint32_t tm) {
	fence_before();
	__syncthreads();
	if (threadIdx.x < 32) tmem_dealloc(tm, 64);
}

// One tile with its own set-up and release.
__device__ __forceinline__ bool infer_tile(unsigned char* sm, const uint4* __restrict__ img, const float* x, float* y) {
	const uint32_t tm = infer_begin(sm, img);
	uint32_t phase = 0;
	const bool ok = infer_step(sm, tm, phase, x, y);
	infer_end(tm);
	return ok;
}

}  // namespace mlp
}  // namespace trg
