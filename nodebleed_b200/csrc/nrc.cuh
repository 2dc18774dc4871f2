// Neural radiance cache MLP (sm_100a): 64 inputs, 5 hidden layers of 64
// ReLU units, 3 linear outputs, no biases; BF16 operands on the tensor cores
// with FP32 accumulation, FP32 master weights updated by Adam.
//
// Weights of layer l are stored [out][in] (row-major); the backward pass
// reads a transposed copy [in][out].  The output layer has 3 outputs padded
// to 8 (forward) / 16 (transposed copy) with zero rows.
//
// Inference and the forward/backward pass of training run on the tcgen05
// tensor cores: 128-row tiles in shared memory (128-byte swizzled K-major
// operands), FP32 accumulators in TMEM; one thread issues a layer's UMMAs
// and the tile's 128 threads (one row each) turn the accumulator into the
// next layer's operand (in inference, four such tile pipelines per SM
// overlap one another).  The weight gradients dW_l = dz_l^T act_l are
// split-K UMMAs over the batch (M = N = 64, the batch rows as K, both
// operands MN-major).

#ifndef NB_NRC_CUH
#define NB_NRC_CUH

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace nb {

constexpr int kMlpIn = 64;
constexpr int kMlpHidden = 64;
constexpr int kMlpSquare = 5;              // 64x64 matrices
constexpr int kMlpOutPad = 8;              // output rows in the fwd copy
constexpr int kMlpOutPadT = 16;            // output cols in the bwd copy
constexpr int kMlpSq = kMlpHidden * kMlpHidden;
// parameter offsets (elements) of the FP32 master / forward BF16 copy
constexpr int kMlpParams = kMlpSquare * kMlpSq + kMlpOutPad * kMlpHidden;
// transposed BF16 copy: 5 square + [64][16]
constexpr int kMlpParamsT = kMlpSquare * kMlpSq + kMlpHidden * kMlpOutPadT;

// --------------------------------------------------------------- helpers --


__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
	__nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
	return *reinterpret_cast<uint32_t *>(&v);
}










// ------------------------------------------------------------- encoding --

// Multiresolution hash grid of the position (Mueller, Evans, Schied and
// Keller, "Instant Neural Graphics Primitives with a Multiresolution Hash
// Encoding", SIGGRAPH 2022): kGridLevels levels of kGridT entries of two
// trainable FP32 features.  Level l lays a lattice of grid_res(l) cells per
// axis over the unit box (16 to 1024, growing by 2^(6/7)); its corners are
// indexed densely where all (res + 1)^3 of them fit the level's table and
// by a spatial hash otherwise (the primes of Teschner et al. 2003), and a
// position's two features are the trilinear blend of its cell's 8 corners.
// The coarse levels carry smooth variation, the fine ones the detail a
// sin/cos encoding of the whole scene box cannot resolve.
constexpr int kGridLevels = 8;
constexpr uint32_t kGridT = 1u << 17;
constexpr int kGridParams = kGridLevels * (int)kGridT * 2;

__host__ __device__ constexpr uint32_t grid_res(int l)
{
	return l == 0 ? 16u : l == 1 ? 28u : l == 2 ? 52u : l == 3 ? 95u :
	  l == 4 ? 172u : l == 5 ? 312u : l == 6 ? 565u : 1024u;
}

// Entry (float2 index) of lattice corner (x, y, z) of level l; scenes of a
// batch after the first hash with their own code, so they do not share
// entries by design (they may collide, as hashed corners do).
__host__ __device__ __forceinline__ uint32_t grid_index(int l, uint32_t x,
                                                        uint32_t y, uint32_t z,
                                                        uint32_t scene)
{
	uint32_t r1 = grid_res(l) + 1u;
	uint32_t i;
	if (scene == 0u && r1 * r1 * r1 <= kGridT)
		i = x + r1 * (y + r1 * z);
	else
		i = x ^ (y * 2654435761u) ^ (z * 805459861u) ^ (scene * 0x9e3779b9u);
	return (i & (kGridT - 1u)) + (uint32_t)l * kGridT;
}

// Cell and in-cell position of x (in [0,1]) on level l.
__device__ __forceinline__ void grid_cell(int l, float x, uint32_t *c,
                                          float *w)
{
	uint32_t res = grid_res(l);
	float p = __fmul_rn(x, (float)res);
	uint32_t ci = min((uint32_t)p, res - 1u);
	*c = ci;
	*w = __fsub_rn(p, (float)ci);
}

// Trilinear weight of corner b (bit a: upper corner on axis a).
__device__ __forceinline__ float grid_weight(int b, const float w[3])
{
	float wx = (b & 1) ? w[0] : __fsub_rn(1.0f, w[0]);
	float wy = (b & 2) ? w[1] : __fsub_rn(1.0f, w[1]);
	float wz = (b & 4) ? w[2] : __fsub_rn(1.0f, w[2]);
	return __fmul_rn(__fmul_rn(wx, wy), wz);
}

// The two features of level l at position x (unit box).
__device__ __forceinline__ float2 grid_level(const float2 *__restrict__ g,
                                             const float x[3], uint32_t scene,
                                             int l)
{
	uint32_t c[3];
	float w[3];
#pragma unroll
	for (int a = 0; a < 3; a++)
		grid_cell(l, x[a], &c[a], &w[a]);
	float f0 = 0.0f, f1 = 0.0f;
#pragma unroll
	for (int b = 0; b < 8; b++) {
		float2 v = __ldg(g + grid_index(l, c[0] + (b & 1),
		  c[1] + ((b >> 1) & 1), c[2] + ((b >> 2) & 1), scene));
		float wt = grid_weight(b, w);
		f0 = __fmaf_rn(wt, v.x, f0);
		f1 = __fmaf_rn(wt, v.y, f1);
	}
	return make_float2(f0, f1);
}

// The 2 kGridLevels grid features of position x (unit box).
__device__ __forceinline__ void grid_features(const float2 *__restrict__ g,
                                              const float x[3],
                                              uint32_t scene, float *f)
{
#pragma unroll
	for (int l = 0; l < kGridLevels; l++) {
		float2 v = grid_level(g, x, scene, l);
		f[2 * l] = v.x;
		f[2 * l + 1] = v.y;
	}
}

// Raw cache inputs (12 floats: world position, outgoing direction, shading
// normal, albedo) -> 64 BF16 features:
//   0..15  hash grid of the position in the scene box (level l: 2l, 2l+1;
//          zero without a grid)
//   16..33 the same position, per axis sin/cos(2^k pi x), k = 0..2
//   34..41 direction (theta/pi, phi/2pi), sin/cos(2^k pi u), k = 0..1
//   42..44 (normal + 1) / 2,  45..47 albedo,  48..63 zero (in a batch of
//   scenes: one of 50..63 is 1, telling scenes 2..15 apart, see nrc_encode)
struct NrcBox {
	float lo[3], inv[3]; // position -> [0,1]^3
};

// Position in the unit box and scene index of a raw input: the frame's
// entries hold positions already mapped into their scene's box (k_shade),
// with the scene's feature code 2 k (k = 1..14, 0 for the first scene of a
// batch and for single-scene contexts) added to x; `scene_code` decodes it
// (the box is then the identity).
__device__ __forceinline__ uint32_t nrc_position(const float *in,
                                                 const NrcBox &B,
                                                 bool scene_code, float x[3])
{
	float px = in[0];
	uint32_t scene = 0u;
	if (scene_code) {
		int k = (int)floorf(px * 0.5f);
		if (k >= 1 && k <= 14) {
			px = px - (float)(2 * k);
			scene = (uint32_t)k;
		}
	}
#pragma unroll
	for (int a = 0; a < 3; a++)
		x[a] = fminf(fmaxf(((a == 0 ? px : in[a]) - B.lo[a]) * B.inv[a],
		  0.0f), 1.0f);
	return scene;
}

// grid: the hash grid's FP32 table (kGridParams floats), or null.
__device__ __forceinline__ void nrc_encode(const float *in, const NrcBox &B,
                                           uint4 *out, bool scene_code = false,
                                           const float2 *grid = nullptr)
{
	float f[64];
#pragma unroll
	for (int i = 0; i < 64; i++)
		f[i] = 0.0f;
	float x[3];
	uint32_t scene = nrc_position(in, B, scene_code, x);
	// constant indices only, so f stays in registers
#pragma unroll
	for (uint32_t k = 1; k <= 14; k++)
		f[49 + k] = scene == k ? 1.0f : 0.0f;
	if (grid)
		grid_features(grid, x, scene, f);
#pragma unroll
	for (int a = 0; a < 3; a++) {
#pragma unroll
		for (int k = 0; k < 3; k++) {
			float s, c;
			// sin/cos(2^k pi x) = sin/cos(2 pi * frac(x 2^(k-1)))
			float u = x[a] * ldexpf(1.0f, k - 1);
			u = u - floorf(u);
			sincospif(2.0f * u, &s, &c);
			f[16 + a * 6 + 2 * k] = s;
			f[16 + a * 6 + 2 * k + 1] = c;
		}
	}
	float dz = fminf(fmaxf(in[5], -1.0f), 1.0f);
	float th = acosf(dz) * 0.318309886f;
	float ph = atan2f(in[4], in[3]) * 0.159154943f + 0.5f;
	float ang[2] = {th, ph};
#pragma unroll
	for (int j = 0; j < 2; j++)
#pragma unroll
		for (int k = 0; k < 2; k++) {
			float s, c;
			sincospif(ldexpf(1.0f, k) * ang[j], &s, &c);
			f[34 + j * 4 + 2 * k] = s;
			f[34 + j * 4 + 2 * k + 1] = c;
		}
#pragma unroll
	for (int a = 0; a < 3; a++) {
		f[42 + a] = 0.5f * (in[6 + a] + 1.0f);
		f[45 + a] = in[9 + a];
	}
#pragma unroll
	for (int i = 0; i < 64; i += 8) {
		uint4 v;
		v.x = pack_bf16(f[i], f[i + 1]);
		v.y = pack_bf16(f[i + 2], f[i + 3]);
		v.z = pack_bf16(f[i + 4], f[i + 5]);
		v.w = pack_bf16(f[i + 6], f[i + 7]);
		out[i / 8] = v;
	}
}

// -------------------------------------------- inference (tcgen05 / UMMA) --
//
// 128-row tiles.  Operands in shared memory in the K-major 128-byte
// swizzled layout of the UMMA descriptors: a row of 64 BF16 is 128 bytes,
// 8-row groups are 1024-byte atoms (stride byte offset) whose 16-byte
// chunks are XOR-permuted by the row within the atom, so the tensor core
// and the row-per-thread epilogue both read and write without bank
// conflicts; a K-step of 16 advances the descriptor by 32 bytes.  One
// thread issues tcgen05.mma (kind::f16, BF16 in, FP32 accumulate, M = 128,
// N = 64, 4 K-steps of 16) into a 64-column TMEM accumulator and commits to
// an mbarrier; the 4 warps read their 32 TMEM lanes (one row per thread),
// apply ReLU, round to BF16 and write the next layer's A tile.  Every wait
// on the mbarrier is bounded: on a timeout the kernel raises *err, stops
// issuing and still frees its TMEM.

constexpr int kTcRows = 128;                 // rows per tile (UMMA M)
constexpr int kTcTile = kTcRows * 64;        // bf16 elements of a tile
constexpr int kTcW = 5 * 64 * 64 + 16 * 64;  // weights, output layer as 16 rows
// mbarrier wait limit in SM clock cycles (about 1.1 s at 1965 MHz): a poll
// (mbarrier.try_wait) suspends the thread for about 7,800 cycles on B200,
// so the limit is set in time, not in polls
constexpr long long kTcWaitCycles = 1ll << 31;
constexpr int kTcGroups = 4;                 // tile pipelines per CTA
constexpr int kTcThreads = 128 * kTcGroups;  // 4 warps per pipeline
constexpr int kTcCols = 64 * kTcGroups;      // TMEM columns of a CTA

// Byte offset of element (row, k) of a K-major [rows][64] bf16 operand in
// the 128-byte swizzled layout (operand base 1024-byte aligned).
__device__ __forceinline__ uint32_t tc_off(uint32_t row, uint32_t k)
{
	return (row >> 3) * 1024u + (row & 7u) * 128u +
	  (((k >> 3) ^ row) & 7u) * 16u + (k & 7u) * 2u;
}

// Shared-memory matrix descriptor (sm_100 UMMA): start address, leading
// byte offset (unused by swizzled K-major layouts, 16 bytes), stride byte
// offset 1024 (16-byte units), version 1, layout type 2 (128-byte swizzle).
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr)
{
	uint64_t d = 0;
	d |= (uint64_t)((saddr >> 4) & 0x3fffu);
	d |= (uint64_t)1u << 16;
	d |= (uint64_t)((1024u >> 4) & 0x3fffu) << 32;
	d |= (uint64_t)1u << 46;
	d |= (uint64_t)2u << 61;
	return d;
}

// Instruction descriptor: F32 accumulate, BF16 A and B, both K-major,
// N = n, M = 128.
__device__ __forceinline__ uint32_t tc_idesc(uint32_t n)
{
	return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) |
	  ((uint32_t)(kTcRows >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t da,
                                       uint64_t db, uint32_t idesc,
                                       uint32_t accumulate)
{
	asm volatile(
	  "{\n\t.reg .pred p;\n\t"
	  "setp.ne.b32 p, %4, 0;\n\t"
	  "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
	  :: "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void tc_commit(uint32_t bar)
{
	asm volatile(
	  "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64"
	  " [%0];" :: "r"(bar) : "memory");
}

// Wait for the mbarrier phase `parity` for at most `limit` SM clock cycles
// (the kernels use kTcWaitCycles); false on a timeout.
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity,
                                        long long limit = kTcWaitCycles)
{
	const long long t0 = clock64();
	for (;;) {
		uint32_t done;
		asm volatile(
		  "{\n\t.reg .pred p;\n\t"
		  "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		  "selp.u32 %0, 1, 0, p;\n\t}\n"
		  : "=r"(done) : "r"(bar), "r"(parity) : "memory");
		if (done)
			return true;
		if (clock64() - t0 > limit)
			return false;
	}
}

// 64 consecutive FP32 accumulator columns of this thread's TMEM lane
// (raw bits); waits for the load.
__device__ __forceinline__ void tc_ld64(uint32_t taddr, uint32_t *r)
{
	asm volatile(
	  "tcgen05.ld.sync.aligned.32x32b.x64.b32 "
	  "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
	  "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32,%33,%34,%35,"
	  "%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,%48,%49,%50,%51,%52,"
	  "%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63},"
	  " [%64];"
	  : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
	    "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]),
	    "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
	    "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
	    "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
	    "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
	    "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]),
	    "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]),
	    "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]),
	    "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]), "=r"(r[50]),
	    "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
	    "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]),
	    "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
	  : "r"(taddr));
	asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 4 consecutive FP32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tc_ld4(uint32_t taddr, float *v)
{
	uint32_t r[4];
	asm volatile(
	  "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
	  : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(taddr));
	asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
	for (int i = 0; i < 4; i++)
		v[i] = __uint_as_float(r[i]);
}

// 16-byte global -> shared copy (cp.async, L2 only); src_bytes 0 fills
// the 16 bytes with zeros.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src,
                                           uint32_t src_bytes)
{
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;"
	  :: "r"(dst), "l"(src), "r"(src_bytes) : "memory");
}

// Check of the bounded wait on this device (one thread): a wait limited to
// `cycles` on an mbarrier phase that nothing completes must time out
// (out[0] = 1), and after one arrival the same wait must succeed
// (out[1] = 1).  out[2] = clock cycles the timed-out wait took.
__global__ void k_wait_check(uint32_t cycles, uint32_t *out)
{
	__shared__ __align__(8) uint64_t mb;
	if (threadIdx.x != 0)
		return;
	uint32_t b = (uint32_t)__cvta_generic_to_shared(&mb);
	asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(b));
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	long long c0 = clock64();
	bool early = tc_wait(b, 0u, (long long)cycles);
	long long c1 = clock64();
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(b)
	  : "memory");
	bool done = tc_wait(b, 0u, (long long)cycles);
	out[0] = early ? 0u : 1u;
	out[1] = done ? 1u : 0u;
	out[2] = (uint32_t)min(c1 - c0, (long long)0xffffffff);
}

struct MlpTcSmem {
	__nv_bfloat16 w[kTcW];               // B operands, swizzled layout
	__nv_bfloat16 a[kTcGroups][kTcTile]; // A operands of layers 1..5
	__nv_bfloat16 f[kTcGroups][kTcTile]; // feature tile (layer 0's A)
	uint64_t bar[kTcGroups];
	uint32_t ok[kTcGroups];              // the issuer's wait result
	uint32_t tmem;
};
// every operand starts on a 1024-byte swizzle atom
static_assert(kTcW * 2 % 1024 == 0 && kTcTile * 2 % 1024 == 0,
              "UMMA operands must stay 1024-byte aligned");

// Barrier of the 128 threads of group g (named barrier 1 + g).
__device__ __forceinline__ void tc_group_sync(uint32_t g)
{
	asm volatile("bar.sync %0, 128;" :: "r"(1u + g) : "memory");
}

// Q = false: out[i] = (r, g, b, 0) = MLP(feats[i]) for i < n.
// Q = true (the frame's cache queries): query i is the entry qe[4i..4i+3]
// (position, direction, normal, albedo in .xyz; path index bits and the
// throughput in .w), encoded in registers straight into the feature tile;
// its output is added to the path's radiance, L[path] += T * max(y, 0)
// (entries whose path index is npath or more are skipped).
// n = min(*ncount, n) with ncount set.  kTcGroups groups of 4 warps, each an
// independent pipeline over 128-row tiles (its own TMEM accumulator of 64
// columns, feature and A buffers and mbarrier) sharing the weights: while
// the tensor core works for one group, the others run their epilogues.  The
// next tile's features go into the feature buffer as soon as layer 0 has
// read it.  One CTA per SM.
template <bool Q>
__global__ void __launch_bounds__(kTcThreads, 1)
k_mlp_fwd_tc(const __nv_bfloat16 *wbf, const __nv_bfloat16 *feats, uint32_t n,
             float4 *out, const uint32_t *ncount, uint32_t *err,
             const float4 *qe, NrcBox box, float4 *pL, uint32_t npath,
             bool scode, const uint4 *gq)
{
	if (ncount)
		n = min(*ncount, n);
	extern __shared__ __align__(1024) unsigned char tc_smem[];
	// the swizzle pattern repeats every 1024 bytes of the shared-memory
	// address: start the operands on such a boundary (the launch adds
	// 1 KB of slack)
	const uint32_t base = (uint32_t)__cvta_generic_to_shared(tc_smem);
	MlpTcSmem &S = *reinterpret_cast<MlpTcSmem *>(tc_smem +
	  ((1024u - (base & 1023u)) & 1023u));
	const uint32_t tid = threadIdx.x, warp = tid >> 5;
	const uint32_t g = tid >> 7, gt = tid & 127u; // group, thread in group
	const uint32_t sw = (uint32_t)__cvta_generic_to_shared(S.w);
	const uint32_t sa = (uint32_t)__cvta_generic_to_shared(S.a[g]);
	const uint32_t sf = (uint32_t)__cvta_generic_to_shared(S.f[g]);
	const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&S.bar[g]);
	unsigned char *abytes = reinterpret_cast<unsigned char *>(S.a[g]);
	uint32_t tiles = (n + kTcRows - 1u) / kTcRows;
	const uint32_t tstep = gridDim.x * (uint32_t)kTcGroups;
	unsigned char *fbytes = reinterpret_cast<unsigned char *>(S.f[g]);
	// path index bits and throughput of this thread's query in the next
	// tile and in the current one (Q)
	float4 meta_next = make_float4(0.0f, 0.0f, 0.0f, 0.0f), meta = meta_next;
	// this thread's feature row of tile tt (zeros past n) into the group's
	// feature buffer
	auto fetch = [&](uint32_t tt) {
		uint32_t rr = tt * kTcRows + gt;
		bool in = rr < n;
		if constexpr (Q) {
			uint4 pk[8];
			if (in) {
				const float4 *e = qe + 4ull * rr;
				float4 a = __ldg(e), b = __ldg(e + 1), c = __ldg(e + 2),
				  d = __ldg(e + 3);
				float raw[12] = {a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z,
				  d.x, d.y, d.z};
				nrc_encode(raw, box, pk, scode);
				// the hash grid's features 0..15, gathered beforehand by
				// k_grid_query_feats at full occupancy
				if (gq) {
					pk[0] = __ldg(gq + 2ull * rr);
					pk[1] = __ldg(gq + 2ull * rr + 1u);
				}
				meta_next = make_float4(a.w, b.w, c.w, d.w);
			} else {
#pragma unroll
				for (int q = 0; q < 8; q++)
					pk[q] = make_uint4(0, 0, 0, 0);
			}
#pragma unroll
			for (uint32_t q = 0; q < 8u; q++)
				*reinterpret_cast<uint4 *>(fbytes + tc_off(gt, q * 8u)) =
				  pk[q];
		} else {
			const uint4 *src = reinterpret_cast<const uint4 *>(feats +
			  (size_t)(in ? rr : 0u) * 64u);
#pragma unroll
			for (uint32_t kc = 0; kc < 8u; kc++)
				cp_async16(sf + tc_off(gt, kc * 8u), src + kc, in ? 16u : 0u);
			asm volatile("cp.async.commit_group;" ::: "memory");
		}
	};
	const uint32_t t0 = blockIdx.x * (uint32_t)kTcGroups + g;
	if (t0 < tiles)
		fetch(t0);
	// weights: layer l (rows 64, output layer 16 with rows 8..15 zero) in
	// the swizzled layout, layer bases 8 KB apart
	for (uint32_t i = tid; i < 5u * 64u * 8u + 16u * 8u;
	     i += (uint32_t)kTcThreads) {
		uint32_t row = i >> 3, kc = i & 7u; // row over all layers
		uint32_t l = row >> 6, r = row & 63u;
		uint4 v = make_uint4(0, 0, 0, 0);
		if (l < 5u || r < (uint32_t)kMlpOutPad)
			v = __ldg(reinterpret_cast<const uint4 *>(wbf + (size_t)row *
			  64u) + kc);
		*reinterpret_cast<uint4 *>(reinterpret_cast<unsigned char *>(S.w) +
		  l * 8192u + tc_off(r, kc * 8u)) = v;
	}
	if (warp == 0) {
		asm volatile(
		  "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
		  :: "r"((uint32_t)__cvta_generic_to_shared(&S.tmem)),
		  "n"(kTcCols));
		asm volatile(
		  "tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
	}
	if (tid < (uint32_t)kTcGroups) {
		uint32_t b = (uint32_t)__cvta_generic_to_shared(&S.bar[tid]);
		asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(b));
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
	const uint32_t tmem = S.tmem + g * 64u;
	const uint32_t tlane = tmem + (((warp & 3u) * 32u) << 16);
	uint32_t parity = 0;
	bool ok = true;
	for (uint32_t t = t0; t < tiles && ok; t += tstep) {
		uint32_t row = t * kTcRows + gt;
		// this thread's part of the feature tile has landed
		asm volatile("cp.async.wait_all;" ::: "memory");
		meta = meta_next;
		float o[4] = {0.0f, 0.0f, 0.0f, 0.0f};
		for (int l = 0; l <= kMlpSquare; l++) {
			// generic-proxy / cp.async writes visible to the tensor core
			asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
			asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
			tc_group_sync(g);
			asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
			uint32_t nn = l == kMlpSquare ? 16u : 64u;
			if (gt == 0) {
				uint32_t idesc = tc_idesc(nn);
				uint32_t src = l == 0 ? sf : sa;
#pragma unroll
				for (uint32_t ks = 0; ks < 4u; ks++)
					tc_mma(tmem, tc_desc(src + ks * 32u),
					  tc_desc(sw + (uint32_t)l * 8192u + ks * 32u), idesc,
					  ks > 0u ? 1u : 0u);
				tc_commit(bar);
				// one thread polls (bounded); the group barrier hands
				// the answer to the others
				S.ok[g] = tc_wait(bar, parity) ? 1u : 0u;
			}
			parity ^= 1u;
			tc_group_sync(g);
			ok = S.ok[g] != 0u;
			if (!ok)
				break;
			asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
			// layer 0 has read the feature tile: fetch the next one
			if (l == 0 && t + tstep < tiles)
				fetch(t + tstep);
			if (l < kMlpSquare) {
				// ReLU, BF16, next layer's A (this thread's row)
				uint32_t v[64];
				tc_ld64(tlane, v);
#pragma unroll
				for (uint32_t q = 0; q < 8u; q++) {
					uint4 pk;
					pk.x = pack_bf16(
					  fmaxf(__uint_as_float(v[8 * q]), 0.0f),
					  fmaxf(__uint_as_float(v[8 * q + 1]), 0.0f));
					pk.y = pack_bf16(
					  fmaxf(__uint_as_float(v[8 * q + 2]), 0.0f),
					  fmaxf(__uint_as_float(v[8 * q + 3]), 0.0f));
					pk.z = pack_bf16(
					  fmaxf(__uint_as_float(v[8 * q + 4]), 0.0f),
					  fmaxf(__uint_as_float(v[8 * q + 5]), 0.0f));
					pk.w = pack_bf16(
					  fmaxf(__uint_as_float(v[8 * q + 6]), 0.0f),
					  fmaxf(__uint_as_float(v[8 * q + 7]), 0.0f));
					*reinterpret_cast<uint4 *>(abytes + tc_off(gt, q * 8u)) =
					  pk;
				}
			} else {
				tc_ld4(tlane, o);
			}
		}
		if (ok && row < n) {
			if constexpr (Q) {
				uint32_t path = __float_as_uint(meta.x);
				if (path < npath) {
					float4 L = pL[path];
					L.x += meta.y * fmaxf(o[0], 0.0f);
					L.y += meta.z * fmaxf(o[1], 0.0f);
					L.z += meta.w * fmaxf(o[2], 0.0f);
					pL[path] = L;
				}
			} else {
				out[row] = make_float4(o[0], o[1], o[2], 0.0f);
			}
		}
	}
	asm volatile("cp.async.wait_all;" ::: "memory");
	if (!ok && gt == 0)
		atomicAdd(err, 1u);
	asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
	__syncthreads();
	if (warp == 0)
		asm volatile(
		  "tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(S.tmem),
		  "n"(kTcCols));
}

// --------------------------------------------------------------- training --

// Training, pass 1 on tcgen05: forward and backward of 128-row tiles, one
// tile pipeline (4 warps, one row per thread) per CTA.  UMMAs as in
// inference (M = 128 rows, N = 64, K-steps of 16, FP32 accumulators in
// TMEM, 128-byte swizzled K-major operands):
//   forward  l = 0..5: z_l = act_l W_l^T, act_{l+1} = bf16(relu(z_l))
//   backward l = 5..1: dA_l = dz_l W_l (B = the transposed copy [in][out],
//            one K-step for the 16-wide output layer), dz_{l-1} =
//            bf16(dA_l) where act_l > 0, else 0.
// All six layer inputs stay in shared memory for the ReLU derivative.
// Writes every layer's input (gact, [6][npad][64]), every layer's output
// gradient (gdz, [6][npad][64], the output layer's in columns 0..15, zero
// past 3) for pass 2, and a loss partial per CTA (relative L2 loss
// mean((y - t)^2 / (y^2 + 0.01)) over the batch and three channels, y
// detached in the denominator); rows at or past npad are not written.
// With ncount set, the batch is samples [off, off + n) of the
// min(*ncount, cap) produced on the device, off = offset mod that count.
// Waits are bounded; a timeout counts into *err and the CTA stops.
constexpr int kFbRows = kTcRows;
struct MlpFbSmem {
	__nv_bfloat16 w[kTcW];             // forward weights, layers 0..5
	__nv_bfloat16 wt[5 * 64 * 64];     // transposed weights, layers 1..5
	__nv_bfloat16 act[6][kTcTile];     // inputs of layers 0..5
	__nv_bfloat16 dz[kTcTile];         // output gradient of one layer
	uint64_t bar;
	uint32_t ok;
	uint32_t tmem;
	float loss;
};
static_assert(sizeof(__nv_bfloat16) * 5 * 64 * 64 % 1024 == 0,
              "UMMA operands must stay 1024-byte aligned");

// Store 8 16-byte chunks (one 64-wide bf16 row) to a global row.
__device__ __forceinline__ void st_row_global(__nv_bfloat16 *g,
                                              const uint4 *v)
{
#pragma unroll
	for (int q = 0; q < 8; q++)
		reinterpret_cast<uint4 *>(g)[q] = v[q];
}

__global__ void __launch_bounds__(kFbRows, 1)
k_mlp_fb_tc(const __nv_bfloat16 *wbf, const __nv_bfloat16 *wbt,
            const __nv_bfloat16 *feats, const float4 *targets, uint32_t n,
            uint32_t npad, __nv_bfloat16 *gact, __nv_bfloat16 *gdz,
            float *loss, const uint32_t *ncount, uint32_t offset,
            uint32_t cap, uint32_t *err)
{
	if (ncount) {
		uint32_t total = min(*ncount, cap);
		uint32_t off = total ? offset % total : 0u;
		uint32_t avail = total - off;
		feats += (size_t)off * kMlpIn;
		targets += off;
		n = min(n, avail);
	}
	extern __shared__ __align__(1024) unsigned char tc_smem[];
	const uint32_t base = (uint32_t)__cvta_generic_to_shared(tc_smem);
	MlpFbSmem &S = *reinterpret_cast<MlpFbSmem *>(tc_smem +
	  ((1024u - (base & 1023u)) & 1023u));
	const uint32_t tid = threadIdx.x, warp = tid >> 5;
	const uint32_t sw = (uint32_t)__cvta_generic_to_shared(S.w);
	const uint32_t swt = (uint32_t)__cvta_generic_to_shared(S.wt);
	const uint32_t sdz = (uint32_t)__cvta_generic_to_shared(S.dz);
	const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&S.bar);
	unsigned char *dzb = reinterpret_cast<unsigned char *>(S.dz);
	// forward weights: layer l at l * 8 KB, output layer 16 rows (8..15
	// zero); transposed weights of layer l at (l - 1) * 8 KB, the output
	// layer's 16 columns in K-chunks 0..1 (the rest zero).  cp.async keeps
	// all of a thread's copies in flight at once.
	for (uint32_t i = tid; i < 5u * 64u * 8u + 16u * 8u; i += kFbRows) {
		uint32_t row = i >> 3, kc = i & 7u;
		uint32_t l = row >> 6, r = row & 63u;
		bool in = l < 5u || r < (uint32_t)kMlpOutPad;
		cp_async16(sw + l * 8192u + tc_off(r, kc * 8u),
		  wbf + (in ? (size_t)row * 64u + kc * 8u : 0u), in ? 16u : 0u);
	}
	asm volatile("cp.async.commit_group;" ::: "memory");
	for (uint32_t i = tid; i < 5u * 64u * 8u; i += kFbRows) {
		uint32_t sl = i >> 9, r = (i >> 3) & 63u, kc = i & 7u;
		uint32_t l = sl + 1u;
		bool in = l < 5u || kc < 2u;
		size_t src = l < 5u ? (size_t)l * kMlpSq + r * 64u + kc * 8u :
		  (size_t)l * kMlpSq + r * (uint32_t)kMlpOutPadT + kc * 8u;
		cp_async16(swt + sl * 8192u + tc_off(r, kc * 8u),
		  wbt + (in ? src : 0u), in ? 16u : 0u);
	}
	asm volatile("cp.async.commit_group;" ::: "memory");
	// the forward weights have landed; the transposed ones may still be in
	// flight until the first backward layer
	asm volatile("cp.async.wait_group 1;" ::: "memory");
	if (warp == 0) {
		asm volatile(
		  "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;"
		  :: "r"((uint32_t)__cvta_generic_to_shared(&S.tmem)));
		asm volatile(
		  "tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
	}
	if (tid == 0) {
		asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(bar));
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
		S.loss = 0.0f;
	}
	asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
	const uint32_t tmem = S.tmem;
	const uint32_t tlane = tmem + ((warp * 32u) << 16);
	const float inv = n ? 1.0f / (3.0f * (float)n) : 0.0f;
	const uint32_t tiles = (npad + kFbRows - 1u) / kFbRows;
	uint32_t parity = 0;
	bool ok = true;
	float lsum = 0.0f;
	// one layer's UMMAs (ks K-steps of A x B^T into TMEM) by thread 0,
	// then a bounded wait; every thread learns the outcome
	auto run_layer = [&](uint32_t sa, uint32_t sb, uint32_t nn,
	                     uint32_t ksteps) {
		asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
		asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
		__syncthreads();
		asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
		if (tid == 0) {
			uint32_t idesc = tc_idesc(nn);
			for (uint32_t ks = 0; ks < ksteps; ks++)
				tc_mma(tmem, tc_desc(sa + ks * 32u), tc_desc(sb + ks * 32u),
				  idesc, ks > 0u ? 1u : 0u);
			tc_commit(bar);
			S.ok = tc_wait(bar, parity) ? 1u : 0u;
		}
		parity ^= 1u;
		__syncthreads();
		asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
		return S.ok != 0u;
	};
	for (uint32_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
		const uint32_t rr = t * kFbRows + tid;
		const bool live = rr < npad;
		// act_0 = the features of this thread's row (zero past n)
		{
			uint4 v[8];
#pragma unroll
			for (uint32_t kc = 0; kc < 8u; kc++) {
				v[kc] = rr < n ? __ldg(reinterpret_cast<const uint4 *>(
				  feats + (size_t)rr * 64u) + kc) : make_uint4(0, 0, 0, 0);
				*reinterpret_cast<uint4 *>(reinterpret_cast<unsigned char *>(
				  S.act[0]) + tc_off(tid, kc * 8u)) = v[kc];
			}
			if (live)
				st_row_global(gact + (size_t)rr * 64u, v);
		}
		float y[4] = {0.0f, 0.0f, 0.0f, 0.0f};
		for (uint32_t l = 0; l <= (uint32_t)kMlpSquare; l++) {
			ok = run_layer((uint32_t)__cvta_generic_to_shared(S.act[l]),
			  sw + l * 8192u, l == (uint32_t)kMlpSquare ? 16u : 64u, 4u);
			if (!ok)
				break;
			if (l < (uint32_t)kMlpSquare) {
				uint32_t v[64];
				tc_ld64(tlane, v);
				uint4 pk[8];
#pragma unroll
				for (uint32_t q = 0; q < 8u; q++) {
					pk[q].x = pack_bf16(
					  fmaxf(__uint_as_float(v[8 * q]), 0.0f),
					  fmaxf(__uint_as_float(v[8 * q + 1]), 0.0f));
					pk[q].y = pack_bf16(
					  fmaxf(__uint_as_float(v[8 * q + 2]), 0.0f),
					  fmaxf(__uint_as_float(v[8 * q + 3]), 0.0f));
					pk[q].z = pack_bf16(
					  fmaxf(__uint_as_float(v[8 * q + 4]), 0.0f),
					  fmaxf(__uint_as_float(v[8 * q + 5]), 0.0f));
					pk[q].w = pack_bf16(
					  fmaxf(__uint_as_float(v[8 * q + 6]), 0.0f),
					  fmaxf(__uint_as_float(v[8 * q + 7]), 0.0f));
					*reinterpret_cast<uint4 *>(
					  reinterpret_cast<unsigned char *>(S.act[l + 1u]) +
					  tc_off(tid, q * 8u)) = pk[q];
				}
				if (live)
					st_row_global(gact + ((size_t)(l + 1u) * npad + rr) *
					  64u, pk);
			} else {
				tc_ld4(tlane, y);
			}
		}
		if (!ok)
			break;
		// relative L2 loss and the output layer's gradient (this row)
		float g[3] = {0.0f, 0.0f, 0.0f};
		if (rr < n) {
			float4 tv = __ldg(targets + rr);
			float tt[3] = {tv.x, tv.y, tv.z};
#pragma unroll
			for (int c = 0; c < 3; c++) {
				float d = y[c] - tt[c], den = y[c] * y[c] + 0.01f;
				lsum += d * d / den;
				g[c] = 2.0f * d / den * inv;
			}
		}
		{
			uint4 pk[8];
			pk[0] = make_uint4(pack_bf16(g[0], g[1]), pack_bf16(g[2], 0.0f),
			  0u, 0u);
#pragma unroll
			for (int q = 1; q < 8; q++)
				pk[q] = make_uint4(0, 0, 0, 0);
			*reinterpret_cast<uint4 *>(dzb + tc_off(tid, 0u)) = pk[0];
			*reinterpret_cast<uint4 *>(dzb + tc_off(tid, 8u)) = pk[1];
			if (live)
				st_row_global(gdz + ((size_t)kMlpSquare * npad + rr) * 64u,
				  pk);
		}
		// backward: dz_{l-1} = (dz_l W_l) where act_l > 0
		asm volatile("cp.async.wait_all;" ::: "memory");
		for (uint32_t l = (uint32_t)kMlpSquare; l >= 1u; l--) {
			ok = run_layer(sdz, swt + (l - 1u) * 8192u, 64u,
			  l == (uint32_t)kMlpSquare ? 1u : 4u);
			if (!ok)
				break;
			uint32_t v[64];
			tc_ld64(tlane, v);
			const unsigned char *ab =
			  reinterpret_cast<const unsigned char *>(S.act[l]);
			uint4 pk[8];
#pragma unroll
			for (uint32_t q = 0; q < 8u; q++) {
				uint4 a = *reinterpret_cast<const uint4 *>(ab +
				  tc_off(tid, q * 8u));
				uint32_t aw[4] = {a.x, a.y, a.z, a.w};
				uint32_t o[4];
#pragma unroll
				for (int h = 0; h < 4; h++) {
					// relu'(z) from the stored input act_l = relu(z)
					bool p0 = (int16_t)(aw[h] & 0xffffu) > 0;
					bool p1 = (int16_t)(aw[h] >> 16) > 0;
					o[h] = pack_bf16(
					  p0 ? __uint_as_float(v[8 * q + 2 * h]) : 0.0f,
					  p1 ? __uint_as_float(v[8 * q + 2 * h + 1]) : 0.0f);
				}
				pk[q] = make_uint4(o[0], o[1], o[2], o[3]);
				if (l > 1u)
					*reinterpret_cast<uint4 *>(dzb + tc_off(tid, q * 8u)) =
					  pk[q];
			}
			if (live)
				st_row_global(gdz + ((size_t)(l - 1u) * npad + rr) * 64u,
				  pk);
		}
	}
	if (!ok && tid == 0)
		atomicAdd(err, 1u);
	atomicAdd(&S.loss, lsum);
	asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
	__syncthreads();
	if (tid == 0)
		loss[blockIdx.x] = S.loss;
	if (warp == 0)
		asm volatile(
		  "tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;" :: "r"(S.tmem));
}

// Training, pass 2: weight gradients dW_l[out][in] = sum_rows dz_l[row][out]
// act_l[row][in] as split-K UMMAs.  CTA (l = blockIdx.y, split blockIdx.x)
// sums rows [split * rows_per, ...) of layer l: chunks of 128 rows of dz_l
// and act_l stream into shared memory (cp.async, two stages) in the
// 128-byte swizzled layout, which read with the rows as K is the MN-major
// operand layout of both (A = dz^T: M = 64 outputs, B = act^T: N = 64
// inputs); one thread issues M64 N64 K16 UMMAs, 8 per chunk, into a
// 64-column TMEM accumulator.  An M = 64 accumulator puts output row i in
// TMEM lane (i mod 16) + 32 (i / 16): warp w's lanes 0..15 hold outputs
// 16w..16w+15.  The partial goes to part[split][layer l slice] (rows
// 0..7 of the output layer); the Adam kernel sums the splits.  Waits are
// bounded; a timeout counts into *err.
constexpr int kDwChunk = 128;
struct MlpDwSmem {
	__nv_bfloat16 dz[2][kDwChunk * 64];
	__nv_bfloat16 act[2][kDwChunk * 64];
	// slack behind the last operand: no descriptor stride can reach past
	// the allocation
	unsigned char guard[2048];
	uint64_t bar;
	uint32_t ok;
	uint32_t tmem;
};

// MN-major operand descriptor: 128-byte swizzle, 8-row K blocks 1024
// bytes apart; the one 64-wide MN block makes the leading offset unused
// (1024, inside the chunk).
__device__ __forceinline__ uint64_t tc_desc_mn(uint32_t saddr)
{
	uint64_t d = 0;
	d |= (uint64_t)((saddr >> 4) & 0x3fffu);
	d |= (uint64_t)((1024u >> 4) & 0x3fffu) << 16;
	d |= (uint64_t)((1024u >> 4) & 0x3fffu) << 32;
	d |= (uint64_t)1u << 46;
	d |= (uint64_t)2u << 61;
	return d;
}

__global__ void __launch_bounds__(128) k_mlp_dw_tc(const __nv_bfloat16 *gact,
                                                   const __nv_bfloat16 *gdz,
                                                   uint32_t npad,
                                                   uint32_t rows_per,
                                                   float *part,
                                                   uint32_t *err)
{
	extern __shared__ __align__(1024) unsigned char tc_smem[];
	const uint32_t base = (uint32_t)__cvta_generic_to_shared(tc_smem);
	MlpDwSmem &S = *reinterpret_cast<MlpDwSmem *>(tc_smem +
	  ((1024u - (base & 1023u)) & 1023u));
	const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
	const uint32_t l = blockIdx.y;
	const uint32_t nout = l == (uint32_t)kMlpSquare ? (uint32_t)kMlpOutPad : 64u;
	const __nv_bfloat16 *act = gact + (size_t)l * npad * 64;
	const __nv_bfloat16 *dzp = gdz + (size_t)l * npad * 64;
	const uint32_t r0 = blockIdx.x * rows_per;
	const uint32_t r1 = min(npad, r0 + rows_per);
	const uint32_t nch = r1 > r0 ? (r1 - r0 + kDwChunk - 1u) / kDwChunk : 0u;
	const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&S.bar);
	// rows [c0, c0 + rows) of dz_l and act_l into stage st
	auto fetch = [&](uint32_t c, uint32_t st) {
		uint32_t c0 = r0 + c * kDwChunk;
		uint32_t rows = min((uint32_t)kDwChunk, r1 - c0);
		uint32_t sd = (uint32_t)__cvta_generic_to_shared(S.dz[st]);
		uint32_t sa = (uint32_t)__cvta_generic_to_shared(S.act[st]);
		for (uint32_t i = tid; i < rows * 8u; i += 128u) {
			uint32_t r = i >> 3, q = i & 7u;
			cp_async16(sd + tc_off(r, q * 8u), dzp + (size_t)(c0 + r) * 64u +
			  q * 8u, 16u);
			cp_async16(sa + tc_off(r, q * 8u), act + (size_t)(c0 + r) * 64u +
			  q * 8u, 16u);
		}
		asm volatile("cp.async.commit_group;" ::: "memory");
	};
	if (warp == 0) {
		asm volatile(
		  "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;"
		  :: "r"((uint32_t)__cvta_generic_to_shared(&S.tmem)));
		asm volatile(
		  "tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
	}
	if (tid == 0) {
		asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(bar));
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	if (nch > 0u)
		fetch(0u, 0u);
	asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
	const uint32_t tmem = S.tmem;
	// F32 accumulate, BF16 A and B, both MN-major, N = 64, M = 64
	const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) |
	  (1u << 16) | ((64u >> 3) << 17) | ((64u >> 4) << 24);
	uint32_t parity = 0;
	bool ok = true;
	for (uint32_t c = 0; c < nch && ok; c++) {
		const uint32_t st = c & 1u;
		// the stage being refilled was read by chunk c - 1's UMMAs, which
		// completed before this iteration
		if (c + 1u < nch) {
			fetch(c + 1u, st ^ 1u);
			asm volatile("cp.async.wait_group 1;" ::: "memory");
		} else {
			asm volatile("cp.async.wait_all;" ::: "memory");
		}
		asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
		asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
		__syncthreads();
		asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
		if (tid == 0) {
			uint32_t rows = min((uint32_t)kDwChunk, r1 - (r0 + c * kDwChunk));
			uint32_t sd = (uint32_t)__cvta_generic_to_shared(S.dz[st]);
			uint32_t sa = (uint32_t)__cvta_generic_to_shared(S.act[st]);
			for (uint32_t ks = 0; ks < rows / 16u; ks++)
				tc_mma(tmem, tc_desc_mn(sd + ks * 2048u),
				  tc_desc_mn(sa + ks * 2048u), idesc,
				  (c > 0u || ks > 0u) ? 1u : 0u);
			tc_commit(bar);
			S.ok = tc_wait(bar, parity) ? 1u : 0u;
		}
		parity ^= 1u;
		__syncthreads();
		ok = S.ok != 0u;
	}
	asm volatile("cp.async.wait_all;" ::: "memory");
	asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
	// this split's slice of layer l (every element, zeros included)
	uint32_t v[64];
	tc_ld64(tmem + ((warp * 32u) << 16), v);
	const uint32_t o = warp * 16u + lane;
	if (lane < 16u && o < nout) {
		float *gp = part + (size_t)blockIdx.x * kMlpParams +
		  (size_t)l * kMlpSq + (size_t)o * 64u;
		bool any = nch > 0u && ok;
#pragma unroll
		for (uint32_t j = 0; j < 64u; j += 4u)
			*reinterpret_cast<float4 *>(gp + j) = any ? make_float4(
			  __uint_as_float(v[j]), __uint_as_float(v[j + 1]),
			  __uint_as_float(v[j + 2]), __uint_as_float(v[j + 3])) :
			  make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	}
	if (!ok && tid == 0)
		atomicAdd(err, 1u);
	asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
	__syncthreads();
	if (warp == 0)
		asm volatile(
		  "tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;" :: "r"(S.tmem));
}

// Sum the per-CTA partial gradients; optionally write the sum (g_out) and
// take one Adam step on the FP32 master weights, refreshing both BF16 copies.
// Output-layer rows 3..7 stay zero.
__global__ void k_mlp_adam(float *wf, float *m, float *v, const float *part,
                           int nparts, float *g_out, int update, float lr,
                           float beta1, float beta2, float eps, float bc1,
                           float bc2, __nv_bfloat16 *wbf, __nv_bfloat16 *wbt)
{
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpParams;
	     i += gridDim.x * blockDim.x) {
		float g = 0.0f;
		for (int p = 0; p < nparts; p++)
			g += part[(size_t)p * kMlpParams + i];
		int l = i / kMlpSq;
		int o = (i - l * kMlpSq) / 64, in = i & 63;
		bool pad = l == kMlpSquare && o >= 3;
		if (pad)
			g = 0.0f;
		if (g_out)
			g_out[i] = g;
		float w = wf[i];
		if (update && !pad) {
			float mi = beta1 * m[i] + (1.0f - beta1) * g;
			float vi = beta2 * v[i] + (1.0f - beta2) * g * g;
			m[i] = mi;
			v[i] = vi;
			w -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
			wf[i] = w;
		}
		__nv_bfloat16 wb = __float2bfloat16_rn(pad ? 0.0f : w);
		wbf[i] = wb;
		if (l < kMlpSquare)
			wbt[l * kMlpSq + in * 64 + o] = wb;
		else
			wbt[kMlpSquare * kMlpSq + in * kMlpOutPadT + o] = wb;
	}
}

// --------------------------------------------- encoding and frame kernels --

__global__ void k_nrc_encode(const float *raw, uint32_t n, NrcBox B,
                             __nv_bfloat16 *feats, const float2 *grid)
{
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
	     i += gridDim.x * blockDim.x)
		nrc_encode(raw + 12ull * i, B,
		  reinterpret_cast<uint4 *>(feats + 64ull * i), false, grid);
}

// Hash-grid features of cache queries (entries of 4 float4, position in
// the first), one thread per (query, level): out[8 q + l] = the level's two
// features as BF16 (what nrc_encode packs into features 2l, 2l + 1).
// n = min(*count, cap) queries (count null: cap).
__global__ void k_grid_query_feats(const float4 *qe, const uint32_t *count,
                                   uint32_t cap, NrcBox B, bool scode,
                                   const float2 *grid, uint32_t *out)
{
	uint32_t n = count ? min(*count, cap) : cap;
	const uint32_t work = n * (uint32_t)kGridLevels;
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < work;
	     t += gridDim.x * blockDim.x) {
		uint32_t r = t / (uint32_t)kGridLevels;
		int l = (int)(t % (uint32_t)kGridLevels);
		float4 a = __ldg(qe + 4ull * r);
		float in[3] = {a.x, a.y, a.z};
		float x[3];
		uint32_t scene = nrc_position(in, B, scode, x);
		float2 v = grid_level(grid, x, scene, l);
		out[t] = pack_bf16(v.x, v.y);
	}
}

// The training batch's rows: samples [off, off + n) of the
// min(*ncount, cap) made on the device, off = offset mod that count (as
// k_mlp_fb_tc takes them); without ncount, rows [0, n).
__device__ __forceinline__ uint32_t batch_rows(const uint32_t *ncount,
                                               uint32_t offset, uint32_t cap,
                                               uint32_t n, uint32_t *off)
{
	*off = 0u;
	if (!ncount)
		return n;
	uint32_t total = min(*ncount, cap);
	*off = total ? offset % total : 0u;
	return min(n, total - *off);
}

// Features of cache queries / training records produced by k_shade: the
// first four float4 of each entry (stride float4s) hold position, outgoing
// direction, normal and albedo in .xyz.  Entries [off, off + n) of the
// batch_rows selection, written to feats[off ...].
__global__ void k_nrc_encode_entries(const float4 *e, uint32_t stride,
                                     const uint32_t *count, uint32_t offset,
                                     uint32_t cap, uint32_t n, NrcBox B,
                                     __nv_bfloat16 *feats, bool scode,
                                     const float2 *grid)
{
	uint32_t off;
	n = batch_rows(count, offset, cap, n, &off);
	for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n;
	     r += gridDim.x * blockDim.x) {
		uint32_t i = off + r;
		const float4 *q = e + (size_t)stride * i;
		float4 a = q[0], b = q[1], c = q[2], d = q[3];
		float raw[12] = {a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z,
		  d.x, d.y, d.z};
		nrc_encode(raw, B, reinterpret_cast<uint4 *>(feats + 64ull * i),
		  scode, grid);
	}
}

// Gradient of the hash grid from a training batch's layer-0 output
// gradient (dz0: [rows][64] BF16, as k_mlp_fb_tc writes it): per row
// dL/dfeature_j = sum_o dz0[o] W0[o][j] for the 16 grid features (W0 the
// BF16 copy the forward pass used), spread over each level's 8 cell
// corners with their trilinear weights into gg (FP32 pairs, vector
// atomics).  One thread per (row, level), so a 16k-row batch fills the GPU.
// Rows are the entries of batch_rows (stride float4s each, raw inputs as
// for k_nrc_encode_entries, position box B); without ncount, raw holds 12
// floats per row (the public raw layout).
__global__ void __launch_bounds__(256) k_grid_grad(
  const float4 *e, const float *raw, uint32_t stride, const uint32_t *ncount,
  uint32_t offset, uint32_t cap, uint32_t n, NrcBox B, bool scode,
  const __nv_bfloat16 *dz0, const __nv_bfloat16 *wbf, float2 *gg)
{
	// W0's grid columns, transposed; the odd row pitch spreads the levels
	// of one o over different banks
	__shared__ float w0[2 * kGridLevels][65];
	for (uint32_t i = threadIdx.x; i < 64u * 2u * kGridLevels;
	     i += blockDim.x) {
		uint32_t j = i / 64u, o = i % 64u;
		w0[j][o] = __bfloat162float(wbf[o * 64u + j]);
	}
	__syncthreads();
	uint32_t off;
	n = batch_rows(ncount, offset, cap, n, &off);
	const uint32_t work = n * (uint32_t)kGridLevels;
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < work;
	     t += gridDim.x * blockDim.x) {
		uint32_t r = t / (uint32_t)kGridLevels;
		int l = (int)(t % (uint32_t)kGridLevels);
		const uint4 *dzr = reinterpret_cast<const uint4 *>(dz0 + 64ull * r);
		float d0 = 0.0f, d1 = 0.0f;
#pragma unroll
		for (int q = 0; q < 8; q++) {
			uint4 v = dzr[q];
			uint32_t wv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
			for (int h = 0; h < 8; h++) {
				float d = __uint_as_float((h & 1) ? (wv[h >> 1] & 0xffff0000u) :
				  (wv[h >> 1] << 16));
				d0 = __fmaf_rn(d, w0[2 * l][8 * q + h], d0);
				d1 = __fmaf_rn(d, w0[2 * l + 1][8 * q + h], d1);
			}
		}
		if (d0 == 0.0f && d1 == 0.0f)
			continue;
		float in[3];
		if (ncount) {
			float4 a = e[(size_t)stride * (off + r)];
			in[0] = a.x;
			in[1] = a.y;
			in[2] = a.z;
		} else {
			for (int k = 0; k < 3; k++)
				in[k] = raw[12ull * r + k];
		}
		float x[3];
		uint32_t scene = nrc_position(in, B, scode, x);
		uint32_t c[3];
		float w[3];
#pragma unroll
		for (int a = 0; a < 3; a++)
			grid_cell(l, x[a], &c[a], &w[a]);
#pragma unroll
		for (int b = 0; b < 8; b++) {
			uint32_t k = grid_index(l, c[0] + (b & 1), c[1] + ((b >> 1) & 1),
			  c[2] + ((b >> 2) & 1), scene);
			float wt = grid_weight(b, w);
			atomicAdd(gg + k, make_float2(__fmul_rn(wt, d0),
			  __fmul_rn(wt, d1)));
		}
	}
}

// One Adam step of the hash grid from the gradient gg (then cleared), four
// parameters per thread; g_out receives the gradient when not null.  Lazy
// (sparse) Adam: only parameters the batch touched (nonzero gradient) move
// and decay their moments; the others, most of a large table, are not read
// at all.  A parameter's first update is the dense one.
__global__ void k_grid_adam(float4 *__restrict__ t, float4 *__restrict__ m,
                            float4 *__restrict__ v, float4 *__restrict__ gg,
                            float4 *__restrict__ g_out, int update, float lr,
                            float beta1, float beta2, float eps, float bc1,
                            float bc2)
{
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kGridParams / 4;
	     i += gridDim.x * blockDim.x) {
		float4 g4 = gg[i];
		bool any = g4.x != 0.0f || g4.y != 0.0f || g4.z != 0.0f ||
		  g4.w != 0.0f;
		if (g_out)
			g_out[i] = g4;
		if (!any)
			continue;
		gg[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
		if (!update)
			continue;
		float4 m4 = m[i], v4 = v[i], t4 = t[i];
		float *gp = &g4.x, *mp = &m4.x, *vp = &v4.x, *tp = &t4.x;
#pragma unroll
		for (int k = 0; k < 4; k++) {
			float g = gp[k];
			if (g == 0.0f)
				continue;
			float mi = beta1 * mp[k] + (1.0f - beta1) * g;
			float vi = beta2 * vp[k] + (1.0f - beta2) * g * g;
			mp[k] = mi;
			vp[k] = vi;
			tp[k] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
		}
		m[i] = m4;
		v[i] = v4;
		t[i] = t4;
	}
}

// Training target of a record: the radiance its path gathered from this
// vertex on, divided by the throughput on arrival.
__global__ void k_nrc_targets(const float4 *rec, const uint32_t *count,
                              uint32_t cap, const float4 *pL, float4 *tgt)
{
	uint32_t n = min(*count, cap);
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
	     i += gridDim.x * blockDim.x) {
		const float4 *e = rec + 6u * i;
		uint32_t path = __float_as_uint(e[0].w);
		float4 L = pL[path], Lb = e[4], T = e[5];
		float4 t;
		t.x = T.x > 0.0f ? (L.x - Lb.x) / T.x : 0.0f;
		t.y = T.y > 0.0f ? (L.y - Lb.y) / T.y : 0.0f;
		t.z = T.z > 0.0f ? (L.z - Lb.z) / T.z : 0.0f;
		t.w = 0.0f;
		tgt[i] = t;
	}
}

} // namespace nb

#endif
