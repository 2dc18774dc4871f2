// C ABI of the B200 path-tracing core (include/rendgpu.h).
//
// One context per `struct rdata`, found through a small registry keyed by
// the rdata pointer (the reference API passes only that pointer).  Uploads
// convert the reference BVH8 to the GPU layout (layout.cpp); a frame is the
// fixed launch sequence of kernels.cuh on the context's stream.

#include <cfloat>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/rendgpu.h"
#include "kernels.cuh"
#include "layout.hpp"
#include "nrc.cuh"

namespace nb {
namespace {

constexpr int kStackSmall = 24;
constexpr int kStackLarge = 48;
constexpr int kTraceBlock = 128;

// Device allocation that grows on demand.
struct DevBuf {
	void  *p = nullptr;
	size_t cap = 0;
	cudaError_t ensure(size_t bytes)
	{
		if (bytes <= cap && p)
			return cudaSuccess;
		if (p)
			cudaFree(p);
		p = nullptr;
		cap = 0;
		size_t b = bytes ? bytes : 16;
		cudaError_t e = cudaMalloc(&p, b);
		if (e == cudaSuccess)
			cap = b;
		return e;
	}
	void release()
	{
		if (p)
			cudaFree(p);
		p = nullptr;
		cap = 0;
	}
	template <class T> T *as() const { return static_cast<T *>(p); }
};

struct Ctx {
	nb_rdata    *rd = nullptr;
	rendgpu_cfg  cfg{};
	int          device = 0;
	int          nsm = 148;
	cudaStream_t stream = nullptr;
	// scene
	DevBuf blas, tris, tlas, irefs, insts, nrms, mtls, lights;
	std::unordered_map<uint32_t, uint32_t> root_of; // triofs -> BLAS root
	std::unordered_map<uint32_t, uint32_t> depth_of; // triofs -> BLAS depth
	uint32_t blas_depth = 0, tlas_depth = 0;
	std::vector<nb_glight> host_lights;
	float    light_area = 0.0f;
	bool     have_static = false, have_dynamic = false;
	uint32_t ntris = 0, nnodes = 0;
	// frame
	DevBuf q0, q1, hits, shadow, scol, pT, pL, rng, acc, buf, cnt, rays;
	uint32_t W = 0, H = 0, spp = 0, npaths = 0;
	bool     have_frame = false;
	// batch scratch: rays, raw hits, output; berr = [count, errors, work]
	DevBuf brays, braw, bhits, berr;
	// neural radiance cache: FP32 master weights, Adam moments, BF16
	// forward / transposed copies, per-CTA gradient partials and losses
	DevBuf mlp_wf, mlp_m, mlp_v, mlp_wbf, mlp_wbt, mlp_part, mlp_loss;
	uint32_t mlp_step = 0;
	bool     mlp_ready = false;
	NrcBox   box{};
	DevBuf   nq, nfeat, npred, nrec, rfeat, rtgt; // radiance-cache frame data
	uint32_t nq_cap = 0, nrec_cap = 0, nrc_stride = 1;
	uint32_t nrc_frames = 0; // radiance-cache frames rendered so far
	uint32_t train_grid = 0; // CTAs of the last training step
	// stats / errors
	rendgpu_stats st{};
	int          last = 0;
	std::string  msg;
	cudaEvent_t  ev[64] = {};
	int          nev = 0;
};

std::mutex g_mu;
std::unordered_map<const void *, Ctx *> g_ctx;

Ctx *find_ctx(const void *rd)
{
	std::lock_guard<std::mutex> lk(g_mu);
	auto it = g_ctx.find(rd);
	return it == g_ctx.end() ? nullptr : it->second;
}

int fail(Ctx *c, int code, const std::string &m)
{
	if (c) {
		c->last = code;
		c->msg = m;
	}
	return code;
}

int cuda_fail(Ctx *c, cudaError_t e, const char *where)
{
	return fail(c, RENDGPU_ECUDA, std::string(where) + ": " +
	  cudaGetErrorString(e));
}

#define NB_CK(c, call)                                                   \
	do {                                                              \
		cudaError_t e_ = (call);                                  \
		if (e_ != cudaSuccess)                                    \
			return cuda_fail((c), e_, #call);                 \
	} while (0)

uint32_t need_stack(const Ctx *c)
{
	return c->tlas_depth + c->blas_depth + 2u;
}

DScene scene_of(const Ctx *c)
{
	DScene S;
	S.blas = c->blas.as<nb_qnode>();
	S.tris = c->tris.as<float4>();
	S.tlas = c->tlas.as<nb_qnode>();
	S.irefs = c->irefs.as<uint32_t>();
	S.insts = c->insts.as<float4>();
	S.nrms = c->nrms.as<nb_rnrm>();
	S.mtls = c->mtls.as<nb_rmtl>();
	S.lights = c->lights.as<float4>();
	S.nlights = (uint32_t)c->host_lights.size();
	S.light_area = c->light_area;
	S.bg[0] = c->rd->bgcol.x;
	S.bg[1] = c->rd->bgcol.y;
	S.bg[2] = c->rd->bgcol.z;
	return S;
}

// Schedule of the trace kernels: cfg.sched 1..3; 0 = the default, the
// Ylitie-style schedule (fastest measured on the 1920x1080 4 spp workload:
// 789 vs 664 (step) vs 544 (phase) Mrays/s).
int sched_of(const Ctx *c)
{
	switch (c->cfg.sched) {
	case 1: return kSchedStep;
	case 2: return kSchedPhase;
	default: return kSchedYlitie;
	}
}

// Occupancy-sized persistent grid; allows dynamic shared memory above
// 48 KB for the deep-stack variants on first use.
int trace_grid(Ctx *c, const void *fn, int stack)
{
	size_t smem0 = (size_t)stack * kTraceBlock * sizeof(uint2);
	if (smem0 > 48 * 1024)
		cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
		  (int)smem0);
	int per_sm = 0;
	size_t smem = (size_t)stack * kTraceBlock * sizeof(uint2);
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn,
	  kTraceBlock, smem) != cudaSuccess || per_sm < 1)
		per_sm = 1;
	return per_sm * c->nsm;
}

template <int SCHED, int STACK, bool COUNT>
void trace_kernel(Ctx *c, const float4 *rays, const uint32_t *count,
                  uint32_t *work, float4 *hits, uint32_t *errs,
                  unsigned long long *nrays)
{
	auto fn = k_trace<SCHED, STACK, COUNT>;
	size_t smem = (size_t)STACK * kTraceBlock * sizeof(uint2);
	fn<<<trace_grid(c, (const void *)fn, STACK), kTraceBlock, smem,
	  c->stream>>>(scene_of(c), rays, count, work, hits, errs, nrays,
	  c->rays.as<unsigned long long>() + 2);
}

template <int SCHED, int STACK>
void trace_kernel_c(Ctx *c, const float4 *rays, const uint32_t *count,
                    uint32_t *work, float4 *hits, uint32_t *errs,
                    unsigned long long *nrays)
{
	if (c->cfg.flags & RENDGPU_FLAG_COUNT)
		trace_kernel<SCHED, STACK, true>(c, rays, count, work, hits, errs,
		  nrays);
	else
		trace_kernel<SCHED, STACK, false>(c, rays, count, work, hits, errs,
		  nrays);
}

template <int STACK>
void trace_kernel_s(Ctx *c, const float4 *rays, const uint32_t *count,
                    uint32_t *work, float4 *hits, uint32_t *errs,
                    unsigned long long *nrays)
{
	switch (sched_of(c)) {
	case kSchedPhase:
		trace_kernel_c<kSchedPhase, STACK>(c, rays, count, work, hits, errs,
		  nrays);
		break;
	case kSchedYlitie:
		trace_kernel_c<kSchedYlitie, STACK>(c, rays, count, work, hits,
		  errs, nrays);
		break;
	default:
		trace_kernel_c<kSchedStep, STACK>(c, rays, count, work, hits, errs,
		  nrays);
	}
}

// Launch a closest-hit trace of `count` (device) rays: raw hits.
int launch_trace(Ctx *c, const float4 *rays, const uint32_t *count,
                 uint32_t *work, float4 *hits, uint32_t *errs,
                 unsigned long long *nrays)
{
	uint32_t need = need_stack(c);
	if (need <= (uint32_t)kStackSmall)
		trace_kernel_s<kStackSmall>(c, rays, count, work, hits, errs,
		  nrays);
	else if (need <= (uint32_t)kStackLarge)
		trace_kernel_s<kStackLarge>(c, rays, count, work, hits, errs,
		  nrays);
	else
		return fail(c, RENDGPU_ELIMIT, "BVH too deep for the traversal "
		  "stack");
	NB_CK(c, cudaGetLastError());
	return 0;
}

template <int SCHED, int STACK>
void shadow_kernel(Ctx *c, FrameDev &F)
{
	auto fn = k_shadow<SCHED, STACK>;
	size_t smem = (size_t)STACK * kTraceBlock * sizeof(uint2);
	fn<<<trace_grid(c, (const void *)fn, STACK), kTraceBlock, smem,
	  c->stream>>>(scene_of(c), F);
}

template <int STACK>
void shadow_kernel_s(Ctx *c, FrameDev &F)
{
	switch (sched_of(c)) {
	case kSchedPhase:
		shadow_kernel<kSchedPhase, STACK>(c, F);
		break;
	case kSchedYlitie:
		shadow_kernel<kSchedYlitie, STACK>(c, F);
		break;
	default:
		shadow_kernel<kSchedStep, STACK>(c, F);
	}
}

int launch_shadow(Ctx *c, FrameDev &F)
{
	uint32_t need = need_stack(c);
	if (need <= (uint32_t)kStackSmall)
		shadow_kernel_s<kStackSmall>(c, F);
	else if (need <= (uint32_t)kStackLarge)
		shadow_kernel_s<kStackLarge>(c, F);
	else
		return fail(c, RENDGPU_ELIMIT, "BVH too deep for the traversal "
		  "stack");
	NB_CK(c, cudaGetLastError());
	return 0;
}

template <int STACK>
void occl_kernel(Ctx *c, const float4 *rays, const uint32_t *count,
                 uint32_t *work, uint8_t *occl, uint32_t *errs)
{
	auto fn = k_occluded<kSchedYlitie, STACK>;
	size_t smem = (size_t)STACK * kTraceBlock * sizeof(uint2);
	fn<<<trace_grid(c, (const void *)fn, STACK), kTraceBlock, smem,
	  c->stream>>>(scene_of(c), rays, count, work, occl, errs);
}

int launch_occluded(Ctx *c, const float4 *rays, const uint32_t *count,
                    uint32_t *work, uint8_t *occl, uint32_t *errs)
{
	uint32_t need = need_stack(c);
	if (need <= (uint32_t)kStackSmall)
		occl_kernel<kStackSmall>(c, rays, count, work, occl, errs);
	else if (need <= (uint32_t)kStackLarge)
		occl_kernel<kStackLarge>(c, rays, count, work, occl, errs);
	else
		return fail(c, RENDGPU_ELIMIT, "BVH too deep for the traversal "
		  "stack");
	NB_CK(c, cudaGetLastError());
	return 0;
}

FrameDev frame_of(Ctx *c)
{
	FrameDev F;
	F.q[0] = c->q0.as<float4>();
	F.q[1] = c->q1.as<float4>();
	F.hits = c->hits.as<float4>();
	F.shadow = c->shadow.as<float4>();
	F.scol = c->scol.as<float4>();
	F.pT = c->pT.as<float4>();
	F.pL = c->pL.as<float4>();
	F.rng = c->rng.as<uint2>();
	F.acc = c->acc.as<float>();
	F.buf = c->buf.as<uint32_t>();
	F.cnt = c->cnt.as<uint32_t>();
	F.rays = c->rays.as<unsigned long long>();
	F.W = c->W;
	F.H = c->H;
	F.spp = c->spp;
	F.npaths = c->npaths;
	return F;
}

int ready(Ctx *c, bool frame)
{
	if (!c)
		return RENDGPU_EINVAL;
	if (!c->have_static || !c->have_dynamic)
		return fail(c, RENDGPU_ESTATE, "upload_static and upload_dynamic "
		  "must come first");
	if (frame && !c->have_frame)
		return fail(c, RENDGPU_ESTATE, "rendgpu_resaccum must come first");
	return 0;
}

int grid_for(const Ctx *c, uint32_t n, int block)
{
	uint32_t g = (n + (uint32_t)block - 1u) / (uint32_t)block;
	uint32_t cap = (uint32_t)c->nsm * 8u;
	return (int)(g < 1u ? 1u : (g > cap ? cap : g));
}

void ev_record(Ctx *c)
{
	if (!(c->cfg.flags & RENDGPU_FLAG_TIMING) || c->nev >= 64)
		return;
	if (!c->ev[c->nev])
		cudaEventCreate(&c->ev[c->nev]);
	cudaEventRecord(c->ev[c->nev], c->stream);
	c->nev++;
}

float ev_ms(Ctx *c, int a, int b)
{
	float ms = 0.0f;
	if (a < c->nev && b < c->nev)
		cudaEventElapsedTime(&ms, c->ev[a], c->ev[b]);
	return ms;
}

// ------------------------------------------------ neural radiance cache --

constexpr float kAdamBeta1 = 0.9f, kAdamBeta2 = 0.99f, kAdamEps = 1e-15f;

float nrc_lr(const Ctx *c)
{
	float lr;
	std::memcpy(&lr, &c->cfg.reserved[0], sizeof(lr));
	return lr > 0.0f ? lr : 1e-2f;
}

// Xavier-uniform FP32 master weights from a seeded PCG32 stream, zero Adam
// moments, BF16 copies refreshed on the device.
int nrc_reset(Ctx *c, uint64_t seed)
{
	NB_CK(c, c->mlp_wf.ensure(kMlpParams * sizeof(float)));
	NB_CK(c, c->mlp_m.ensure(kMlpParams * sizeof(float)));
	NB_CK(c, c->mlp_v.ensure(kMlpParams * sizeof(float)));
	NB_CK(c, c->mlp_wbf.ensure(kMlpParams * sizeof(__nv_bfloat16)));
	NB_CK(c, c->mlp_wbt.ensure(kMlpParamsT * sizeof(__nv_bfloat16)));
	NB_CK(c, c->mlp_loss.ensure(1024 * sizeof(float)));
	std::vector<float> w(kMlpParams, 0.0f);
	uint64_t st = 0, inc = (seed << 1) | 1u;
	auto next = [&]() {
		uint64_t old = st;
		st = old * 6364136223846793005ull + inc;
		uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
		uint32_t rot = (uint32_t)(old >> 59u);
		return (xs >> rot) | (xs << ((32u - rot) & 31u));
	};
	next();
	st += 0x853c49e6748fea9bull;
	next();
	// Xavier uniform for the hidden layers; the output layer starts at
	// zero so an untrained cache adds no energy
	for (int l = 0; l < kMlpSquare; l++) {
		int nout = 64;
		float bound = std::sqrt(6.0f / (64.0f + (float)nout));
		for (int o = 0; o < nout; o++)
			for (int i = 0; i < 64; i++) {
				float u = (float)(next() >> 8) * 0x1p-24f;
				w[l * kMlpSq + o * 64 + i] = (2.0f * u - 1.0f) * bound;
			}
	}
	NB_CK(c, cudaMemcpyAsync(c->mlp_wf.p, w.data(), w.size() * 4,
	  cudaMemcpyHostToDevice, c->stream));
	NB_CK(c, cudaMemsetAsync(c->mlp_m.p, 0, kMlpParams * 4, c->stream));
	NB_CK(c, cudaMemsetAsync(c->mlp_v.p, 0, kMlpParams * 4, c->stream));
	NB_CK(c, cudaMemsetAsync(c->mlp_wbt.p, 0, kMlpParamsT * 2, c->stream));
	k_mlp_adam<<<grid_for(c, kMlpParams, 256), 256, 0, c->stream>>>(
	  c->mlp_wf.as<float>(), c->mlp_m.as<float>(), c->mlp_v.as<float>(),
	  nullptr, 0, nullptr, 0, 0.0f, kAdamBeta1, kAdamBeta2, kAdamEps, 1.0f,
	  1.0f, c->mlp_wbf.as<__nv_bfloat16>(), c->mlp_wbt.as<__nv_bfloat16>());
	NB_CK(c, cudaGetLastError());
	c->mlp_step = 0;
	c->mlp_ready = true;
	return 0;
}

// Frames of unbiased tracing that train the cache before it ends paths
// (cfg.reserved[1]; 0 = 8).
uint32_t nrc_warmup(const Ctx *c)
{
	return c->cfg.reserved[1] ? c->cfg.reserved[1] : 8u;
}

constexpr uint32_t kNrcBatch = 16384;    // training samples per Adam step
constexpr uint32_t kNrcSteps = 4;        // Adam steps per frame
constexpr uint32_t kNrcTrainPaths = 65536; // training paths per frame (2^16)

// Radiance-cache buffers of a frame: queries and their features/outputs
// for every path, records for the training paths' vertices.
int nrc_frame_buffers(Ctx *c)
{
	if (!c->mlp_ready) {
		int rc = nrc_reset(c, c->cfg.seed);
		if (rc)
			return rc;
	}
	uint32_t np = c->npaths;
	// about 2^16 training paths, and never more than 1 path in 16
	c->nrc_stride = std::max(16u, np / kNrcTrainPaths);
	uint32_t verts = c->cfg.max_depth > 1 ? c->cfg.max_depth - 1 : 1;
	// warm-up frames record from every path; later frames overwrite the
	// capacity-limited prefix only, so cap at 4 batches per frame worth of
	// vertices beyond the steady-state need
	uint32_t ntrain = np / c->nrc_stride + 1;
	c->nq_cap = np;
	c->nrec_cap = std::max(ntrain * verts + 64, kNrcSteps * kNrcBatch);
	NB_CK(c, c->nq.ensure((size_t)np * 64));
	NB_CK(c, c->nfeat.ensure((size_t)np * 128));
	NB_CK(c, c->npred.ensure((size_t)np * 16));
	NB_CK(c, c->nrec.ensure((size_t)c->nrec_cap * 96));
	NB_CK(c, c->rfeat.ensure((size_t)c->nrec_cap * 128));
	NB_CK(c, c->rtgt.ensure((size_t)c->nrec_cap * 16));
	return 0;
}

// Forward pass of n (or, with ncount, of min(*ncount, n)) queries.
int nrc_infer(Ctx *c, const void *feats, uint32_t n, float4 *out,
              const uint32_t *ncount = nullptr)
{
	if (n == 0)
		return 0;
	int per_sm = 0;
	size_t smem = kMlpParams * sizeof(__nv_bfloat16);
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mlp_fwd, 128,
	  smem);
	uint32_t tiles = (n + 15u) / 16u;
	uint32_t grid = std::min<uint32_t>((tiles + 3u) / 4u,
	  (uint32_t)std::max(per_sm, 1) * (uint32_t)c->nsm);
	k_mlp_fwd<<<grid, 128, smem, c->stream>>>(c->mlp_wbf.as<__nv_bfloat16>(),
	  static_cast<const __nv_bfloat16 *>(feats), n, out, ncount);
	NB_CK(c, cudaGetLastError());
	return 0;
}

// Gradient of a batch (and optionally one Adam step).  g_out (device,
// kMlpParams floats) receives the summed gradient when not null; *loss the
// batch loss when not null (synchronises).
int nrc_train(Ctx *c, const void *feats, const float4 *targets, uint32_t n,
              int update, float *g_out, float *loss,
              const uint32_t *ncount = nullptr, uint32_t offset = 0,
              uint32_t cap = 0)
{
	if (n == 0)
		return 0;
	static bool attr = false;
	size_t smem = sizeof(MlpTrainSmem);
	if (!attr) {
		NB_CK(c, cudaFuncSetAttribute(k_mlp_grad,
		  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
		attr = true;
	}
	uint32_t tiles = (n + 15u) / 16u;
	uint32_t grid = std::min<uint32_t>((tiles + 15u) / 16u,
	  (uint32_t)c->nsm);
	grid = std::max(grid, 1u);
	NB_CK(c, c->mlp_part.ensure((size_t)grid * kMlpParams * sizeof(float)));
	c->train_grid = grid;
	k_mlp_grad<<<grid, 128, smem, c->stream>>>(c->mlp_wbf.as<__nv_bfloat16>(),
	  c->mlp_wbt.as<__nv_bfloat16>(), static_cast<const __nv_bfloat16 *>(feats),
	  targets, n, c->mlp_part.as<float>(), c->mlp_loss.as<float>(), ncount,
	  offset, cap);
	NB_CK(c, cudaGetLastError());
	if (update)
		c->mlp_step++;
	float bc1 = 1.0f - std::pow(kAdamBeta1, (float)std::max(c->mlp_step, 1u));
	float bc2 = 1.0f - std::pow(kAdamBeta2, (float)std::max(c->mlp_step, 1u));
	k_mlp_adam<<<grid_for(c, kMlpParams, 256), 256, 0, c->stream>>>(
	  c->mlp_wf.as<float>(), c->mlp_m.as<float>(), c->mlp_v.as<float>(),
	  c->mlp_part.as<float>(), (int)grid, g_out, update, nrc_lr(c),
	  kAdamBeta1, kAdamBeta2, kAdamEps, bc1, bc2,
	  c->mlp_wbf.as<__nv_bfloat16>(), c->mlp_wbt.as<__nv_bfloat16>());
	NB_CK(c, cudaGetLastError());
	if (loss) {
		std::vector<float> l(grid);
		NB_CK(c, cudaMemcpyAsync(l.data(), c->mlp_loss.p, grid * 4,
		  cudaMemcpyDeviceToHost, c->stream));
		NB_CK(c, cudaStreamSynchronize(c->stream));
		double sum = 0.0;
		for (float x : l)
			sum += x;
		*loss = (float)(sum / (3.0 * n));
	}
	return 0;
}

int render_frame(Ctx *c)
{
	int rc = ready(c, true);
	if (rc)
		return rc;
	nb_rdata *rd = c->rd;
	if (rd->width != c->W || rd->height != c->H || rd->spp != c->spp)
		return fail(c, RENDGPU_ESTATE, "rdata size changed since "
		  "rendgpu_resaccum");
	FrameDev F = frame_of(c);
	FrameArgs A;
	A.seed = c->cfg.seed;
	A.frame = rd->samples;
	A.depth = c->cfg.mode == RENDGPU_MODE_PRIMARY ? 1u : c->cfg.max_depth;
	A.mode = c->cfg.mode;
	A.nrc_stride = 1;
	A.nrc_offset = 0;
	bool nrc = c->cfg.mode == RENDGPU_MODE_NRC;
	if (nrc) {
		int rc2 = nrc_frame_buffers(c);
		if (rc2)
			return rc2;
		A.nrc_stride = c->nrc_stride;
		A.nrc_offset = (rd->samples * 7919u) % c->nrc_stride;
		// warm-up: the first frames trace every path unbiased (as
		// training paths) while the cache trains
		if (c->nrc_frames < nrc_warmup(c))
			A.nrc_stride = 1;
		c->nrc_frames++;
	}
	const nb_rcam &cam = rd->cam;
	A.eye[0] = cam.eye.x; A.eye[1] = cam.eye.y; A.eye[2] = cam.eye.z;
	A.ri[0] = cam.ri.x; A.ri[1] = cam.ri.y; A.ri[2] = cam.ri.z;
	A.up[0] = cam.up.x; A.up[1] = cam.up.y; A.up[2] = cam.up.z;
	A.fwd[0] = cam.fwd.x; A.fwd[1] = cam.fwd.y; A.fwd[2] = cam.fwd.z;
	A.rw = cam.rw8[0];
	A.rh = cam.rh8[0];
	A.fovfdist = cam.fovfdist8[0];
	A.aspect = cam.aspect8[0];
	A.fdist = cam.fdist8[0];
	A.focrad = cam.focrad8[0];
	A.tanfangle = cam.tanfangle;
	F.nq = c->nq.as<float4>();
	F.nrec = c->nrec.as<float4>();
	F.nq_cap = c->nq_cap;
	F.nrec_cap = c->nrec_cap;
	DScene S = scene_of(c);
	c->nev = 0;
	c->st.launches = 0;
	c->st.trace_launches = 0;
	NB_CK(c, cudaMemsetAsync(c->cnt.p, 0, 64 * sizeof(uint32_t), c->stream));
	NB_CK(c, cudaMemsetAsync(c->rays.p, 0, 4 * sizeof(unsigned long long),
	  c->stream));
	ev_record(c); // 0
	uint32_t tiles = ((c->W + 7u) >> 3) * ((c->H + 3u) >> 2) * 32u * c->spp;
	k_gen<<<grid_for(c, tiles, 256), 256, 0, c->stream>>>(F, A);
	NB_CK(c, cudaGetLastError());
	c->st.launches++;
	ev_record(c); // 1
	std::vector<int> trace_ev, shadow_ev;
	for (uint32_t k = 0; k < A.depth; k++) {
		uint32_t cur = k & 1u;
		trace_ev.push_back(c->nev);
		ev_record(c);
		rc = launch_trace(c, F.q[cur], F.cnt + cur, F.cnt + 4, F.hits,
		  F.cnt + 3, F.rays);
		if (rc)
			return rc;
		ev_record(c);
		c->st.launches++;
		c->st.trace_launches++;
		NB_CK(c, cudaMemsetAsync(F.cnt + (cur ^ 1u), 0, sizeof(uint32_t),
		  c->stream));
		NB_CK(c, cudaMemsetAsync(F.cnt + 2, 0, sizeof(uint32_t),
		  c->stream));
		k_shade<<<grid_for(c, c->npaths, 256), 256, 0, c->stream>>>(S, F,
		  A, cur, k);
		NB_CK(c, cudaGetLastError());
		c->st.launches++;
		if (A.mode != RENDGPU_MODE_PRIMARY) {
			shadow_ev.push_back(c->nev);
			ev_record(c);
			rc = launch_shadow(c, F);
			if (rc)
				return rc;
			ev_record(c);
			c->st.launches++;
		}
	}
	int nrc_ev = c->nev;
	if (nrc) {
		// cache inference for the queries of this frame
		ev_record(c);
		k_nrc_encode_entries<<<grid_for(c, c->nq_cap, 128), 128, 0,
		  c->stream>>>(F.nq, 4u, F.cnt + 40, c->nq_cap, c->box,
		  c->nfeat.as<__nv_bfloat16>());
		rc = nrc_infer(c, c->nfeat.p, c->nq_cap, c->npred.as<float4>(),
		  F.cnt + 40);
		if (rc)
			return rc;
		k_nrc_apply<<<grid_for(c, c->nq_cap, 256), 256, 0, c->stream>>>(
		  F.nq, F.cnt + 40, c->nq_cap, c->npred.as<float4>(), F.pL);
		NB_CK(c, cudaGetLastError());
		c->st.launches += 3;
		ev_record(c);
	}
	int acc_ev = c->nev;
	ev_record(c);
	float inv = 1.0f / (float)(rd->samples + rd->spp);
	k_accum<<<grid_for(c, c->W * c->H, 256), 256, 0, c->stream>>>(F, inv);
	NB_CK(c, cudaGetLastError());
	c->st.launches++;
	ev_record(c);
	int train_ev = c->nev;
	if (nrc) {
		// train on this frame's records: targets from the finished paths,
		// then kNrcSteps Adam steps of kNrcBatch samples each
		ev_record(c);
		k_nrc_targets<<<grid_for(c, c->nrec_cap, 256), 256, 0, c->stream>>>(
		  F.nrec, F.cnt + 41, c->nrec_cap, F.pL, c->rtgt.as<float4>());
		k_nrc_encode_entries<<<grid_for(c, c->nrec_cap, 128), 128, 0,
		  c->stream>>>(F.nrec, 6u, F.cnt + 41, c->nrec_cap, c->box,
		  c->rfeat.as<__nv_bfloat16>());
		NB_CK(c, cudaGetLastError());
		for (uint32_t s = 0; s < kNrcSteps; s++) {
			rc = nrc_train(c, c->rfeat.p, c->rtgt.as<float4>(), kNrcBatch, 1,
			  nullptr, nullptr, F.cnt + 41, s * kNrcBatch, c->nrec_cap);
			if (rc)
				return rc;
		}
		c->st.launches += 2 + 2 * kNrcSteps;
		ev_record(c);
	}
	unsigned long long hr[4];
	uint32_t hc[64];
	NB_CK(c, cudaMemcpyAsync(hr, c->rays.p, sizeof(hr),
	  cudaMemcpyDeviceToHost, c->stream));
	NB_CK(c, cudaMemcpyAsync(hc, c->cnt.p, sizeof(hc),
	  cudaMemcpyDeviceToHost, c->stream));
	NB_CK(c, cudaStreamSynchronize(c->stream));
	c->st.closest_rays = hr[0];
	c->st.node_visits = hr[2];
	c->st.tri_tests = hr[3];
	c->st.shadow_rays = hr[1];
	c->st.rays = hr[0] + hr[1];
	c->st.device_errors = hc[3];
	if (nrc) {
		// loss of the last Adam step (partials of its CTAs)
		float lp[1024];
		uint32_t ng = std::min<uint32_t>(c->train_grid, 1024);
		NB_CK(c, cudaMemcpy(lp, c->mlp_loss.p, ng * 4,
		  cudaMemcpyDeviceToHost));
		double sl = 0.0;
		for (uint32_t i = 0; i < ng; i++)
			sl += lp[i];
		uint32_t used = std::min(std::min(hc[41], c->nrec_cap), kNrcBatch);
		c->st.nrc_loss = used ? (float)(sl / (3.0 * used)) : 0.0f;
	}
	c->st.nrc_queries = nrc ? std::min(hc[40], c->nq_cap) : 0;
	c->st.nrc_records = nrc ? std::min(hc[41], c->nrec_cap) : 0;
	for (int k = 0; k < 16; k++) {
		c->st.bounce_closest[k] = hc[8 + k];
		c->st.bounce_shadow[k] = hc[24 + k];
	}
	c->st.max_stack = need_stack(c);
	if (c->cfg.flags & RENDGPU_FLAG_TIMING) {
		c->st.ms_frame = ev_ms(c, 0, c->nev - 1);
		float tr = 0.0f, sh = 0.0f;
		for (int e : trace_ev)
			tr += ev_ms(c, e, e + 1);
		for (int e : shadow_ev)
			sh += ev_ms(c, e, e + 1);
		c->st.ms_trace = tr;
		c->st.ms_shadow = sh;
		c->st.ms_nrc = nrc ? ev_ms(c, nrc_ev, nrc_ev + 1) +
		  ev_ms(c, train_ev, train_ev + 1) : 0.0f;
		c->st.ms_shade = c->st.ms_frame - tr - sh - c->st.ms_nrc;
		(void)acc_ev;
	}
	if (hc[3])
		return fail(c, RENDGPU_EDEVICE, "rays abandoned on the device "
		  "(traversal stack overflow)");
	return 0;
}

void free_ctx(Ctx *c)
{
	DevBuf *bufs[] = {&c->blas, &c->tris, &c->tlas, &c->irefs, &c->insts,
	  &c->nrms, &c->mtls, &c->lights, &c->q0, &c->q1, &c->hits, &c->shadow,
	  &c->scol, &c->pT, &c->pL, &c->rng, &c->acc, &c->buf, &c->cnt,
	  &c->rays, &c->brays, &c->braw, &c->bhits, &c->berr, &c->mlp_wf,
	  &c->mlp_m, &c->mlp_v, &c->mlp_wbf, &c->mlp_wbt, &c->mlp_part,
	  &c->mlp_loss, &c->nq, &c->nfeat, &c->npred, &c->nrec, &c->rfeat,
	  &c->rtgt};
	for (DevBuf *b : bufs)
		b->release();
	for (int i = 0; i < 64; i++)
		if (c->ev[i])
			cudaEventDestroy(c->ev[i]);
	if (c->stream)
		cudaStreamDestroy(c->stream);
	delete c;
}

uint64_t held_bytes(const Ctx *c)
{
	const DevBuf *bufs[] = {&c->blas, &c->tris, &c->tlas, &c->irefs,
	  &c->insts, &c->nrms, &c->mtls, &c->lights, &c->q0, &c->q1, &c->hits,
	  &c->shadow, &c->scol, &c->pT, &c->pL, &c->rng, &c->acc, &c->buf,
	  &c->cnt, &c->rays, &c->brays, &c->braw, &c->bhits, &c->berr,
	  &c->mlp_wf, &c->mlp_m, &c->mlp_v, &c->mlp_wbf, &c->mlp_wbt,
	  &c->mlp_part, &c->mlp_loss, &c->nq, &c->nfeat, &c->npred, &c->nrec,
	  &c->rfeat, &c->rtgt};
	uint64_t s = 0;
	for (const DevBuf *b : bufs)
		s += b->cap;
	return s;
}

// ------------------------------------------------ allocation-free tracing --
//
// rendgpu_trace_rays_device_noalloc keeps its scratch (three counters and the
// raw hits of up to kNoAllocMaxRays rays, 4 MiB + 256 B) in this file-scope
// device array instead of context buffers that grow with cudaMalloc.  Every
// GPU that loads the library holds the array until the process exits.  Host
// code only ever sees a host-side stand-in under the array's name, so the
// device address is looked up with cudaGetSymbolAddress once per device and
// cached.

constexpr uint32_t kNoAllocMaxRays = 1u << 18;
constexpr size_t kNoAllocHeader = 256;

static __device__ __align__(256) unsigned char
  g_noalloc_scratch[kNoAllocHeader + (size_t)kNoAllocMaxRays * 16];

std::mutex g_noalloc_mu;
void *g_noalloc_addr[64];

// Device address of the scratch array on the current device `dev` (first
// use on a device performs the lookup).
int noalloc_scratch(Ctx *c, int dev, unsigned char **base)
{
	if (dev < 0 || dev >= 64)
		return fail(c, RENDGPU_EINVAL, "device ordinal above 63");
	std::lock_guard<std::mutex> lk(g_noalloc_mu);
	if (!g_noalloc_addr[dev]) {
		void *p = nullptr;
		cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		if (e != cudaSuccess || !p)
			return cuda_fail(c, e, "cudaGetSymbolAddress(scratch)");
		g_noalloc_addr[dev] = p;
	}
	*base = static_cast<unsigned char *>(g_noalloc_addr[dev]);
	return 0;
}

// Count, error and work counters of one call, written on the device so the
// call needs no host-to-device copy.
__global__ void k_noalloc_begin(uint32_t *hdr, uint32_t n)
{
	if (threadIdx.x == 0) {
		hdr[0] = n;
		hdr[1] = 0u;
		hdr[2] = 0u;
	}
}

} // namespace
} // namespace nb

using namespace nb;

extern "C" {

int rendgpu_init(struct rdata *rdp, const struct rendgpu_cfg *cfg)
{
	if (!rdp || !cfg || cfg->size < sizeof(rendgpu_cfg) - 8 * sizeof(uint32_t))
		return RENDGPU_EINVAL;
	if (find_ctx(rdp))
		return RENDGPU_ESTATE;
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
		return RENDGPU_ENODEV;
	if (cfg->device < 0 || cfg->device >= ndev)
		return RENDGPU_EINVAL;
	if (cfg->mode > RENDGPU_MODE_NRC || cfg->max_depth < 1 ||
	  cfg->max_depth > 1024 || cfg->sched > 3)
		return RENDGPU_EINVAL;
	Ctx *c = new Ctx;
	c->rd = reinterpret_cast<nb_rdata *>(rdp);
	c->cfg = *cfg;
	c->device = cfg->device;
	if (cudaSetDevice(c->device) != cudaSuccess ||
	  cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount,
	  c->device) != cudaSuccess ||
	  cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) !=
	  cudaSuccess) {
		free_ctx(c);
		return RENDGPU_ECUDA;
	}
	if (c->cnt.ensure(64 * sizeof(uint32_t)) != cudaSuccess ||
	  c->rays.ensure(4 * sizeof(unsigned long long)) != cudaSuccess ||
	  c->berr.ensure(16) != cudaSuccess) {
		free_ctx(c);
		return RENDGPU_ENOMEM;
	}
	std::lock_guard<std::mutex> lk(g_mu);
	g_ctx[rdp] = c;
	return 0;
}

int rendgpu_release(struct rdata *rdp)
{
	Ctx *c = nullptr;
	{
		std::lock_guard<std::mutex> lk(g_mu);
		auto it = g_ctx.find(rdp);
		if (it == g_ctx.end())
			return RENDGPU_EINVAL;
		c = it->second;
		g_ctx.erase(it);
	}
	cudaSetDevice(c->device);
	cudaStreamSynchronize(c->stream);
	free_ctx(c);
	return 0;
}

int rendgpu_upload_static(struct rdata *rdp)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	NB_CK(c, cudaSetDevice(c->device));
	nb_rdata *rd = c->rd;
	if (!rd->bnodes || !rd->tris || !rd->nrms || !rd->mtls || !rd->insts)
		return fail(c, RENDGPU_EINVAL, "render data not initialised");
	if (rd->instcnt == 0 || rd->instcnt > (1u << NB_INST_ID_BITS))
		return fail(c, RENDGPU_ELIMIT, "instance count outside 1..4096 "
		  "(INST_ID_BITS = 12, rend.c:24)");
	std::vector<nb_qnode> nodes;
	std::vector<nb_gtri> tris;
	c->root_of.clear();
	c->depth_of.clear();
	c->blas_depth = 0;
	uint32_t maxtri = 0, maxmtl = 0;
	for (uint32_t i = 0; i < rd->instcnt; i++) {
		const nb_rinst &ri = rd->insts[i];
		if (ri.tricnt == 0)
			return fail(c, RENDGPU_EINVAL, "instance without triangles");
		if (ri.tricnt > (1u << (32 - NB_INST_ID_BITS)))
			return fail(c, RENDGPU_ELIMIT, "mesh above 2^20 triangles");
		maxtri = std::max(maxtri, ri.triofs + ri.tricnt);
		if (c->root_of.count(ri.triofs))
			continue;
		uint32_t root = 0;
		bvh_stats bs;
		std::string err;
		if (!convert_blas(rd, ri.triofs, nodes, tris, &root, &bs, &err))
			return fail(c, RENDGPU_EINVAL, "BLAS of triofs " +
			  std::to_string(ri.triofs) + ": " + err);
		c->root_of[ri.triofs] = root;
		c->depth_of[ri.triofs] = bs.depth;
		c->blas_depth = std::max(c->blas_depth, bs.depth);
	}
	for (uint32_t t = 0; t < maxtri; t++)
		maxmtl = std::max(maxmtl, rd->nrms[t].mtlid + 1u);
	NB_CK(c, c->blas.ensure(nodes.size() * sizeof(nb_qnode)));
	NB_CK(c, c->tris.ensure(tris.size() * sizeof(nb_gtri)));
	NB_CK(c, c->nrms.ensure((size_t)maxtri * sizeof(nb_rnrm)));
	NB_CK(c, c->mtls.ensure((size_t)maxmtl * sizeof(nb_rmtl)));
	NB_CK(c, cudaMemcpyAsync(c->blas.p, nodes.data(), nodes.size() *
	  sizeof(nb_qnode), cudaMemcpyHostToDevice, c->stream));
	NB_CK(c, cudaMemcpyAsync(c->tris.p, tris.data(), tris.size() *
	  sizeof(nb_gtri), cudaMemcpyHostToDevice, c->stream));
	NB_CK(c, cudaMemcpyAsync(c->nrms.p, rd->nrms, (size_t)maxtri *
	  sizeof(nb_rnrm), cudaMemcpyHostToDevice, c->stream));
	NB_CK(c, cudaMemcpyAsync(c->mtls.p, rd->mtls, (size_t)maxmtl *
	  sizeof(nb_rmtl), cudaMemcpyHostToDevice, c->stream));
	NB_CK(c, cudaStreamSynchronize(c->stream));
	c->ntris = (uint32_t)tris.size();
	c->nnodes = (uint32_t)nodes.size();
	c->have_static = true;
	c->have_dynamic = false;
	return 0;
}

int rendgpu_upload_dynamic(struct rdata *rdp)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	if (!c->have_static)
		return fail(c, RENDGPU_ESTATE, "upload_static must come first");
	NB_CK(c, cudaSetDevice(c->device));
	nb_rdata *rd = c->rd;
	std::vector<nb_qnode> nodes;
	std::vector<uint32_t> irefs;
	bvh_stats bs;
	std::string err;
	if (!convert_tlas(rd, nodes, irefs, &bs, &err))
		return fail(c, RENDGPU_EINVAL, "TLAS: " + err);
	c->tlas_depth = bs.depth;
	std::vector<nb_ginst> gi(rd->instcnt);
	for (uint32_t i = 0; i < rd->instcnt; i++) {
		const nb_rinst &ri = rd->insts[i];
		auto it = c->root_of.find(ri.triofs);
		if (it == c->root_of.end())
			return fail(c, RENDGPU_ESTATE, "instance mesh not uploaded "
			  "by upload_static");
		std::memcpy(gi[i].m, ri.globinv, sizeof(gi[i].m));
		gi[i].root = it->second;
		gi[i].triofs = ri.triofs;
		gi[i].flags = ri.flags;
		gi[i].pad = 0;
	}
	c->light_area = build_lights(rd, c->host_lights);
	{
		float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
		float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
		for (uint32_t i = 0; i < rd->instcnt; i++) {
			const nb_aabb &b = rd->aabbs[i];
			float bl[3] = {b.min.x, b.min.y, b.min.z};
			float bh[3] = {b.max.x, b.max.y, b.max.z};
			for (int a = 0; a < 3; a++) {
				lo[a] = std::min(lo[a], bl[a]);
				hi[a] = std::max(hi[a], bh[a]);
			}
		}
		for (int a = 0; a < 3; a++) {
			c->box.lo[a] = lo[a];
			c->box.inv[a] = hi[a] > lo[a] ? 1.0f / (hi[a] - lo[a]) : 1.0f;
		}
	}
	NB_CK(c, c->tlas.ensure(nodes.size() * sizeof(nb_qnode)));
	NB_CK(c, c->irefs.ensure(irefs.size() * sizeof(uint32_t)));
	NB_CK(c, c->insts.ensure(gi.size() * sizeof(nb_ginst)));
	NB_CK(c, c->lights.ensure(c->host_lights.size() * sizeof(nb_glight)));
	NB_CK(c, cudaMemcpyAsync(c->tlas.p, nodes.data(), nodes.size() *
	  sizeof(nb_qnode), cudaMemcpyHostToDevice, c->stream));
	NB_CK(c, cudaMemcpyAsync(c->irefs.p, irefs.data(), irefs.size() *
	  sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
	NB_CK(c, cudaMemcpyAsync(c->insts.p, gi.data(), gi.size() *
	  sizeof(nb_ginst), cudaMemcpyHostToDevice, c->stream));
	if (!c->host_lights.empty())
		NB_CK(c, cudaMemcpyAsync(c->lights.p, c->host_lights.data(),
		  c->host_lights.size() * sizeof(nb_glight),
		  cudaMemcpyHostToDevice, c->stream));
	NB_CK(c, cudaStreamSynchronize(c->stream));
	c->st.h2d_bytes = nodes.size() * sizeof(nb_qnode) + irefs.size() *
	  sizeof(uint32_t) + gi.size() * sizeof(nb_ginst) +
	  c->host_lights.size() * sizeof(nb_glight);
	c->have_dynamic = true;
	if (need_stack(c) > (uint32_t)kStackLarge)
		return fail(c, RENDGPU_ELIMIT, "BVH too deep for the traversal "
		  "stack");
	return 0;
}

int rendgpu_resaccum(struct rdata *rdp)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	NB_CK(c, cudaSetDevice(c->device));
	nb_rdata *rd = c->rd;
	uint64_t np = (uint64_t)rd->width * rd->height * (rd->spp ? rd->spp : 1);
	if (np == 0 || np > 0x7fffffffull)
		return fail(c, RENDGPU_ELIMIT, "width*height*spp outside "
		  "1..2^31-1");
	uint64_t npix = (uint64_t)rd->width * rd->height;
	NB_CK(c, c->q0.ensure(np * 32));
	NB_CK(c, c->q1.ensure(np * 32));
	NB_CK(c, c->hits.ensure(np * 16));
	NB_CK(c, c->shadow.ensure(np * 32));
	NB_CK(c, c->scol.ensure(np * 16));
	NB_CK(c, c->pT.ensure(np * 16));
	NB_CK(c, c->pL.ensure(np * 16));
	NB_CK(c, c->rng.ensure(np * 8));
	NB_CK(c, c->acc.ensure(npix * 12));
	NB_CK(c, c->buf.ensure(npix * 4));
	c->W = rd->width;
	c->H = rd->height;
	c->spp = rd->spp ? rd->spp : 1;
	c->npaths = (uint32_t)np;
	c->have_frame = true;
	NB_CK(c, cudaMemsetAsync(c->acc.p, 0, npix * 12, c->stream));
	NB_CK(c, cudaMemsetAsync(c->buf.p, 0, npix * 4, c->stream));
	NB_CK(c, cudaStreamSynchronize(c->stream));
	return 0;
}

int rendgpu_clraccum(struct rdata *rdp)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	if (!c->have_frame)
		return fail(c, RENDGPU_ESTATE, "rendgpu_resaccum must come first");
	NB_CK(c, cudaSetDevice(c->device));
	NB_CK(c, cudaMemsetAsync(c->acc.p, 0, (size_t)c->W * c->H * 12,
	  c->stream));
	return 0;
}

int rendgpu_render(void *rdp)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return 0;
	nb_rdata *rd = c->rd;
	// Claim the frame as rend_render claims blocks (rend.c:3623): only
	// the first caller of a frame renders.
	if (__atomic_fetch_add(&rd->blknum, 1, __ATOMIC_SEQ_CST) != 0)
		return 0;
	if (cudaSetDevice(c->device) != cudaSuccess) {
		fail(c, RENDGPU_ECUDA, "cudaSetDevice");
		return 0;
	}
	c->last = 0;
	int rc = render_frame(c);
	if (rc) {
		c->last = rc;
		return 0;
	}
	__atomic_fetch_add(&rd->rays, (unsigned int)c->st.rays,
	  __ATOMIC_SEQ_CST);
	return 0;
}

int rendgpu_readback(struct rdata *rdp, int which)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	if (!c->have_frame)
		return fail(c, RENDGPU_ESTATE, "rendgpu_resaccum must come first");
	NB_CK(c, cudaSetDevice(c->device));
	nb_rdata *rd = c->rd;
	size_t npix = (size_t)c->W * c->H;
	c->st.d2h_bytes = 0;
	if ((which & 1) && rd->acc) {
		NB_CK(c, cudaMemcpyAsync(rd->acc, c->acc.p, npix * 12,
		  cudaMemcpyDeviceToHost, c->stream));
		c->st.d2h_bytes += npix * 12;
	}
	if ((which & 2) && rd->buf) {
		NB_CK(c, cudaMemcpyAsync(rd->buf, c->buf.p, npix * 4,
		  cudaMemcpyDeviceToHost, c->stream));
		c->st.d2h_bytes += npix * 4;
	}
	NB_CK(c, cudaStreamSynchronize(c->stream));
	return 0;
}

int rendgpu_trace_rays_device(struct rdata *rdp, const void *rays,
                              uint32_t n, void *hits)
{
	Ctx *c = find_ctx(rdp);
	int rc = ready(c, false);
	if (rc)
		return rc;
	if (n == 0)
		return 0;
	NB_CK(c, cudaSetDevice(c->device));
	NB_CK(c, c->braw.ensure((size_t)n * 16));
	// berr: [0] count, [1] errors, [2] work counter
	uint32_t hdr[3] = {n, 0u, 0u};
	NB_CK(c, cudaMemcpyAsync(c->berr.p, hdr, sizeof(hdr),
	  cudaMemcpyHostToDevice, c->stream));
	uint32_t *b = c->berr.as<uint32_t>();
	const float4 *r4 = static_cast<const float4 *>(rays);
	rc = launch_trace(c, r4, b, b + 2, c->braw.as<float4>(), b + 1, nullptr);
	if (rc)
		return rc;
	k_refine<<<grid_for(c, n, 256), 256, 0, c->stream>>>(scene_of(c), r4, b,
	  c->braw.as<float4>(), static_cast<float4 *>(hits));
	NB_CK(c, cudaGetLastError());
	return 0;
}

int rendgpu_occluded_device(struct rdata *rdp, const void *rays, uint32_t n,
                            void *occl)
{
	Ctx *c = find_ctx(rdp);
	int rc = ready(c, false);
	if (rc)
		return rc;
	if (n == 0)
		return 0;
	NB_CK(c, cudaSetDevice(c->device));
	uint32_t hdr[3] = {n, 0u, 0u};
	NB_CK(c, cudaMemcpyAsync(c->berr.p, hdr, sizeof(hdr),
	  cudaMemcpyHostToDevice, c->stream));
	uint32_t *b = c->berr.as<uint32_t>();
	return launch_occluded(c, static_cast<const float4 *>(rays), b, b + 2,
	  static_cast<uint8_t *>(occl), b + 1);
}

int rendgpu_trace_rays_device_noalloc(struct rdata *rdp, const void *rays,
                                      uint32_t n, void *hits)
{
	Ctx *c = find_ctx(rdp);
	int rc = ready(c, false);
	if (rc)
		return rc;
	if (n == 0)
		return 0;
	if (n > kNoAllocMaxRays)
		return fail(c, RENDGPU_ELIMIT, "rendgpu_trace_rays_device_noalloc: "
		  "n = " + std::to_string(n) + " exceeds the fixed scratch of " +
		  std::to_string(kNoAllocMaxRays) + " rays; split the batch");
	if (!rays || !hits)
		return fail(c, RENDGPU_EINVAL, "null pointer");
	NB_CK(c, cudaSetDevice(c->device));
	unsigned char *base = nullptr;
	rc = noalloc_scratch(c, c->device, &base);
	if (rc)
		return rc;
	uint32_t *hdr = reinterpret_cast<uint32_t *>(base);
	float4 *raw = reinterpret_cast<float4 *>(base + kNoAllocHeader);
	k_noalloc_begin<<<1, 32, 0, c->stream>>>(hdr, n);
	NB_CK(c, cudaGetLastError());
	const float4 *r4 = static_cast<const float4 *>(rays);
	rc = launch_trace(c, r4, hdr, hdr + 2, raw, hdr + 1, nullptr);
	if (rc)
		return rc;
	k_refine<<<grid_for(c, n, 256), 256, 0, c->stream>>>(scene_of(c), r4,
	  hdr, raw, static_cast<float4 *>(hits));
	NB_CK(c, cudaGetLastError());
	return 0;
}

static int batch_errors(Ctx *c)
{
	uint32_t e = 0;
	NB_CK(c, cudaMemcpyAsync(&e, c->berr.as<uint32_t>() + 1, 4,
	  cudaMemcpyDeviceToHost, c->stream));
	NB_CK(c, cudaStreamSynchronize(c->stream));
	c->st.device_errors = e;
	if (e)
		return fail(c, RENDGPU_EDEVICE, "rays abandoned on the device "
		  "(traversal stack overflow)");
	return 0;
}

int rendgpu_trace_rays(struct rdata *rdp, const struct rendgpu_ray *rays,
                       uint32_t n, struct rendgpu_hit *hits)
{
	Ctx *c = find_ctx(rdp);
	int rc = ready(c, false);
	if (rc)
		return rc;
	if (n == 0)
		return 0;
	if (!rays || !hits)
		return fail(c, RENDGPU_EINVAL, "null pointer");
	NB_CK(c, cudaSetDevice(c->device));
	NB_CK(c, c->brays.ensure((size_t)n * 32));
	NB_CK(c, c->bhits.ensure((size_t)n * 16));
	NB_CK(c, cudaMemcpyAsync(c->brays.p, rays, (size_t)n * 32,
	  cudaMemcpyHostToDevice, c->stream));
	rc = rendgpu_trace_rays_device(rdp, c->brays.p, n, c->bhits.p);
	if (rc)
		return rc;
	NB_CK(c, cudaMemcpyAsync(hits, c->bhits.p, (size_t)n * 16,
	  cudaMemcpyDeviceToHost, c->stream));
	return batch_errors(c);
}

int rendgpu_occluded(struct rdata *rdp, const struct rendgpu_ray *rays,
                     uint32_t n, uint8_t *occl)
{
	Ctx *c = find_ctx(rdp);
	int rc = ready(c, false);
	if (rc)
		return rc;
	if (n == 0)
		return 0;
	if (!rays || !occl)
		return fail(c, RENDGPU_EINVAL, "null pointer");
	NB_CK(c, cudaSetDevice(c->device));
	NB_CK(c, c->brays.ensure((size_t)n * 32));
	NB_CK(c, c->bhits.ensure((size_t)n));
	NB_CK(c, cudaMemcpyAsync(c->brays.p, rays, (size_t)n * 32,
	  cudaMemcpyHostToDevice, c->stream));
	rc = rendgpu_occluded_device(rdp, c->brays.p, n, c->bhits.p);
	if (rc)
		return rc;
	NB_CK(c, cudaMemcpyAsync(occl, c->bhits.p, (size_t)n,
	  cudaMemcpyDeviceToHost, c->stream));
	return batch_errors(c);
}

int rendgpu_nrc_reset(struct rdata *rdp, uint64_t seed)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	NB_CK(c, cudaSetDevice(c->device));
	return nrc_reset(c, seed);
}

int rendgpu_nrc_weights(struct rdata *rdp, float *host, int write)
{
	Ctx *c = find_ctx(rdp);
	if (!c || !host)
		return RENDGPU_EINVAL;
	if (!c->mlp_ready)
		return fail(c, RENDGPU_ESTATE, "rendgpu_nrc_reset must come first");
	NB_CK(c, cudaSetDevice(c->device));
	if (write) {
		NB_CK(c, cudaMemcpyAsync(c->mlp_wf.p, host, kMlpParams * 4,
		  cudaMemcpyHostToDevice, c->stream));
		k_mlp_adam<<<grid_for(c, kMlpParams, 256), 256, 0, c->stream>>>(
		  c->mlp_wf.as<float>(), c->mlp_m.as<float>(), c->mlp_v.as<float>(),
		  nullptr, 0, nullptr, 0, 0.0f, kAdamBeta1, kAdamBeta2, kAdamEps,
		  1.0f, 1.0f, c->mlp_wbf.as<__nv_bfloat16>(),
		  c->mlp_wbt.as<__nv_bfloat16>());
		NB_CK(c, cudaGetLastError());
	} else {
		NB_CK(c, cudaMemcpyAsync(host, c->mlp_wf.p, kMlpParams * 4,
		  cudaMemcpyDeviceToHost, c->stream));
	}
	NB_CK(c, cudaStreamSynchronize(c->stream));
	return 0;
}

int rendgpu_nrc_encode_device(struct rdata *rdp, const float *raw, uint32_t n,
                              void *feats)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	if (!c->have_dynamic)
		return fail(c, RENDGPU_ESTATE, "upload_dynamic must come first");
	if (n == 0)
		return 0;
	NB_CK(c, cudaSetDevice(c->device));
	k_nrc_encode<<<grid_for(c, n, 128), 128, 0, c->stream>>>(raw, n, c->box,
	  static_cast<__nv_bfloat16 *>(feats));
	NB_CK(c, cudaGetLastError());
	return 0;
}

int rendgpu_nrc_infer_device(struct rdata *rdp, const void *feats, uint32_t n,
                             float *out)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	if (!c->mlp_ready)
		return fail(c, RENDGPU_ESTATE, "rendgpu_nrc_reset must come first");
	NB_CK(c, cudaSetDevice(c->device));
	return nrc_infer(c, feats, n, reinterpret_cast<float4 *>(out));
}

int rendgpu_nrc_train_device(struct rdata *rdp, const void *feats,
                             const float *targets, uint32_t n, int update,
                             float *grad, float *loss)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	if (!c->mlp_ready)
		return fail(c, RENDGPU_ESTATE, "rendgpu_nrc_reset must come first");
	NB_CK(c, cudaSetDevice(c->device));
	return nrc_train(c, feats, reinterpret_cast<const float4 *>(targets), n,
	  update, grad, loss);
}

int rendgpu_relmse_device(struct rdata *rdp, const float *ref, double *out)
{
	Ctx *c = find_ctx(rdp);
	if (!c || !ref || !out)
		return RENDGPU_EINVAL;
	if (!c->have_frame)
		return fail(c, RENDGPU_ESTATE, "rendgpu_resaccum must come first");
	NB_CK(c, cudaSetDevice(c->device));
	uint32_t n = c->W * c->H * 3u;
	NB_CK(c, c->mlp_loss.ensure(1024 * sizeof(float)));
	double *d = reinterpret_cast<double *>(c->mlp_loss.p);
	NB_CK(c, cudaMemsetAsync(d, 0, sizeof(double), c->stream));
	uint32_t samples = c->rd->samples ? c->rd->samples : 1u;
	k_relmse<<<grid_for(c, n, 256), 256, 0, c->stream>>>(c->acc.as<float>(),
	  1.0f / (float)samples, ref, n, d);
	NB_CK(c, cudaGetLastError());
	double h = 0.0;
	NB_CK(c, cudaMemcpyAsync(&h, d, sizeof(double), cudaMemcpyDeviceToHost,
	  c->stream));
	NB_CK(c, cudaStreamSynchronize(c->stream));
	*out = h / (double)n;
	return 0;
}

int rendgpu_sync(struct rdata *rdp)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	NB_CK(c, cudaSetDevice(c->device));
	NB_CK(c, cudaStreamSynchronize(c->stream));
	return 0;
}

int rendgpu_get_stream(struct rdata *rdp, void **stream)
{
	Ctx *c = find_ctx(rdp);
	if (!c || !stream)
		return RENDGPU_EINVAL;
	*stream = (void *)c->stream;
	return 0;
}

int rendgpu_get_stats(struct rdata *rdp, struct rendgpu_stats *st)
{
	Ctx *c = find_ctx(rdp);
	if (!c || !st)
		return RENDGPU_EINVAL;
	c->st.device_bytes = held_bytes(c);
	c->st.max_stack = need_stack(c);
	*st = c->st;
	return 0;
}

int rendgpu_get_lights(struct rdata *rdp, float *out, uint32_t cap,
                       float *total_area)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	if (!c->have_dynamic)
		return fail(c, RENDGPU_ESTATE, "upload_dynamic must come first");
	uint32_t n = (uint32_t)c->host_lights.size();
	if (out) {
		uint32_t m = n < cap ? n : cap;
		std::memcpy(out, c->host_lights.data(), (size_t)m *
		  sizeof(nb_glight));
	}
	if (total_area)
		*total_area = c->light_area;
	return (int)n;
}

int rendgpu_last_error(struct rdata *rdp)
{
	Ctx *c = find_ctx(rdp);
	return c ? c->last : RENDGPU_EINVAL;
}

const char *rendgpu_strerror(struct rdata *rdp)
{
	Ctx *c = find_ctx(rdp);
	return c ? c->msg.c_str() : "no GPU context for this rdata";
}

} // extern "C"
