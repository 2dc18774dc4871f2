// C ABI of the B200 path-tracing core (include/rendgpu.h).
//
// One context per `struct rdata`, found through a small registry keyed by
// the rdata pointer (the reference API passes only that pointer), or one
// context for a batch of rdatas (rendgpu_batch_*): a single-scene context
// is a batch of one.  Uploads convert each scene's reference BVH8 to the GPU
// layout (layout.cpp) and append it to shared arrays with its offsets baked
// in; a frame is the fixed launch sequence of kernels.cuh over all scenes'
// paths on the context's stream, optionally captured once into a CUDA graph
// and replayed.

#include <algorithm>
#include <cfloat>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/rendgpu.h"
#include "kernels.cuh"
#include "layout.hpp"
#include "nrc.cuh"
#include "tlas_build.cuh"
#include "tlas_cta.cuh"

namespace nb {
namespace {

// Traversal stack depths with compiled kernel variants (entries of 8
// bytes per thread in shared memory), and the default trace block size.
constexpr int kStacks[3] = {24, 32, 48};

// Largest instance count whose per-frame TLAS update uses the collapsed
// one-CTA build by default (above it the level-by-level build is cheaper
// per frame than what its tree saves in traversal).
constexpr uint32_t kCollapseMaxInst = 2048;
constexpr int kStackMax = 48;
// A deliberately small stack, compiled for the ray-batch calls only and used
// only when rendgpu_tune.force asks for it: rays whose traversal needs more
// entries are abandoned, which tests the device's overflow handling.
constexpr int kStackForced = 8;
constexpr int kTraceBlock = 256; // +0.6% over 128 on the 1080p workload
constexpr uint32_t kMaxScenes = 4096;
constexpr int kMaxEvents = 512;

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

// One scene of a context: its render data and where its pieces sit in the
// context's shared arrays.
struct SceneHost {
	nb_rdata *rd = nullptr;
	std::unordered_map<uint32_t, uint32_t> root_of; // triofs -> BLAS root
	// triofs -> (first, count) of the BLAS's triangles in the device array
	std::unordered_map<uint32_t, std::pair<uint32_t, uint32_t>> tri_range;
	// triofs -> mesh-local ids of its emissive triangles
	std::unordered_map<uint32_t, std::vector<uint32_t>> emitters;
	uint32_t nrm_base = 0, mtl_base = 0, inst_base = 0, ntri = 0, nmtl = 0;
	uint32_t blas_depth = 0, tlas_depth = 0, tlas_root = 0;
	uint32_t depth = 1;   // max path depth of this scene
	std::vector<nb_glight> lights;
	uint32_t light_off = 0;
	float    light_area = 0.0f;
	// frame layout (rendgpu_resaccum)
	uint32_t W = 0, H = 0, spp = 0;
	uint32_t path_base = 0, pix_base = 0, slot_base = 0, nslots = 0;
	// 8-bit resolve (rendgpu_set_resolve): 0 = the reference's pack
	uint32_t resolve = 0;
	float    exposure = 1.0f;
	NrcBox   nbox{}; // radiance-cache encoding box (rendgpu_upload_dynamic)
};

struct Ctx {
	std::vector<SceneHost> sc;
	nb_rdata    *rd = nullptr;  // sc[0].rd
	bool         batch = false; // created by rendgpu_batch_init
	rendgpu_cfg  cfg{};
	rendgpu_tune tune{};        // 0 fields: defaults
	int          device = 0;
	int          nsm = 148;
	cudaStream_t stream = nullptr;
	// scenes: BLAS nodes and triangles, TLAS nodes and instance refs,
	// instances, normals, materials, lights; scene parameter table
	DevBuf blas, tris, tlas, irefs, insts, nrms, mtls, lights, sp;
	uint32_t blas_depth = 0, tlas_depth = 0; // max over scenes
	bool     have_static = false, have_dynamic = false;
	uint32_t ntris = 0, nnodes = 0, ninst = 0;
	std::vector<ScenePar> par;  // host copy of the table
	// frame: queues (capacity qcap entries), per-path state (npaths)
	DevBuf q0, q1, hits, shadow, scol, pT, pL, rng, acc, buf, cnt, rays, scn;
	DevBuf sortbuf; // ray reordering: key histogram and offsets
	uint32_t npaths = 0, npix = 0, nslots = 0, qcap = 0;
	// two concurrent waves (two_waves): the second half of the camera
	// slots runs on wstream with its own queues and counters, forked from
	// and joined back into `stream`
	bool         two_waves = false;
	bool         dual_frame = false; // the enqueued frame runs both waves
	cudaStream_t wstream = nullptr;
	cudaEvent_t  ev_wfork = nullptr, ev_wjoin = nullptr;
	DevBuf q0b, q1b, hitsb, shadowb, scolb, cntb;
	bool     have_frame = false;
	// captured frame (RENDGPU_FLAG_GRAPH and batches)
	cudaGraphExec_t graph = nullptr;
	bool     capturing = false;
	uint32_t graph_launches = 0, graph_trace_launches = 0;
	std::vector<unsigned long long> scn_host;
	// batch scratch: rays, raw hits, output; berr = [count, errors, work]
	DevBuf brays, braw, bhits, berr;
	// neural radiance cache: FP32 master weights, Adam moments, BF16
	// forward / transposed copies, per-CTA gradient partials and losses
	DevBuf mlp_wf, mlp_m, mlp_v, mlp_wbf, mlp_wbt, mlp_part, mlp_loss;
	DevBuf mlp_act, mlp_dz; // training: layer inputs and output gradients
	// the position hash grid: FP32 table, Adam moments, gradient
	DevBuf grid_t, grid_m, grid_v, grid_g;
	DevBuf qgrid; // the queries' grid features (16 BF16 each)
	// side stream of the grid's training kernels and its fork/join events
	cudaStream_t aux = nullptr;
	cudaEvent_t  ev_fork = nullptr, ev_grad = nullptr, ev_join = nullptr;
	uint32_t mlp_step = 0;
	bool     mlp_ready = false;
	NrcBox   box{};
	DevBuf   nq, nrec, rfeat, rtgt; // radiance-cache frame data
	// deferred training: frame f's records (nrec / nrecb by rec_parity)
	// train the cache on tstream during frame f + 1; nsnap keeps each
	// buffer's record count
	DevBuf       nrecb, nsnap;
	cudaStream_t tstream = nullptr;
	cudaEvent_t  ev_tfork = nullptr, ev_tdone = nullptr;
	bool         train_pending = false;
	uint32_t     rec_parity = 0;
	DevBuf   waitchk;                // rendgpu_check_bounded_wait
	uint32_t nq_cap = 0, nrec_cap = 0, nrc_stride = 1;
	uint32_t nrc_frames = 0; // radiance-cache frames rendered so far
	uint32_t train_grid = 0; // CTAs of the last training step
	// parity capture (rendgpu_capture): per captured bounce, cap_n closest
	// rays, their hits, cap_n shadow rays and 4 counts
	DevBuf   capbuf;
	uint32_t cap_mask = 0, cap_n = 0;
	// device-side scene update (rendgpu_update_instances*): per-instance
	// BLAS root boxes, new matrices, world boxes, TLAS build queues, slot
	// ranges and instance order (refit), build info, emitter sources, area
	DevBuf   dyn_idx, dyn_ctr; // device TLAS build: order, counters
	DevBuf   dyn_bvh;          // single-CTA build: binary tree, tables
	DevBuf   dyn_root, dyn_glob, dyn_wbox, dyn_q, dyn_ranges, dyn_order,
	         dyn_info, dyn_emit, dyn_area, dyn_trange;
	uint32_t dyn_nemit = 0;
	bool     dyn_built = false;  // a device TLAS build ran (refit possible)
	bool     dyn_active = false; // the device holds the current instances
	// stats / errors
	rendgpu_stats st{};
	int          last = 0;
	std::string  msg;
	cudaEvent_t  ev[kMaxEvents] = {};
	int          nev = 0;
};

std::mutex g_mu;
std::unordered_map<const void *, Ctx *> g_ctx;
std::unordered_set<const void *> g_batches; // live rendgpu_batch handles

Ctx *find_batch(const rendgpu_batch *b)
{
	std::lock_guard<std::mutex> lk(g_mu);
	return g_batches.count(b) ? reinterpret_cast<Ctx *>(
	  const_cast<rendgpu_batch *>(b)) : nullptr;
}

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

// Traversal stack of the trace kernels: the tuned depth when it holds the
// deepest TLAS + BLAS chain, else the smallest compiled depth that does
// (0: none does).
int stack_of(const Ctx *c)
{
	if (c->tune.force && c->tune.stack)
		return (int)c->tune.stack; // tests of the overflow handling
	uint32_t need = need_stack(c);
	for (int st : kStacks)
		if ((uint32_t)st == c->tune.stack && need <= (uint32_t)st)
			return st;
	for (int st : kStacks)
		if (need <= (uint32_t)st)
			return st;
	return 0;
}

int block_of(const Ctx *c)
{
	uint32_t b = c->tune.block;
	return b == 64u || b == 128u || b == 256u ? (int)b : kTraceBlock;
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
	S.sp = c->sp.as<ScenePar>();
	S.nscenes = (uint32_t)c->sc.size();
	return S;
}

// Schedule of the trace kernels: tune.sched, else cfg.sched, 1..3; 0 = the
// default, the Ylitie-style schedule (fastest measured on the 1920x1080
// 4 spp workload: 789 vs 664 (step) vs 544 (phase) Mrays/s).
int sched_of(const Ctx *c)
{
	switch (c->tune.sched ? c->tune.sched : c->cfg.sched) {
	case 1: return kSchedStep;
	case 2: return kSchedPhase;
	default: return kSchedYlitie;
	}
}

// Occupancy-sized persistent grid; allows dynamic shared memory above
// 48 KB for the deep-stack variants on first use.
int trace_grid(Ctx *c, const void *fn, int stack, int block)
{
	size_t smem = (size_t)stack * block * sizeof(uint2);
	if (smem > 48 * 1024)
		cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
		  (int)smem);
	int per_sm = 0;
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block,
	  smem) != cudaSuccess || per_sm < 1)
		per_sm = 1;
	return per_sm * c->nsm;
}

template <int SCHED, int STACK, bool COUNT>
void trace_kernel(Ctx *c, const float4 *rays, const uint32_t *count,
                  uint32_t *work, float4 *hits, uint32_t *errs,
                  unsigned long long *nrays)
{
	auto fn = k_trace<SCHED, STACK, COUNT>;
	int block = block_of(c);
	size_t smem = (size_t)STACK * block * sizeof(uint2);
	fn<<<trace_grid(c, (const void *)fn, STACK, block), block, smem,
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

int forced_only(Ctx *c)
{
	return fail(c, RENDGPU_EINVAL, "a forced 8-entry traversal stack serves "
	  "the ray-batch calls only");
}

int too_deep(Ctx *c)
{
	return fail(c, RENDGPU_ELIMIT, "BVH too deep for the traversal stack "
	  "(TLAS + BLAS depth + 2 = " + std::to_string(need_stack(c)) +
	  " > " + std::to_string(kStackMax) + ")");
}

// Launch a closest-hit trace of `count` (device) rays: raw hits.
int launch_trace(Ctx *c, const float4 *rays, const uint32_t *count,
                 uint32_t *work, float4 *hits, uint32_t *errs,
                 unsigned long long *nrays)
{
	switch (stack_of(c)) {
	case kStackForced:
		trace_kernel<kSchedYlitie, kStackForced, false>(c, rays, count, work,
		  hits, errs, nrays);
		break;
	case 24:
		trace_kernel_s<24>(c, rays, count, work, hits, errs, nrays);
		break;
	case 32:
		trace_kernel_s<32>(c, rays, count, work, hits, errs, nrays);
		break;
	case 48:
		trace_kernel_s<48>(c, rays, count, work, hits, errs, nrays);
		break;
	default:
		return too_deep(c);
	}
	NB_CK(c, cudaGetLastError());
	return 0;
}

template <int SCHED, int STACK>
void shadow_kernel(Ctx *c, FrameDev &F, uint32_t k)
{
	auto fn = k_shadow<SCHED, STACK>;
	int block = block_of(c);
	size_t smem = (size_t)STACK * block * sizeof(uint2);
	fn<<<trace_grid(c, (const void *)fn, STACK, block), block, smem,
	  c->stream>>>(scene_of(c), F, k);
}

template <int STACK>
void shadow_kernel_s(Ctx *c, FrameDev &F, uint32_t k)
{
	switch (sched_of(c)) {
	case kSchedPhase:
		shadow_kernel<kSchedPhase, STACK>(c, F, k);
		break;
	case kSchedYlitie:
		shadow_kernel<kSchedYlitie, STACK>(c, F, k);
		break;
	default:
		shadow_kernel<kSchedStep, STACK>(c, F, k);
	}
}

int launch_shadow(Ctx *c, FrameDev &F, uint32_t k)
{
	switch (stack_of(c)) {
	case kStackForced:
		return forced_only(c);
	case 24:
		shadow_kernel_s<24>(c, F, k);
		break;
	case 32:
		shadow_kernel_s<32>(c, F, k);
		break;
	case 48:
		shadow_kernel_s<48>(c, F, k);
		break;
	default:
		return too_deep(c);
	}
	NB_CK(c, cudaGetLastError());
	return 0;
}

template <int STACK, bool COUNT>
void fused_kernel(Ctx *c, FrameDev &F, const float4 *rays,
                  const uint32_t *count, uint32_t ks)
{
	auto fn = k_trace_fused<STACK, COUNT>;
	int block = block_of(c);
	size_t smem = (size_t)STACK * block * sizeof(uint2);
	fn<<<trace_grid(c, (const void *)fn, STACK, block), block, smem,
	  c->stream>>>(scene_of(c), F, rays, count, ks);
}

template <int STACK>
void fused_kernel_s(Ctx *c, FrameDev &F, const float4 *rays,
                    const uint32_t *count, uint32_t ks)
{
	if (c->cfg.flags & RENDGPU_FLAG_COUNT)
		fused_kernel<STACK, true>(c, F, rays, count, ks);
	else
		fused_kernel<STACK, false>(c, F, rays, count, ks);
}

// Closest hits of queue `rays` and the shadow rays of bounce ks in one
// launch.
int launch_fused(Ctx *c, FrameDev &F, const float4 *rays,
                 const uint32_t *count, uint32_t ks)
{
	switch (stack_of(c)) {
	case kStackForced:
		return forced_only(c);
	case 24:
		fused_kernel_s<24>(c, F, rays, count, ks);
		break;
	case 32:
		fused_kernel_s<32>(c, F, rays, count, ks);
		break;
	case 48:
		fused_kernel_s<48>(c, F, rays, count, ks);
		break;
	default:
		return too_deep(c);
	}
	NB_CK(c, cudaGetLastError());
	return 0;
}

template <int STACK>
void occl_kernel(Ctx *c, const float4 *rays, const uint32_t *count,
                 uint32_t *work, uint8_t *occl, uint32_t *errs)
{
	auto fn = k_occluded<kSchedYlitie, STACK>;
	int block = block_of(c);
	size_t smem = (size_t)STACK * block * sizeof(uint2);
	fn<<<trace_grid(c, (const void *)fn, STACK, block), block, smem,
	  c->stream>>>(scene_of(c), rays, count, work, occl, errs);
}

int launch_occluded(Ctx *c, const float4 *rays, const uint32_t *count,
                    uint32_t *work, uint8_t *occl, uint32_t *errs)
{
	switch (stack_of(c)) {
	case kStackForced:
		occl_kernel<kStackForced>(c, rays, count, work, occl, errs);
		break;
	case 24:
		occl_kernel<24>(c, rays, count, work, occl, errs);
		break;
	case 32:
		occl_kernel<32>(c, rays, count, work, occl, errs);
		break;
	case 48:
		occl_kernel<48>(c, rays, count, work, occl, errs);
		break;
	default:
		return too_deep(c);
	}
	NB_CK(c, cudaGetLastError());
	return 0;
}

// Ray reordering applies to single-scene frames without the cache (whose
// query and record order would change with it).
bool sorts(const Ctx *c)
{
	return c->tune.sort && c->sc.size() == 1 &&
	  c->cfg.mode != RENDGPU_MODE_NRC;
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
	F.scn = c->scn.as<unsigned long long>();
	F.npaths = c->npaths;
	F.npix = c->npix;
	F.nq = c->nq.as<float4>();
	F.nrec = (c->rec_parity ? c->nrecb : c->nrec).as<float4>();
	F.nq_cap = c->nq_cap;
	F.nrec_cap = c->nrec_cap;
	F.ncnt = F.cnt + 40;
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
	if (!(c->cfg.flags & RENDGPU_FLAG_TIMING) || c->capturing ||
	  c->nev >= kMaxEvents)
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

// The position hash grid is on unless cfg.reserved[5] bit 0 turns it off
// (the grid features are then zero).
bool nrc_grid(const Ctx *c)
{
	return !(c->cfg.reserved[5] & 1u);
}

const float2 *grid_of(Ctx *c)
{
	return nrc_grid(c) ? c->grid_t.as<float2>() : nullptr;
}

// Xavier-uniform FP32 master weights from a seeded PCG32 stream, zero Adam
// moments, BF16 copies refreshed on the device; the hash grid's entries
// uniform in +-1e-4 from the same stream (as instant-NGP initialises them).
int nrc_reset(Ctx *c, uint64_t seed)
{
	c->train_pending = false; // records of earlier frames no longer train
	if (!c->aux) {
		NB_CK(c, cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking));
		for (cudaEvent_t *e : {&c->ev_fork, &c->ev_grad, &c->ev_join})
			NB_CK(c, cudaEventCreateWithFlags(e, cudaEventDisableTiming));
	}
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
	NB_CK(c, c->grid_t.ensure(kGridParams * sizeof(float)));
	NB_CK(c, c->grid_m.ensure(kGridParams * sizeof(float)));
	NB_CK(c, c->grid_v.ensure(kGridParams * sizeof(float)));
	NB_CK(c, c->grid_g.ensure(kGridParams * sizeof(float)));
	std::vector<float> gt(kGridParams);
	for (float &x : gt)
		x = ((float)(next() >> 8) * 0x1p-24f * 2.0f - 1.0f) * 1e-4f;
	NB_CK(c, cudaMemcpyAsync(c->grid_t.p, gt.data(), gt.size() * 4,
	  cudaMemcpyHostToDevice, c->stream));
	NB_CK(c, cudaMemsetAsync(c->grid_m.p, 0, kGridParams * 4, c->stream));
	NB_CK(c, cudaMemsetAsync(c->grid_v.p, 0, kGridParams * 4, c->stream));
	NB_CK(c, cudaMemsetAsync(c->grid_g.p, 0, kGridParams * 4, c->stream));
	// (pageable sources: the copies have read them when they return)
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
// (cfg.reserved[1]; 0 = 1).  A warm-up frame costs about twice a cache
// frame and barely lowers the error: equal-time time x relMSE measured
// 1.97 / 2.00 / 2.04 / 2.05 for 1 / 2 / 3 / 4 warm-up frames on the 1080p
// scale scene, and 2.89 / 3.12 / 3.55 for 1 / 2 / 4 on the stress scene.
uint32_t nrc_warmup(const Ctx *c)
{
	return c->cfg.reserved[1] ? c->cfg.reserved[1] : 1u;
}

// Bounce at which training paths end in the cache after the warm-up
// (cfg.reserved[2]; 0 = 3, i.e. vertex 4: two recorded vertices of
// unbiased suffix per training path).
uint32_t nrc_train_end(const Ctx *c)
{
	return c->cfg.reserved[2] ? c->cfg.reserved[2] : 3u;
}

constexpr uint32_t kNrcBatch = 16384;    // training samples per Adam step
// Adam steps per frame (cfg.reserved[3]; 0 = 6: on the 1080p scale scene
// 4, 6, 8 and 12 steps measured equal-time relMSE ratios of 1.53, 1.57,
// 1.53 and 1.49)
uint32_t nrc_steps(const Ctx *c)
{
	return c->cfg.reserved[3] ? std::min(c->cfg.reserved[3], 64u) : 6u;
}
// Training paths per frame (cfg.reserved[6]; 0 = 2^16).
uint32_t nrc_train_paths(const Ctx *c)
{
	return c->cfg.reserved[6] ? c->cfg.reserved[6] : 65536u;
}

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
	// about nrc_train_paths training paths, and by default never more than
	// 1 path in 16 (1 in 4 when the count is set)
	c->nrc_stride = std::max(c->cfg.reserved[6] ? 4u : 16u,
	  np / std::max(nrc_train_paths(c), 1u));
	uint32_t verts = c->cfg.max_depth > 1 ? c->cfg.max_depth - 1 : 1;
	// warm-up frames record from every path; later frames overwrite the
	// capacity-limited prefix only, so cap at 4 batches per frame worth of
	// vertices beyond the steady-state need
	uint32_t ntrain = np / c->nrc_stride + 1;
	c->nq_cap = np;
	uint32_t cap = std::max(ntrain * verts + 64, nrc_steps(c) * kNrcBatch);
	if (cap != c->nrec_cap)
		c->train_pending = false; // the record buffers may move
	c->nrec_cap = cap;
	NB_CK(c, c->nq.ensure((size_t)np * 64));
	NB_CK(c, c->nrec.ensure((size_t)c->nrec_cap * 96));
	NB_CK(c, c->nrecb.ensure((size_t)c->nrec_cap * 96));
	NB_CK(c, c->nsnap.ensure(2 * sizeof(uint32_t)));
	if (!c->tstream) {
		NB_CK(c, cudaStreamCreateWithFlags(&c->tstream,
		  cudaStreamNonBlocking));
		for (cudaEvent_t *e : {&c->ev_tfork, &c->ev_tdone})
			NB_CK(c, cudaEventCreateWithFlags(e, cudaEventDisableTiming));
	}
	NB_CK(c, c->rfeat.ensure((size_t)c->nrec_cap * 128));
	NB_CK(c, c->rtgt.ensure((size_t)c->nrec_cap * 16));
	return 0;
}

// Null or not 16-byte aligned (vector loads, cp.async and float4 stores
// of the cache kernels need 16 bytes).
inline bool misaligned16(const void *p)
{
	return !p || (reinterpret_cast<uintptr_t>(p) & 15u) != 0;
}

// Inference kernel of one kind: dynamic shared memory set once, one CTA
// of kTcGroups tile pipelines per SM (the whole register file).
template <bool Q>
int fwd_tc_setup(Ctx *c, uint32_t n, uint32_t *grid, size_t *smem)
{
	*smem = sizeof(MlpTcSmem) + 1024; // + alignment slack
	NB_CK(c, cudaFuncSetAttribute(k_mlp_fwd_tc<Q>,
	  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem));
	uint32_t tiles = (n + (uint32_t)kTcRows - 1u) / (uint32_t)kTcRows;
	*grid = std::max(std::min<uint32_t>((tiles + kTcGroups - 1u) / kTcGroups,
	  (uint32_t)c->nsm), 1u);
	return 0;
}

// Forward pass of n queries' features on the tcgen05 tensor cores; a
// timed-out wait on the device counts into the device error word.
int nrc_infer(Ctx *c, const void *feats, uint32_t n, float4 *out)
{
	if (n == 0)
		return 0;
	uint32_t grid;
	size_t smem;
	int rc = fwd_tc_setup<false>(c, n, &grid, &smem);
	if (rc)
		return rc;
	k_mlp_fwd_tc<false><<<grid, kTcThreads, smem, c->stream>>>(
	  c->mlp_wbf.as<__nv_bfloat16>(), static_cast<const __nv_bfloat16 *>(feats),
	  n, out, nullptr, c->berr.as<uint32_t>() + 1, nullptr, c->box, nullptr,
	  0u, false, nullptr);
	NB_CK(c, cudaGetLastError());
	return 0;
}

// Identity encoding box: the frame's entries carry positions k_shade has
// mapped into their scene's box already (with the scene's feature code).
constexpr NrcBox kUnitBox = {{0.0f, 0.0f, 0.0f}, {1.0f, 1.0f, 1.0f}};

// Cache queries (min(*count, cap) entries of 4 float4, made on the device):
// encode, infer and add each output to its path's radiance in one kernel.
// frame: entries written by k_shade (positions in their scene's box, scene
// features); else world positions in the context's box.
int nrc_query(Ctx *c, const float4 *q, const uint32_t *count, uint32_t cap,
              float4 *pL, uint32_t npath, uint32_t *errs, bool frame)
{
	if (cap == 0)
		return 0;
	uint32_t grid;
	size_t smem;
	int rc = fwd_tc_setup<true>(c, cap, &grid, &smem);
	if (rc)
		return rc;
	NrcBox box = frame ? kUnitBox : c->box;
	const uint4 *gq = nullptr;
	if (nrc_grid(c)) {
		// the queries' grid features first, gathered at full occupancy
		NB_CK(c, c->qgrid.ensure((size_t)cap * 32));
		k_grid_query_feats<<<grid_for(c, cap * (uint32_t)kGridLevels, 256),
		  256, 0, c->stream>>>(q, count, cap, box, frame, grid_of(c),
		  c->qgrid.as<uint32_t>());
		NB_CK(c, cudaGetLastError());
		gq = c->qgrid.as<uint4>();
	}
	k_mlp_fwd_tc<true><<<grid, kTcThreads, smem, c->stream>>>(
	  c->mlp_wbf.as<__nv_bfloat16>(), nullptr, cap, nullptr, count, errs, q,
	  box, pL, npath, frame, gq);
	NB_CK(c, cudaGetLastError());
	return 0;
}

// Where a training batch's positions come from, for the hash grid's
// gradient: entries of `stride` float4s (selected as the batch's rows are,
// with the device count) or raw inputs of 12 floats per row; their box and
// scene-code flag as the encoding used them.  g_out (kGridParams floats)
// receives the grid's gradient when not null.
struct GridSrc {
	const float4 *e = nullptr;
	const float  *raw = nullptr;
	uint32_t      stride = 0;
	NrcBox        box{};
	bool          scode = false;
	float        *g_out = nullptr;
};

// Gradient of a batch (and optionally one Adam step).  g_out (device,
// kMlpParams floats) receives the summed gradient when not null; *loss the
// batch loss when not null (synchronises).  With gs (and the grid on) the
// hash grid gets its gradient and Adam step too.
int nrc_train(Ctx *c, const void *feats, const float4 *targets, uint32_t n,
              int update, float *g_out, float *loss,
              const uint32_t *ncount = nullptr, uint32_t offset = 0,
              uint32_t cap = 0, const GridSrc *gs = nullptr)
{
	if (n == 0)
		return 0;
	size_t smem = sizeof(MlpFbSmem) + 1024; // + alignment slack
	NB_CK(c, cudaFuncSetAttribute(k_mlp_fb_tc,
	  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
	// pass 1: forward + backward of 128-row tiles on tcgen05, one tile
	// pipeline per CTA, one CTA per SM
	uint32_t npad = (n + 15u) / 16u * 16u;
	uint32_t tiles = (npad + (uint32_t)kFbRows - 1u) / (uint32_t)kFbRows;
	uint32_t grid = std::max(std::min<uint32_t>(tiles, (uint32_t)c->nsm), 1u);
	NB_CK(c, c->mlp_act.ensure((size_t)6 * npad * 64 * 2));
	NB_CK(c, c->mlp_dz.ensure((size_t)6 * npad * 64 * 2));
	c->train_grid = grid;
	k_mlp_fb_tc<<<grid, kFbRows, smem, c->stream>>>(
	  c->mlp_wbf.as<__nv_bfloat16>(), c->mlp_wbt.as<__nv_bfloat16>(),
	  static_cast<const __nv_bfloat16 *>(feats), targets, n, npad,
	  c->mlp_act.as<__nv_bfloat16>(), c->mlp_dz.as<__nv_bfloat16>(),
	  c->mlp_loss.as<float>(), ncount, offset, cap,
	  c->berr.as<uint32_t>() + 1);
	NB_CK(c, cudaGetLastError());
	if (update)
		c->mlp_step++;
	float bc1 = 1.0f - std::pow(kAdamBeta1, (float)std::max(c->mlp_step, 1u));
	float bc2 = 1.0f - std::pow(kAdamBeta2, (float)std::max(c->mlp_step, 1u));
	// the grid's gradient and Adam step on the side stream, beside pass 2
	// and the MLP's step (they read pass 1's outputs and write only the
	// grid); the MLP's step waits for the gradient, which reads this
	// forward pass's BF16 W0, and the caller's next work for the grid
	bool with_grid = gs && nrc_grid(c) && (gs->e || gs->raw) && c->aux;
	if (with_grid) {
		NB_CK(c, cudaEventRecord(c->ev_fork, c->stream));
		NB_CK(c, cudaStreamWaitEvent(c->aux, c->ev_fork, 0));
		k_grid_grad<<<grid_for(c, n * (uint32_t)kGridLevels, 256), 256, 0,
		  c->aux>>>(gs->e, gs->raw, gs->stride, ncount, offset, cap, n,
		  gs->box, gs->scode, c->mlp_dz.as<__nv_bfloat16>(),
		  c->mlp_wbf.as<__nv_bfloat16>(), c->grid_g.as<float2>());
		NB_CK(c, cudaGetLastError());
		NB_CK(c, cudaEventRecord(c->ev_grad, c->aux));
		k_grid_adam<<<grid_for(c, kGridParams / 4, 256), 256, 0,
		  c->aux>>>(c->grid_t.as<float4>(), c->grid_m.as<float4>(),
		  c->grid_v.as<float4>(), c->grid_g.as<float4>(),
		  reinterpret_cast<float4 *>(gs->g_out), update, nrc_lr(c),
		  kAdamBeta1, kAdamBeta2, kAdamEps, bc1, bc2);
		NB_CK(c, cudaGetLastError());
		NB_CK(c, cudaEventRecord(c->ev_join, c->aux));
	}
	// pass 2: split-K weight-gradient UMMAs, (splits x 6 layers) CTAs
	uint32_t chunks = (npad + (uint32_t)kDwChunk - 1u) / (uint32_t)kDwChunk;
	uint32_t splits = std::min<uint32_t>(32u, chunks);
	uint32_t rows_per = (chunks + splits - 1u) / splits * (uint32_t)kDwChunk;
	splits = (npad + rows_per - 1u) / rows_per;
	NB_CK(c, c->mlp_part.ensure((size_t)splits * kMlpParams * sizeof(float)));
	size_t dsmem = sizeof(MlpDwSmem) + 1024; // + alignment slack
	NB_CK(c, cudaFuncSetAttribute(k_mlp_dw_tc,
	  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsmem));
	k_mlp_dw_tc<<<dim3(splits, kMlpSquare + 1), 128, dsmem, c->stream>>>(
	  c->mlp_act.as<__nv_bfloat16>(), c->mlp_dz.as<__nv_bfloat16>(), npad,
	  rows_per, c->mlp_part.as<float>(), c->berr.as<uint32_t>() + 1);
	NB_CK(c, cudaGetLastError());
	if (with_grid)
		NB_CK(c, cudaStreamWaitEvent(c->stream, c->ev_grad, 0));
	k_mlp_adam<<<grid_for(c, kMlpParams, 256), 256, 0, c->stream>>>(
	  c->mlp_wf.as<float>(), c->mlp_m.as<float>(), c->mlp_v.as<float>(),
	  c->mlp_part.as<float>(), (int)splits, g_out, update, nrc_lr(c),
	  kAdamBeta1, kAdamBeta2, kAdamEps, bc1, bc2,
	  c->mlp_wbf.as<__nv_bfloat16>(), c->mlp_wbt.as<__nv_bfloat16>());
	NB_CK(c, cudaGetLastError());
	if (with_grid)
		NB_CK(c, cudaStreamWaitEvent(c->stream, c->ev_join, 0));
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

// Scene parameter table of this frame from each scene's render data (its
// camera, frame number, sizes and lights); uploaded to the device.
int frame_params(Ctx *c, bool nrc, FrameArgs *A)
{
	size_t n = c->sc.size();
	c->par.assign(n, ScenePar{});
	A->mode = c->cfg.mode;
	A->depth = 1;
	// after the warm-up, cache frames end every path by bounce nrc_end
	bool self_train = nrc && c->nrc_frames >= nrc_warmup(c);
	A->nrc_end = self_train ? nrc_train_end(c) : 0xffffffffu;
	for (size_t i = 0; i < n; i++) {
		const SceneHost &h = c->sc[i];
		const nb_rdata *rd = h.rd;
		if (rd->width != h.W || rd->height != h.H ||
		  (rd->spp ? rd->spp : 1u) != h.spp)
			return fail(c, RENDGPU_ESTATE, "rdata size changed since "
			  "rendgpu_resaccum");
		ScenePar &P = c->par[i];
		P.tlas_root = h.tlas_root;
		P.light_off = h.light_off;
		P.light_cnt = (uint32_t)h.lights.size();
		P.depth = c->cfg.mode == RENDGPU_MODE_PRIMARY ? 1u : h.depth;
		if (self_train)
			P.depth = std::min(P.depth, A->nrc_end + 1u);
		A->depth = std::max(A->depth, P.depth);
		P.W = h.W;
		P.H = h.H;
		P.spp = h.spp;
		P.frame = rd->samples;
		P.path_base = h.path_base;
		P.pix_base = h.pix_base;
		P.slot_base = h.slot_base;
		P.nrc_stride = 1;
		P.nrc_offset = 0;
		if (nrc) {
			// warm-up: the first frames trace every path unbiased (as
			// training paths) while the cache trains
			P.nrc_stride = c->nrc_frames < nrc_warmup(c) ? 1u :
			  c->nrc_stride;
			P.nrc_offset = (rd->samples * 7919u) % P.nrc_stride;
		}
		P.light_area = h.light_area;
		P.inv = 1.0f / (float)(rd->samples + rd->spp);
		P.resolve = h.resolve;
		P.exposure = h.exposure;
		// one cache serves a batch: each scene in its own box, scenes
		// 2..15 with a feature of their own (scene 16 shares scene 2's)
		for (int a = 0; a < 3; a++) {
			P.nrc_lo[a] = h.nbox.lo[a];
			P.nrc_inv[a] = h.nbox.inv[a];
		}
		P.nrc_off = i == 0 ? 0.0f : (float)(2u * ((uint32_t)(i - 1) % 14u +
		  1u));
		P.bg[0] = rd->bgcol.x;
		P.bg[1] = rd->bgcol.y;
		P.bg[2] = rd->bgcol.z;
		const nb_rcam &cam = rd->cam;
		P.eye[0] = cam.eye.x; P.eye[1] = cam.eye.y; P.eye[2] = cam.eye.z;
		P.ri[0] = cam.ri.x; P.ri[1] = cam.ri.y; P.ri[2] = cam.ri.z;
		P.up[0] = cam.up.x; P.up[1] = cam.up.y; P.up[2] = cam.up.z;
		P.fwd[0] = cam.fwd.x; P.fwd[1] = cam.fwd.y; P.fwd[2] = cam.fwd.z;
		P.rw = cam.rw8[0];
		P.rh = cam.rh8[0];
		P.fovfdist = cam.fovfdist8[0];
		P.aspect = cam.aspect8[0];
		P.fdist = cam.fdist8[0];
		P.focrad = cam.focrad8[0];
		P.tanfangle = cam.tanfangle;
		P.seed = c->cfg.seed;
	}
	NB_CK(c, cudaMemcpyAsync(c->sp.p, c->par.data(), n * sizeof(ScenePar),
	  cudaMemcpyHostToDevice, c->stream));
	if (c->dyn_active)
		// the light area of the last device-side update
		NB_CK(c, cudaMemcpyAsync(&c->sp.as<ScenePar>()[0].light_area,
		  c->dyn_area.p, sizeof(float), cudaMemcpyDeviceToDevice,
		  c->stream));
	return 0;
}

void drop_graph(Ctx *c)
{
	if (c->graph)
		cudaGraphExecDestroy(c->graph);
	c->graph = nullptr;
}

// Where the capture of bounce k sits in capbuf: closest rays (cap_n x 32 B),
// their hits (cap_n x 16 B), shadow rays (cap_n x 32 B), 4 counts.
struct CapSlot {
	float4   *rays, *hits, *shadow;
	uint32_t *counts;
};

size_t cap_slot_bytes(uint32_t cap)
{
	return (size_t)cap * 80 + 16;
}

CapSlot cap_slot(const Ctx *c, uint32_t k)
{
	uint32_t s = (uint32_t)__builtin_popcount(c->cap_mask & ((1u << k) - 1u));
	unsigned char *b = c->capbuf.as<unsigned char>() + s *
	  cap_slot_bytes(c->cap_n);
	size_t n = c->cap_n;
	return CapSlot{reinterpret_cast<float4 *>(b),
	  reinterpret_cast<float4 *>(b + n * 32),
	  reinterpret_cast<float4 *>(b + n * 48),
	  reinterpret_cast<uint32_t *>(b + n * 80)};
}

bool captures(const Ctx *c, uint32_t k)
{
	return c->cap_n && k < 32u && ((c->cap_mask >> k) & 1u);
}

// Event indices of the per-kernel timing of one directly launched frame.
struct FrameEvents {
	std::vector<int> trace, shadow;
	int nrc = -1, train = -1;
};

// nrc_steps Adam steps of kNrcBatch training records each from `recs`
// (*count records, targets in rtgt) on c->stream: each step encodes its
// batch with the grid as the last step left it, trains, and moves the grid
// with its own gradient.
int train_records(Ctx *c, const float4 *recs, const uint32_t *count,
                  FrameEvents *E)
{
	E->train = c->nev;
	ev_record(c);
	GridSrc gs;
	gs.e = recs;
	gs.stride = 6u;
	gs.box = kUnitBox;
	gs.scode = true;
	for (uint32_t s = 0; s < nrc_steps(c); s++) {
		k_nrc_encode_entries<<<grid_for(c, kNrcBatch, 128), 128, 0,
		  c->stream>>>(recs, 6u, count, s * kNrcBatch, c->nrec_cap,
		  kNrcBatch, kUnitBox, c->rfeat.as<__nv_bfloat16>(), true,
		  grid_of(c));
		NB_CK(c, cudaGetLastError());
		int rc = nrc_train(c, c->rfeat.p, c->rtgt.as<float4>(), kNrcBatch,
		  1, nullptr, nullptr, count, s * kNrcBatch, c->nrec_cap, &gs);
		if (rc)
			return rc;
	}
	c->st.launches += (nrc_grid(c) ? 6 : 4) * nrc_steps(c);
	ev_record(c);
	return 0;
}

// The launch sequence of one frame: every wave of camera slots through all
// bounces (trace, shade, shadow), cache inference, accumulation, cache
// training.  Sizes and counts are read on the device, so the sequence is
// the same every frame and can be captured once.
int enqueue_frame(Ctx *c, const FrameDev &F, const FrameArgs &A,
                  bool nrc, FrameEvents *E)
{
	DScene S = scene_of(c);
	int rc = 0;
	// reordering: rays are traced and shaded from q[0]; shading appends
	// to q[1], which is sorted back into q[0]
	bool sorting = sorts(c);
	// shadow rays of bounce k traced with the closest hits of bounce k + 1
	bool fused = A.mode != RENDGPU_MODE_PRIMARY && c->tune.fuse != 2u &&
	  sched_of(c) == kSchedYlitie;
	uint32_t *hist = c->sortbuf.as<uint32_t>();
	c->st.launches = 0;
	c->st.trace_launches = 0;
	NB_CK(c, cudaMemsetAsync(c->cnt.p, 0, 64 * sizeof(uint32_t), c->stream));
	NB_CK(c, cudaMemsetAsync(c->rays.p, 0, 4 * sizeof(unsigned long long),
	  c->stream));
	NB_CK(c, cudaMemsetAsync(c->scn.p, 0, c->sc.size() * 2 *
	  sizeof(unsigned long long), c->stream));
	ev_record(c); // 0
	// The previous frame's records train the cache on tstream, forked after
	// this frame's bounce-1 launches so that the training kernels take the
	// SMs the traversal's tails leave idle; the queries wait for it.  Every
	// frame's queries thus see the cache trained on all earlier frames, as
	// when each frame trained at its end.
	bool train_enq = false;
	auto deferred_train = [&]() -> int {
		if (!nrc || !c->train_pending || train_enq)
			return 0;
		train_enq = true;
		const float4 *prev = (c->rec_parity ? c->nrec : c->nrecb).as<float4>();
		const uint32_t *pcnt = c->nsnap.as<uint32_t>() + (c->rec_parity ^ 1u);
		NB_CK(c, cudaEventRecord(c->ev_tfork, c->stream));
		NB_CK(c, cudaStreamWaitEvent(c->tstream, c->ev_tfork, 0));
		cudaStream_t main = c->stream;
		c->stream = c->tstream;
		int r = train_records(c, prev, pcnt, E);
		if (r == 0 && cudaEventRecord(c->ev_tdone, c->tstream) !=
		  cudaSuccess)
			r = fail(c, RENDGPU_ECUDA, "cudaEventRecord (training done)");
		c->stream = main;
		return r;
	};
	// camera rays of slots [lo, hi) of wave W
	auto gen = [&](const FrameDev &W, uint32_t lo, uint32_t hi) -> int {
		NB_CK(c, cudaMemsetAsync(W.cnt, 0, sizeof(uint32_t), c->stream));
		k_gen<<<grid_for(c, hi - lo, 256), 256, 0, c->stream>>>(S, W, A, lo,
		  hi);
		NB_CK(c, cudaGetLastError());
		c->st.launches++;
		return 0;
	};
	// bounce k of wave W (slots [lo, hi)): trace, shade, shadow rays
	auto bounce = [&](FrameDev &F, uint32_t lo, uint32_t hi,
	  uint32_t k) -> int {
		uint32_t cur = sorting ? 0u : (k & 1u);
		E->trace.push_back(c->nev);
		ev_record(c);
		if (fused && k > 0u)
			rc = launch_fused(c, const_cast<FrameDev &>(F), F.q[cur],
			  F.cnt + cur, k - 1u);
		else
			rc = launch_trace(c, F.q[cur], F.cnt + cur, F.cnt + 4,
			  F.hits, F.cnt + 3, F.rays);
		if (rc)
			return rc;
		ev_record(c);
		c->st.launches++;
		c->st.trace_launches++;
		bool cap = lo == 0u && captures(c, k);
		if (cap) {
			// the frame's own closest hits of bounce k
			CapSlot cs = cap_slot(c, k);
			k_capture<<<grid_for(c, c->cap_n, 256), 256, 0,
			  c->stream>>>(S, F.q[cur], F.cnt + cur, F.hits, c->cap_n,
			  cs.rays, cs.hits, cs.counts);
			NB_CK(c, cudaGetLastError());
			c->st.launches++;
		}
		NB_CK(c, cudaMemsetAsync(F.cnt + (cur ^ 1u), 0,
		  sizeof(uint32_t), c->stream));
		NB_CK(c, cudaMemsetAsync(F.cnt + 2, 0, sizeof(uint32_t),
		  c->stream));
		k_shade<<<grid_for(c, hi - lo, 256), 256, 0, c->stream>>>(S, F,
		  A, cur, k);
		NB_CK(c, cudaGetLastError());
		c->st.launches++;
		if (cap) {
			// the shadow rays shading generated at bounce k
			CapSlot cs = cap_slot(c, k);
			k_capture<<<grid_for(c, c->cap_n, 256), 256, 0,
			  c->stream>>>(S, F.shadow, F.cnt + 2, nullptr, c->cap_n,
			  cs.shadow, nullptr, cs.counts + 2);
			NB_CK(c, cudaGetLastError());
			c->st.launches++;
		}
		if (A.mode != RENDGPU_MODE_PRIMARY &&
		  (!fused || k + 1u == A.depth)) {
			E->shadow.push_back(c->nev);
			ev_record(c);
			rc = launch_shadow(c, const_cast<FrameDev &>(F), k);
			if (rc)
				return rc;
			ev_record(c);
			c->st.launches++;
		}
		if (sorting && k + 1u < A.depth) {
			int g = grid_for(c, hi - lo, 256);
			k_sort_hist<<<g, 256, 0, c->stream>>>(F.q[1], F.cnt + 1,
			  c->box, hist);
			k_sort_scan<<<1, 1024, 0, c->stream>>>(hist,
			  hist + kSortKeys);
			k_sort_scatter<<<g, 256, 0, c->stream>>>(F.q[1], F.cnt + 1,
			  c->box, hist + kSortKeys, F.q[0], F.cnt);
			NB_CK(c, cudaGetLastError());
			c->st.launches += 3;
		}
		if (nrc && k == 1u && lo == 0u)
			return deferred_train();
		return 0;
	};
	// the second half of the slots on wstream, concurrently (two_waves)
	bool dual = c->two_waves && !sorting && c->wstream &&
	  c->nslots > c->qcap;
	c->dual_frame = dual;
	if (dual) {
		FrameDev F1 = F;
		F1.q[0] = c->q0b.as<float4>();
		F1.q[1] = c->q1b.as<float4>();
		F1.hits = c->hitsb.as<float4>();
		F1.shadow = c->shadowb.as<float4>();
		F1.scol = c->scolb.as<float4>();
		F1.cnt = c->cntb.as<uint32_t>();
		FrameDev F0 = F;
		NB_CK(c, cudaMemsetAsync(F1.cnt, 0, 64 * sizeof(uint32_t),
		  c->stream));
		NB_CK(c, cudaEventRecord(c->ev_wfork, c->stream));
		NB_CK(c, cudaStreamWaitEvent(c->wstream, c->ev_wfork, 0));
		cudaStream_t main = c->stream;
		uint32_t mid = c->qcap;
		// launches alternate between the waves bounce by bounce (starting
		// the second wave a bounce later, so that the first wave's short
		// training-path bounces of a radiance-cache frame ran beside the
		// second's bounce 1, measured 3% slower cache frames)
		for (uint32_t k = 0; rc == 0 && k <= A.depth; k++) {
			for (int w = 0; rc == 0 && w < 2; w++) {
				c->stream = w ? c->wstream : main;
				uint32_t lo = w ? mid : 0u, hi = w ? c->nslots : mid;
				FrameDev &W = w ? F1 : F0;
				rc = k == 0 ? gen(W, lo, hi) : bounce(W, lo, hi, k - 1u);
			}
		}
		c->stream = c->wstream;
		if (rc == 0 && cudaEventRecord(c->ev_wjoin, c->wstream) !=
		  cudaSuccess)
			rc = fail(c, RENDGPU_ECUDA, "cudaEventRecord (wave join)");
		c->stream = main;
		if (rc)
			return rc;
		NB_CK(c, cudaStreamWaitEvent(main, c->ev_wjoin, 0));
	} else {
		for (uint32_t lo = 0; lo < c->nslots; lo += c->qcap) {
			uint32_t hi = std::min(c->nslots, lo + c->qcap);
			rc = gen(F, lo, hi);
			for (uint32_t k = 0; rc == 0 && k < A.depth; k++)
				rc = bounce(const_cast<FrameDev &>(F), lo, hi, k);
			if (rc)
				return rc;
		}
	}
	if (nrc) {
		rc = deferred_train(); // frames of fewer than two bounces
		if (rc)
			return rc;
		if (train_enq)
			NB_CK(c, cudaStreamWaitEvent(c->stream, c->ev_tdone, 0));
		// cache inference for the queries of this frame
		E->nrc = c->nev;
		ev_record(c);
		rc = nrc_query(c, F.nq, F.cnt + 40, c->nq_cap, F.pL, c->npaths,
		  F.cnt + 3, true);
		if (rc)
			return rc;
		c->st.launches += nrc_grid(c) ? 2 : 1;
		ev_record(c);
	}
	k_accum<<<grid_for(c, c->npix, 256), 256, 0, c->stream>>>(S, F);
	NB_CK(c, cudaGetLastError());
	c->st.launches++;
	if (nrc) {
		// targets of this frame's records from the finished paths (before
		// the next frame's camera rays reset the path radiance) and the
		// record count; the next frame trains on them
		k_nrc_targets<<<grid_for(c, c->nrec_cap, 256), 256, 0, c->stream>>>(
		  F.nrec, F.cnt + 41, c->nrec_cap, F.pL, c->rtgt.as<float4>());
		NB_CK(c, cudaGetLastError());
		NB_CK(c, cudaMemcpyAsync(c->nsnap.as<uint32_t>() + c->rec_parity,
		  F.cnt + 41, sizeof(uint32_t), cudaMemcpyDeviceToDevice,
		  c->stream));
		c->st.launches++;
	}
	ev_record(c); // last
	return 0;
}

// Capture the frame's launch sequence into a graph (once per layout).
int capture_frame(Ctx *c, const FrameDev &F, const FrameArgs &A)
{
	FrameEvents E;
	NB_CK(c, cudaStreamBeginCapture(c->stream,
	  cudaStreamCaptureModeRelaxed));
	c->capturing = true;
	int rc = enqueue_frame(c, F, A, false, &E);
	c->capturing = false;
	cudaGraph_t g = nullptr;
	cudaError_t e = cudaStreamEndCapture(c->stream, &g);
	if (rc) {
		if (g)
			cudaGraphDestroy(g);
		return rc;
	}
	if (e != cudaSuccess)
		return cuda_fail(c, e, "cudaStreamEndCapture");
	e = cudaGraphInstantiate(&c->graph, g, 0);
	cudaGraphDestroy(g);
	if (e != cudaSuccess) {
		c->graph = nullptr;
		return cuda_fail(c, e, "cudaGraphInstantiate");
	}
	c->graph_launches = c->st.launches;
	c->graph_trace_launches = c->st.trace_launches;
	return 0;
}

bool use_graph(const Ctx *c)
{
	return c->cfg.mode != RENDGPU_MODE_NRC &&
	  (c->batch || (c->cfg.flags & RENDGPU_FLAG_GRAPH));
}

int render_frame(Ctx *c)
{
	int rc = ready(c, true);
	if (rc)
		return rc;
	bool nrc = c->cfg.mode == RENDGPU_MODE_NRC;
	if (nrc) {
		rc = nrc_frame_buffers(c);
		if (rc)
			return rc;
	}
	FrameArgs A;
	rc = frame_params(c, nrc, &A);
	if (rc)
		return rc;
	if (nrc)
		c->nrc_frames++;
	FrameDev F = frame_of(c);
	c->nev = 0;
	FrameEvents E;
	bool graph = use_graph(c);
	if (graph) {
		if (!c->graph) {
			rc = capture_frame(c, F, A);
			if (rc)
				return rc;
		}
		ev_record(c);
		NB_CK(c, cudaGraphLaunch(c->graph, c->stream));
		ev_record(c);
		c->st.launches = c->graph_launches;
		c->st.trace_launches = c->graph_trace_launches;
	} else {
		rc = enqueue_frame(c, F, A, nrc, &E);
		if (rc) {
			c->train_pending = false;
			return rc;
		}
	}
	// radiance cache: this frame's records train during the next frame
	bool trained = nrc && E.train >= 0;
	uint32_t tpar = c->rec_parity ^ 1u; // the buffer trained this frame
	if (nrc) {
		c->train_pending = true;
		c->rec_parity ^= 1u;
	}
	unsigned long long hr[4];
	uint32_t hc[64];
	size_t ns = c->sc.size();
	c->scn_host.assign(2 * ns, 0ull);
	NB_CK(c, cudaMemcpyAsync(hr, c->rays.p, sizeof(hr),
	  cudaMemcpyDeviceToHost, c->stream));
	NB_CK(c, cudaMemcpyAsync(hc, c->cnt.p, sizeof(hc),
	  cudaMemcpyDeviceToHost, c->stream));
	uint32_t hcb[64] = {};
	if (c->dual_frame)
		NB_CK(c, cudaMemcpyAsync(hcb, c->cntb.p, sizeof(hcb),
		  cudaMemcpyDeviceToHost, c->stream));
	if (ns > 1)
		NB_CK(c, cudaMemcpyAsync(c->scn_host.data(), c->scn.p, 2 * ns *
		  sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
	NB_CK(c, cudaStreamSynchronize(c->stream));
	// the second wave's errors and per-bounce ray counts
	hc[3] += hcb[3];
	for (int k = 0; k < 16; k++) {
		hc[8 + k] += hcb[8 + k];
		hc[24 + k] += hcb[24 + k];
	}
	c->st.closest_rays = hr[0];
	c->st.node_visits = hr[2];
	c->st.tri_tests = hr[3];
	c->st.shadow_rays = hr[1];
	c->st.rays = hr[0] + hr[1];
	c->st.device_errors = hc[3];
	if (ns == 1) {
		c->scn_host[0] = hr[0];
		c->scn_host[1] = hr[1];
	}
	c->st.nrc_loss = 0.0f;
	if (trained) {
		// loss of the last Adam step (partials of its CTAs) over the
		// previous frame's records, which trained in this frame (the
		// queries waited for it, and the stream has been synchronised)
		float lp[1024];
		uint32_t ng = std::min<uint32_t>(c->train_grid, 1024);
		uint32_t tcnt = 0;
		NB_CK(c, cudaMemcpy(lp, c->mlp_loss.p, ng * 4,
		  cudaMemcpyDeviceToHost));
		NB_CK(c, cudaMemcpy(&tcnt, c->nsnap.as<uint32_t>() + tpar,
		  sizeof(tcnt), cudaMemcpyDeviceToHost));
		double sl = 0.0;
		for (uint32_t i = 0; i < ng; i++)
			sl += lp[i];
		uint32_t used = std::min(std::min(tcnt, c->nrec_cap), kNrcBatch);
		c->st.nrc_loss = used ? (float)(sl / (3.0 * used)) : 0.0f;
	}
	c->st.nrc_queries = nrc ? std::min(hc[40], c->nq_cap) : 0;
	c->st.nrc_records = nrc ? std::min(hc[41], c->nrec_cap) : 0;
	for (int k = 0; k < 16; k++) {
		c->st.bounce_closest[k] = hc[8 + k];
		c->st.bounce_shadow[k] = hc[24 + k];
	}
	c->st.max_stack = (uint32_t)stack_of(c);
	if (c->cfg.flags & RENDGPU_FLAG_TIMING) {
		c->st.ms_frame = ev_ms(c, 0, c->nev - 1);
		float tr = 0.0f, sh = 0.0f;
		for (int e : E.trace)
			tr += ev_ms(c, e, e + 1);
		for (int e : E.shadow)
			sh += ev_ms(c, e, e + 1);
		c->st.ms_trace = tr;
		c->st.ms_shadow = sh;
		c->st.ms_nrc = nrc ? ev_ms(c, E.nrc, E.nrc + 1) +
		  (trained ? ev_ms(c, E.train, E.train + 1) : 0.0f) : 0.0f;
		// (with two concurrent waves the launches overlap, so their sum
		// can exceed the frame and no shading time is derived)
		c->st.ms_shade = graph || c->dual_frame ? 0.0f :
		  std::max(0.0f, c->st.ms_frame - tr - sh - c->st.ms_nrc);
	}
	if (hc[3])
		return fail(c, RENDGPU_EDEVICE, "device error: rays abandoned "
		  "(traversal stack overflow) or a tensor-core wait timed out");
	return 0;
}

void free_ctx(Ctx *c)
{
	drop_graph(c);
	DevBuf *bufs[] = {&c->blas, &c->tris, &c->tlas, &c->irefs, &c->insts,
	  &c->nrms, &c->mtls, &c->lights, &c->sp, &c->scn, &c->sortbuf, &c->q0, &c->q1, &c->hits, &c->shadow,
	  &c->scol, &c->pT, &c->pL, &c->rng, &c->acc, &c->buf, &c->cnt,
	  &c->rays, &c->brays, &c->braw, &c->bhits, &c->berr, &c->mlp_act,
	  &c->mlp_dz, &c->mlp_wf, &c->grid_t, &c->grid_m, &c->grid_v,
	  &c->grid_g, &c->qgrid,
	  &c->mlp_m, &c->mlp_v, &c->mlp_wbf, &c->mlp_wbt, &c->mlp_part,
	  &c->mlp_loss, &c->nq, &c->nrec, &c->rfeat, &c->waitchk,
	  &c->rtgt, &c->capbuf, &c->dyn_root, &c->dyn_glob, &c->dyn_wbox,
	  &c->dyn_q, &c->dyn_ranges, &c->dyn_order, &c->dyn_info, &c->dyn_emit,
	  &c->dyn_area, &c->dyn_trange, &c->dyn_idx, &c->dyn_ctr, &c->dyn_bvh,
	  &c->q0b,
	  &c->q1b, &c->hitsb, &c->shadowb, &c->scolb, &c->cntb, &c->nrecb,
	  &c->nsnap};
	for (DevBuf *b : bufs)
		b->release();
	for (int i = 0; i < kMaxEvents; i++)
		if (c->ev[i])
			cudaEventDestroy(c->ev[i]);
	for (cudaEvent_t e : {c->ev_fork, c->ev_grad, c->ev_join})
		if (e)
			cudaEventDestroy(e);
	if (c->aux)
		cudaStreamDestroy(c->aux);
	for (cudaEvent_t e : {c->ev_wfork, c->ev_wjoin, c->ev_tfork,
	  c->ev_tdone})
		if (e)
			cudaEventDestroy(e);
	if (c->wstream)
		cudaStreamDestroy(c->wstream);
	if (c->tstream)
		cudaStreamDestroy(c->tstream);
	if (c->stream)
		cudaStreamDestroy(c->stream);
	delete c;
}

uint64_t held_bytes(const Ctx *c)
{
	const DevBuf *bufs[] = {&c->blas, &c->tris, &c->tlas, &c->irefs,
	  &c->insts, &c->nrms, &c->mtls, &c->lights, &c->sp, &c->scn,
	  &c->sortbuf, &c->q0, &c->q1, &c->hits,
	  &c->shadow, &c->scol, &c->pT, &c->pL, &c->rng, &c->acc, &c->buf,
	  &c->cnt, &c->rays, &c->brays, &c->braw, &c->bhits, &c->berr,
	  &c->mlp_act, &c->mlp_dz, &c->grid_t, &c->grid_m, &c->grid_v,
	  &c->grid_g, &c->qgrid,
	  &c->mlp_wf, &c->mlp_m, &c->mlp_v, &c->mlp_wbf, &c->mlp_wbt,
	  &c->mlp_part, &c->mlp_loss, &c->nq, &c->nrec, &c->waitchk,
	  &c->rfeat, &c->rtgt, &c->capbuf, &c->dyn_root, &c->dyn_glob,
	  &c->dyn_wbox, &c->dyn_q, &c->dyn_ranges, &c->dyn_order, &c->dyn_info,
	  &c->dyn_emit, &c->dyn_area, &c->dyn_trange, &c->dyn_idx, &c->dyn_ctr,
	  &c->dyn_bvh, &c->q0b, &c->q1b, &c->hitsb, &c->shadowb, &c->scolb, &c->cntb,
	  &c->nrecb, &c->nsnap};
	uint64_t s = 0;
	for (const DevBuf *b : bufs)
		s += b->cap;
	return s;
}

// A context over n scenes (n = 1 for the rdata API); max_depth[i] (or
// cfg->max_depth when null) bounds scene i's paths.
int new_ctx(nb_rdata *const *rds, uint32_t n, const uint32_t *max_depth,
            const rendgpu_cfg *cfg, Ctx **out)
{
	if (!rds || n == 0 || n > kMaxScenes || !cfg ||
	  cfg->size < sizeof(rendgpu_cfg) - 8 * sizeof(uint32_t))
		return RENDGPU_EINVAL;
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
		return RENDGPU_ENODEV;
	if (cfg->device < 0 || cfg->device >= ndev)
		return RENDGPU_EINVAL;
	if (cfg->mode > RENDGPU_MODE_NRC || cfg->max_depth < 1 ||
	  cfg->max_depth > 1024 || cfg->sched > 3)
		return RENDGPU_EINVAL;
	for (uint32_t i = 0; i < n; i++) {
		if (!rds[i])
			return RENDGPU_EINVAL;
		if (max_depth && (max_depth[i] < 1 || max_depth[i] > 1024))
			return RENDGPU_EINVAL;
	}
	Ctx *c = new Ctx;
	c->rd = rds[0];
	c->sc.resize(n);
	for (uint32_t i = 0; i < n; i++) {
		c->sc[i].rd = rds[i];
		c->sc[i].depth = max_depth ? max_depth[i] : cfg->max_depth;
	}
	c->cfg = *cfg;
	c->tune.block = cfg->block;
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
	  c->berr.ensure(16) != cudaSuccess ||
	  c->sp.ensure(n * sizeof(ScenePar)) != cudaSuccess ||
	  c->scn.ensure(n * 16) != cudaSuccess) {
		free_ctx(c);
		return RENDGPU_ENOMEM;
	}
	if (cudaMemset(c->berr.p, 0, 16) != cudaSuccess) {
		free_ctx(c);
		return RENDGPU_ECUDA;
	}
	*out = c;
	return 0;
}

// ------------------------------------------------------------- uploads --

// BLASes built for the traversal (blas_build.cpp: SAH binary build, optimal
// 8-wide collapse) unless cfg.reserved[4] bit 1 keeps the reference's BVH8
// from rd->bnodes, converted node for node.  Hits do not depend on the tree.
bool own_blas(const Ctx *c)
{
	return !(c->cfg.reserved[4] & 2u);
}

// BLAS of every scene (rend_prepstatic output) into the shared node and
// triangle arrays; normals and materials of all scenes back to back, with
// each scene's material ids offset by its material base.
int upload_static_all(Ctx *c)
{
	NB_CK(c, cudaSetDevice(c->device));
	std::vector<nb_qnode> nodes;
	std::vector<nb_gtri> tris;
	uint32_t nrm_base = 0, mtl_base = 0;
	c->blas_depth = 0;
	for (SceneHost &h : c->sc) {
		nb_rdata *rd = h.rd;
		if (!rd->bnodes || !rd->tris || !rd->nrms || !rd->mtls ||
		  !rd->insts)
			return fail(c, RENDGPU_EINVAL, "render data not initialised");
		if (rd->instcnt == 0 || rd->instcnt > (1u << NB_INST_ID_BITS))
			return fail(c, RENDGPU_ELIMIT, "instance count outside "
			  "1..4096 (INST_ID_BITS = 12, rend.c:24)");
		h.root_of.clear();
		h.tri_range.clear();
		h.blas_depth = 0;
		uint32_t maxtri = 0, maxmtl = 0;
		std::vector<uint32_t> uofs, ucnt; // distinct meshes in order
		for (uint32_t i = 0; i < rd->instcnt; i++) {
			const nb_rinst &ri = rd->insts[i];
			if (ri.tricnt == 0)
				return fail(c, RENDGPU_EINVAL, "instance without "
				  "triangles");
			if (ri.tricnt > (1u << (32 - NB_INST_ID_BITS)))
				return fail(c, RENDGPU_ELIMIT, "mesh above 2^20 "
				  "triangles");
			maxtri = std::max(maxtri, ri.triofs + ri.tricnt);
			if (h.root_of.count(ri.triofs))
				continue;
			h.root_of[ri.triofs] = 0;
			uofs.push_back(ri.triofs);
			ucnt.push_back(ri.tricnt);
		}
		std::vector<blas_out> built;
		std::string err;
		if (own_blas(c) && !build_blas_many(rd, uofs, ucnt, blas_params(),
		  built, &err))
			return fail(c, RENDGPU_EINVAL, err);
		for (size_t k = 0; k < uofs.size(); k++) {
			uint32_t root = 0, depth = 0;
			uint32_t first = (uint32_t)tris.size();
			if (own_blas(c)) {
				append_blas(built[k], nodes, tris, &root);
				depth = built[k].depth;
				built[k] = blas_out();
			} else {
				bvh_stats bs;
				if (!convert_blas(rd, uofs[k], nodes, tris, &root, &bs,
				  &err))
					return fail(c, RENDGPU_EINVAL, "BLAS of triofs " +
					  std::to_string(uofs[k]) + ": " + err);
				depth = bs.depth;
			}
			h.root_of[uofs[k]] = root;
			h.tri_range[uofs[k]] = {first, (uint32_t)tris.size() - first};
			h.blas_depth = std::max(h.blas_depth, depth);
		}
		for (uint32_t t = 0; t < maxtri; t++)
			maxmtl = std::max(maxmtl, rd->nrms[t].mtlid + 1u);
		find_emitters(rd, h.emitters);
		h.nrm_base = nrm_base;
		h.mtl_base = mtl_base;
		h.ntri = maxtri;
		h.nmtl = maxmtl;
		if ((uint64_t)nrm_base + maxtri > 0xffffffffull)
			return fail(c, RENDGPU_ELIMIT, "more than 2^32 triangles");
		nrm_base += maxtri;
		mtl_base += maxmtl;
		c->blas_depth = std::max(c->blas_depth, h.blas_depth);
	}
	NB_CK(c, c->blas.ensure(nodes.size() * sizeof(nb_qnode)));
	NB_CK(c, c->tris.ensure(tris.size() * sizeof(nb_gtri)));
	NB_CK(c, c->nrms.ensure((size_t)nrm_base * sizeof(nb_rnrm)));
	NB_CK(c, c->mtls.ensure((size_t)mtl_base * sizeof(nb_rmtl)));
	NB_CK(c, cudaMemcpyAsync(c->blas.p, nodes.data(), nodes.size() *
	  sizeof(nb_qnode), cudaMemcpyHostToDevice, c->stream));
	NB_CK(c, cudaMemcpyAsync(c->tris.p, tris.data(), tris.size() *
	  sizeof(nb_gtri), cudaMemcpyHostToDevice, c->stream));
	std::vector<nb_rnrm> nr;
	for (const SceneHost &h : c->sc) {
		nb_rnrm *dst = c->nrms.as<nb_rnrm>() + h.nrm_base;
		const nb_rnrm *src = h.rd->nrms;
		if (h.mtl_base) {
			nr.assign(src, src + h.ntri);
			for (nb_rnrm &n : nr)
				n.mtlid += h.mtl_base;
			src = nr.data();
		}
		NB_CK(c, cudaMemcpyAsync(dst, src, (size_t)h.ntri *
		  sizeof(nb_rnrm), cudaMemcpyHostToDevice, c->stream));
		// (a copy from pageable memory returns once the source has been
		// read, so `nr` may be refilled for the next scene)
		NB_CK(c, cudaMemcpyAsync(c->mtls.as<nb_rmtl>() + h.mtl_base,
		  h.rd->mtls, (size_t)h.nmtl * sizeof(nb_rmtl),
		  cudaMemcpyHostToDevice, c->stream));
	}
	NB_CK(c, cudaStreamSynchronize(c->stream));
	c->ntris = (uint32_t)tris.size();
	c->nnodes = (uint32_t)nodes.size();
	drop_graph(c);
	c->have_static = true;
	c->have_dynamic = false;
	return 0;
}

// Inputs of device-side scene updates that an upload fixes (single-scene
// contexts): each instance's BLAS root box as the host bridge forms it (the
// union of the root's child boxes, main.c:133-140), the emitting triangles
// in light-table order, and scratch of the TLAS build.
int dyn_prepare(Ctx *c, uint64_t *bytes)
{
	SceneHost &h = c->sc[0];
	const nb_rdata *rd = h.rd;
	uint32_t n = rd->instcnt;
	std::vector<float4> rb(2 * (size_t)n);
	for (uint32_t i = 0; i < n; i++) {
		const nb_bnode8 *b = &rd->bnodes[(size_t)rd->insts[i].triofs << 1];
		float mi[3] = {b->minx8[0], b->miny8[0], b->minz8[0]};
		float ma[3] = {b->maxx8[0], b->maxy8[0], b->maxz8[0]};
		for (int k = 1; k < 8; k++) {
			mi[0] = b->minx8[k] < mi[0] ? b->minx8[k] : mi[0];
			mi[1] = b->miny8[k] < mi[1] ? b->miny8[k] : mi[1];
			mi[2] = b->minz8[k] < mi[2] ? b->minz8[k] : mi[2];
			ma[0] = b->maxx8[k] > ma[0] ? b->maxx8[k] : ma[0];
			ma[1] = b->maxy8[k] > ma[1] ? b->maxy8[k] : ma[1];
			ma[2] = b->maxz8[k] > ma[2] ? b->maxz8[k] : ma[2];
		}
		rb[2 * i] = make_float4(mi[0], mi[1], mi[2], 0.0f);
		rb[2 * i + 1] = make_float4(ma[0], ma[1], ma[2], 0.0f);
	}
	// each instance's triangles in the device array (tight boxes)
	std::vector<uint2> tr(std::max(n, 1u), make_uint2(0u, 0u));
	for (uint32_t i = 0; i < n; i++) {
		auto it = h.tri_range.find(rd->insts[i].triofs);
		if (it != h.tri_range.end())
			tr[i] = make_uint2(it->second.first, it->second.second);
	}
	std::vector<EmitSrc> es;
	for (uint32_t i = 0; i < n; i++) {
		const nb_rinst &ri = rd->insts[i];
		auto it = h.emitters.find(ri.triofs);
		if (it == h.emitters.end())
			continue;
		for (uint32_t t : it->second) {
			const nb_rnrm *rn = &rd->nrms[ri.triofs + t];
			const nb_rmtl *m = &rd->mtls[rn->mtlid];
			if (!(m->flags & NB_FLAG_EMISSIVE))
				continue;
			const nb_rtri *tr = &rd->tris[ri.triofs + t];
			EmitSrc e;
			std::memset(&e, 0, sizeof(e));
			e.inst = i;
			const nb_vec3 *vv[3] = {&tr->v0, &tr->v1, &tr->v2};
			const nb_vec3 *nn[3] = {&rn->n0, &rn->n1, &rn->n2};
			for (int k = 0; k < 3; k++) {
				e.v[k][0] = vv[k]->x;
				e.v[k][1] = vv[k]->y;
				e.v[k][2] = vv[k]->z;
				e.n[k][0] = nn[k]->x;
				e.n[k][1] = nn[k]->y;
				e.n[k][2] = nn[k]->z;
			}
			e.emit[0] = m->col.x;
			e.emit[1] = m->col.y;
			e.emit[2] = m->col.z;
			es.push_back(e);
		}
	}
	// a degenerate emitter the host table skipped: device updates (which
	// keep every entry) are then refused
	c->dyn_nemit = es.size() == h.lights.size() ? (uint32_t)es.size() :
	  0xffffffffu;
	size_t nn = std::max(n, 1u);
	NB_CK(c, c->dyn_root.ensure(nn * 32));
	NB_CK(c, c->dyn_glob.ensure(nn * 64));
	NB_CK(c, c->dyn_wbox.ensure(nn * 32));
	NB_CK(c, c->dyn_q.ensure(2 * nn * sizeof(TbNode)));
	NB_CK(c, c->dyn_ranges.ensure(nn * 8 * sizeof(uint2)));
	NB_CK(c, c->dyn_order.ensure(nn * sizeof(uint32_t)));
	NB_CK(c, c->dyn_info.ensure(4 * sizeof(uint32_t)));
	NB_CK(c, c->dyn_emit.ensure(std::max<size_t>(es.size(), 1) *
	  sizeof(EmitSrc)));
	NB_CK(c, c->dyn_area.ensure(16));
	NB_CK(c, c->dyn_trange.ensure(tr.size() * sizeof(uint2)));
	NB_CK(c, cudaMemcpyAsync(c->dyn_trange.p, tr.data(), tr.size() *
	  sizeof(uint2), cudaMemcpyHostToDevice, c->stream));
	NB_CK(c, cudaMemcpyAsync(c->dyn_root.p, rb.data(), rb.size() *
	  sizeof(float4), cudaMemcpyHostToDevice, c->stream));
	if (!es.empty())
		NB_CK(c, cudaMemcpyAsync(c->dyn_emit.p, es.data(), es.size() *
		  sizeof(EmitSrc), cudaMemcpyHostToDevice, c->stream));
	NB_CK(c, cudaMemsetAsync(c->dyn_info.p, 0, 4 * sizeof(uint32_t),
	  c->stream));
	// (pageable sources: the copies have read them when they return)
	*bytes = rb.size() * sizeof(float4) + es.size() * sizeof(EmitSrc) +
	  tr.size() * sizeof(uint2);
	c->dyn_built = false;
	c->dyn_active = false;
	return 0;
}

uint32_t device_tlas_limit(const Ctx *c);

// Device TLAS build over the world boxes in dyn_wbox (n instances of the
// single scene), one launch per level up to the depth limit (levels past
// the tree's depth find no open node and return at once); returns the
// depth limit used.
int tlas_build(Ctx *c, uint32_t n, uint32_t *limit, bool collapse)
{
	uint32_t nn = std::max(n, 1u);
	NB_CK(c, c->dyn_idx.ensure((size_t)2 * nn * sizeof(uint16_t)));
	NB_CK(c, c->dyn_ctr.ensure(4 * sizeof(uint32_t)));
	TbArgs A;
	A.wbox = c->dyn_wbox.as<float4>();
	A.n = n;
	A.inst_base = 0u;
	A.nodes = c->tlas.as<nb_qnode>();
	A.node_cap = nn;
	A.irefs = c->irefs.as<uint32_t>();
	A.qa = c->dyn_q.as<TbNode>();
	A.qb = c->dyn_q.as<TbNode>() + nn;
	A.ranges = c->dyn_ranges.as<uint2>();
	A.order = c->dyn_order.as<uint32_t>();
	A.info = c->dyn_info.as<uint32_t>();
	A.idx = c->dyn_idx.as<uint16_t>();
	A.tmp = c->dyn_idx.as<uint16_t>() + nn;
	A.ctr = c->dyn_ctr.as<uint32_t>();
	// the uploaded trees sized the traversal stack; the device tree stays
	// within what it holds
	A.depth_limit = device_tlas_limit(c);
	if (collapse) {
		// one CTA: binary SAH tree, collapse by cost, 8-wide encoding
		size_t m = 2 * (size_t)nn, o_cost = m * sizeof(TcNode);
		size_t o_kd = o_cost + m * 8 * sizeof(float), o_prev = o_kd + m * 8;
		size_t o_q = (o_prev + m + 15) & ~(size_t)15;
		NB_CK(c, c->dyn_bvh.ensure(o_q + 6 * (size_t)nn * sizeof(uint32_t)));
		unsigned char *base = c->dyn_bvh.as<unsigned char>();
		TcArgs T;
		T.A = A;
		T.bn = reinterpret_cast<TcNode *>(base);
		T.cost = reinterpret_cast<float *>(base + o_cost);
		T.kd = base + o_kd;
		T.prev = base + o_prev;
		T.qa = reinterpret_cast<uint32_t *>(base + o_q);
		T.qb = T.qa + 3 * (size_t)nn;
		size_t dyn = tc_dyn_smem(nn);
		NB_CK(c, cudaFuncSetAttribute(k_tlas_cta,
		  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
		k_tlas_cta<<<1, kCbThreads, dyn, c->stream>>>(T);
		NB_CK(c, cudaGetLastError());
		*limit = A.depth_limit;
		return 0;
	}
	k_tlas_init<<<1, 512, 0, c->stream>>>(A);
	NB_CK(c, cudaGetLastError());
	uint64_t open = 1; // at most this many open nodes on a level
	for (uint32_t level = 0; level < A.depth_limit; level++) {
		// the level writes its children into the other queue
		NB_CK(c, cudaMemsetAsync(A.ctr + 2u + ((level & 1u) ^ 1u), 0,
		  sizeof(uint32_t), c->stream));
		uint64_t nodes = std::min<uint64_t>(open, nn);
		uint32_t grid = (uint32_t)std::min<uint64_t>((nodes +
		  kTbLevelWarps - 1) / kTbLevelWarps, (uint64_t)c->nsm * 8u);
		k_tlas_level<<<grid, kTbLevelWarps * 32, 0, c->stream>>>(A, level);
		NB_CK(c, cudaGetLastError());
		open *= 8u;
	}
	k_tlas_finish<<<grid_for(c, nn, 256), 256, 0, c->stream>>>(A);
	NB_CK(c, cudaGetLastError());
	*limit = A.depth_limit;
	return 0;
}

// New object->world matrices (device, 16 floats each, rd->insts order) ->
// instance records, world boxes, TLAS (built, or refitted when asked and a
// device build exists) and light table, all on the context's stream.
int update_instances(Ctx *c, const float *glob, uint32_t n, uint32_t flags)
{
	int rc = ready(c, false);
	if (rc)
		return rc;
	if (c->batch)
		return fail(c, RENDGPU_EINVAL, "device-side scene updates serve "
		  "single-scene contexts");
	SceneHost &h = c->sc[0];
	if (n != h.rd->instcnt)
		return fail(c, RENDGPU_EINVAL, "update: n must equal rd->instcnt");
	if (!glob || (reinterpret_cast<uintptr_t>(glob) & 3u))
		return fail(c, RENDGPU_EINVAL, "update: null or misaligned matrices");
	if (c->dyn_nemit == 0xffffffffu)
		return fail(c, RENDGPU_ESTATE, "update: the uploaded light table "
		  "skipped a degenerate emitter; upload non-degenerate transforms "
		  "first");
	if (flags & ~(uint32_t)(RENDGPU_UPDATE_REFIT | RENDGPU_UPDATE_TIGHT |
	  RENDGPU_UPDATE_COLLAPSE | RENDGPU_UPDATE_LEVELS))
		return fail(c, RENDGPU_EINVAL, "update: unknown flags");
	if ((flags & RENDGPU_UPDATE_COLLAPSE) && (flags & RENDGPU_UPDATE_LEVELS))
		return fail(c, RENDGPU_EINVAL, "update: COLLAPSE and LEVELS "
		  "exclude each other");
	NB_CK(c, cudaSetDevice(c->device));
	bool refit = (flags & RENDGPU_UPDATE_REFIT) && c->dyn_built;
	uint32_t nn = std::max(n, 1u);
	k_inst_update<<<(n + 127u) / 128u, 128, 0, c->stream>>>(glob, n,
	  c->dyn_root.as<float4>(), c->insts.as<float4>(),
	  c->dyn_wbox.as<float4>(), c->berr.as<uint32_t>() + 1);
	NB_CK(c, cudaGetLastError());
	if ((flags & RENDGPU_UPDATE_TIGHT) && n) {
		k_inst_tight<<<n, 256, 0, c->stream>>>(glob, n,
		  c->dyn_trange.as<uint2>(), c->tris.as<float4>(),
		  c->dyn_wbox.as<float4>());
		NB_CK(c, cudaGetLastError());
	}
	if (!refit) {
		uint32_t limit = 0;
		bool collapse = (flags & RENDGPU_UPDATE_COLLAPSE) ||
		  (!(flags & RENDGPU_UPDATE_LEVELS) && n <= kCollapseMaxInst);
		rc = tlas_build(c, n, &limit, collapse);
		if (rc)
			return rc;
		h.tlas_depth = c->tlas_depth = limit;
	} else {
		k_tlas_refit<<<grid_for(c, nn * 32u, 256), 256, 0, c->stream>>>(
		  c->dyn_wbox.as<float4>(), c->dyn_order.as<uint32_t>(),
		  c->dyn_ranges.as<uint2>(), c->dyn_info.as<uint32_t>(),
		  c->tlas.as<nb_qnode>());
	}
	NB_CK(c, cudaGetLastError());
	if (c->dyn_nemit) {
		k_light_update<<<1, 32, 0, c->stream>>>(c->dyn_emit.as<EmitSrc>(),
		  c->dyn_nemit, c->insts.as<float4>(),
		  c->lights.as<float4>() + 5u * h.light_off, c->dyn_area.as<float>());
		NB_CK(c, cudaGetLastError());
	}
	h.tlas_root = 0u;
	c->dyn_built = true;
	c->dyn_active = true;
	c->st.h2d_bytes = 0;
	return 0;
}

// The uploaded TLAS rebuilt on the device over tight instance boxes (the
// bounds of every transformed vertex) instead of the reference's
// corner-transformed root boxes: fewer rays enter instances they never
// touch (config-2 frame 31.3 ms instead of 33.0 ms, measured back to back).
// Single-scene contexts, unless cfg.reserved[4] bit 0 keeps the converted
// reference TLAS.  Instances and lights stay as uploaded; hits do not depend
// on the tree, and its depth stays within the uploaded tree's.
bool rebuilds_tlas(const Ctx *c)
{
	return !c->batch && c->sc.size() == 1 && !(c->cfg.reserved[4] & 1u);
}

// Depth a device-built TLAS may reach: the levels the traversal stack chosen
// for the uploaded trees leaves beside the deepest BLAS (at least the
// converted TLAS's depth).  SAH splits then rarely meet the cap, and the
// context's TLAS depth becomes that bound, so the stack stays the same.
uint32_t device_tlas_limit(const Ctx *c)
{
	uint32_t need = need_stack(c), st = 0;
	for (int s : kStacks)
		if (!st && need <= (uint32_t)s)
			st = (uint32_t)s;
	uint32_t room = st ? st - c->blas_depth - 2u : 0u;
	return std::max(room, c->tlas_depth);
}

int rebuild_tlas_tight(Ctx *c)
{
	SceneHost &h = c->sc[0];
	uint32_t n = h.rd->instcnt, nn = std::max(n, 1u);
	k_inst_glob<<<(n + 127u) / 128u, 128, 0, c->stream>>>(
	  c->insts.as<float4>(), n, c->dyn_glob.as<float>());
	NB_CK(c, cudaGetLastError());
	k_inst_tight<<<n, 256, 0, c->stream>>>(c->dyn_glob.as<float>(), n,
	  c->dyn_trange.as<uint2>(), c->tris.as<float4>(),
	  c->dyn_wbox.as<float4>());
	NB_CK(c, cudaGetLastError());
	uint32_t limit = 0;
	int rc = tlas_build(c, n, &limit, !(c->cfg.reserved[4] & 8u));
	if (rc)
		return rc;
	NB_CK(c, cudaStreamSynchronize(c->stream));
	h.tlas_root = 0u;
	h.tlas_depth = c->tlas_depth = limit;
	c->dyn_built = true;
	return 0;
}

// TLAS, instances and lights of every scene (rend_prepdynamic output).
// Instance references are global, so hit ids carry the instance's index
// among all scenes' instances (at most 4096 in total).
int upload_dynamic_all(Ctx *c)
{
	if (!c->have_static)
		return fail(c, RENDGPU_ESTATE, "upload_static must come first");
	NB_CK(c, cudaSetDevice(c->device));
	// a failed upload leaves no half-updated scene behind: the context
	// needs a successful one before it traces again
	c->have_dynamic = false;
	c->dyn_active = false;
	drop_graph(c);
	std::vector<nb_qnode> nodes;
	std::vector<uint32_t> irefs;
	std::vector<nb_ginst> gi;
	std::vector<nb_glight> lights;
	c->tlas_depth = 0;
	for (SceneHost &h : c->sc) {
		nb_rdata *rd = h.rd;
		h.inst_base = (uint32_t)gi.size();
		if (gi.size() + rd->instcnt > (1u << NB_INST_ID_BITS))
			return fail(c, RENDGPU_ELIMIT, "more than 4096 instances "
			  "in the context (hit ids keep 12 instance bits, "
			  "rend.c:24)");
		bvh_stats bs;
		std::string err;
		if (!convert_tlas(rd, nodes, irefs, h.inst_base, &h.tlas_root, &bs,
		  &err))
			return fail(c, RENDGPU_EINVAL, "TLAS: " + err);
		h.tlas_depth = bs.depth;
		c->tlas_depth = std::max(c->tlas_depth, bs.depth);
		for (uint32_t i = 0; i < rd->instcnt; i++) {
			const nb_rinst &ri = rd->insts[i];
			auto it = h.root_of.find(ri.triofs);
			if (it == h.root_of.end())
				return fail(c, RENDGPU_ESTATE, "instance mesh not "
				  "uploaded by upload_static");
			nb_ginst g;
			std::memcpy(g.m, ri.globinv, sizeof(g.m));
			g.root = it->second;
			g.triofs = h.nrm_base + ri.triofs;
			g.flags = ri.flags;
			g.pad = 0;
			gi.push_back(g);
		}
		h.light_area = build_lights(rd, h.lights, &h.emitters);
		h.light_off = (uint32_t)lights.size();
		lights.insert(lights.end(), h.lights.begin(), h.lights.end());
	}
	for (SceneHost &h : c->sc) {
		// radiance-cache encoding box of each scene: its instance bounds
		const nb_rdata *rd = h.rd;
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
			h.nbox.lo[a] = lo[a];
			h.nbox.inv[a] = hi[a] > lo[a] ? 1.0f / (hi[a] - lo[a]) : 1.0f;
		}
	}
	c->box = c->sc[0].nbox; // the box of the query / encode calls
	c->ninst = (uint32_t)gi.size();
	// device-side updates (single-scene contexts) rebuild the TLAS in place:
	// room for max(instances, 1) nodes
	size_t tlas_nodes = nodes.size();
	if (!c->batch)
		tlas_nodes = std::max(tlas_nodes, (size_t)std::max(c->ninst, 1u));
	NB_CK(c, c->tlas.ensure(tlas_nodes * sizeof(nb_qnode)));
	NB_CK(c, c->irefs.ensure(irefs.size() * sizeof(uint32_t)));
	NB_CK(c, c->insts.ensure(gi.size() * sizeof(nb_ginst)));
	NB_CK(c, c->lights.ensure(lights.size() * sizeof(nb_glight)));
	NB_CK(c, c->sp.ensure(c->sc.size() * sizeof(ScenePar)));
	NB_CK(c, cudaMemcpyAsync(c->tlas.p, nodes.data(), nodes.size() *
	  sizeof(nb_qnode), cudaMemcpyHostToDevice, c->stream));
	NB_CK(c, cudaMemcpyAsync(c->irefs.p, irefs.data(), irefs.size() *
	  sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
	NB_CK(c, cudaMemcpyAsync(c->insts.p, gi.data(), gi.size() *
	  sizeof(nb_ginst), cudaMemcpyHostToDevice, c->stream));
	if (!lights.empty())
		NB_CK(c, cudaMemcpyAsync(c->lights.p, lights.data(),
		  lights.size() * sizeof(nb_glight), cudaMemcpyHostToDevice,
		  c->stream));
	uint64_t dyn_bytes = 0;
	if (!c->batch) {
		int rc = dyn_prepare(c, &dyn_bytes);
		if (rc)
			return rc;
	}
	NB_CK(c, cudaStreamSynchronize(c->stream));
	c->st.h2d_bytes = nodes.size() * sizeof(nb_qnode) + irefs.size() *
	  sizeof(uint32_t) + gi.size() * sizeof(nb_ginst) +
	  lights.size() * sizeof(nb_glight) + dyn_bytes;
	drop_graph(c);
	c->have_dynamic = true;
	if (!stack_of(c))
		return too_deep(c);
	return 0;
}

// Two concurrent waves of half the camera slots each (tune.queue 0): a
// single-scene context with enough slots that each half still fills the
// GPU.  Radiance-cache queries and training records of both waves go to the
// same arrays through the first wave's counters.  Each wave's persistent
// launches end with their slowest rays; with the other wave's launches
// queued on a second stream, its blocks take the SMs those tails leave idle.
// Paths, their PCG32 streams and the accumulation do not depend on the
// waves, so images are the same as with one wave.
constexpr uint64_t kTwoWaveMinSlots = 1u << 20;

bool two_waves_fit(const Ctx *c, uint64_t nslots)
{
	return !c->batch && c->sc.size() == 1 && nslots >= kTwoWaveMinSlots &&
	  !(c->cfg.reserved[4] & 4u);
}

// Frame buffers for every scene's width, height and spp: per-path state
// for all paths, ray queues for one wave of tune.queue camera slots (0:
// two concurrent waves of half the slots where two_waves_fit, else one
// wave of all slots); accumulation cleared.
int alloc_frame(Ctx *c)
{
	NB_CK(c, cudaSetDevice(c->device));
	uint64_t np = 0, npix = 0, nslots = 0;
	for (SceneHost &h : c->sc) {
		const nb_rdata *rd = h.rd;
		uint32_t spp = rd->spp ? rd->spp : 1u;
		uint64_t p = (uint64_t)rd->width * rd->height * spp;
		if (p == 0)
			return fail(c, RENDGPU_ELIMIT, "empty image");
		h.W = rd->width;
		h.H = rd->height;
		h.spp = spp;
		h.path_base = (uint32_t)np;
		h.pix_base = (uint32_t)npix;
		h.slot_base = (uint32_t)nslots;
		h.nslots = ((h.W + 7u) >> 3) * ((h.H + 3u) >> 2) * 32u * spp;
		np += p;
		npix += (uint64_t)rd->width * rd->height;
		nslots += h.nslots;
		if (nslots > 0x7fffffffull)
			return fail(c, RENDGPU_ELIMIT, "width*height*spp over all "
			  "scenes outside 1..2^31-1");
	}
	c->two_waves = !c->tune.queue && two_waves_fit(c, nslots);
	uint64_t q = c->tune.queue ? std::min<uint64_t>(c->tune.queue, nslots) :
	  (c->two_waves ? (nslots + 1) / 2 : nslots);
	q = std::max<uint64_t>(q, 1);
	NB_CK(c, c->q0.ensure(q * 32));
	NB_CK(c, c->q1.ensure(q * 32));
	NB_CK(c, c->hits.ensure(q * 16));
	NB_CK(c, c->shadow.ensure(q * 32));
	NB_CK(c, c->scol.ensure(q * 16));
	if (c->two_waves) {
		NB_CK(c, c->q0b.ensure(q * 32));
		NB_CK(c, c->q1b.ensure(q * 32));
		NB_CK(c, c->hitsb.ensure(q * 16));
		NB_CK(c, c->shadowb.ensure(q * 32));
		NB_CK(c, c->scolb.ensure(q * 16));
		NB_CK(c, c->cntb.ensure(64 * sizeof(uint32_t)));
		if (!c->wstream) {
			NB_CK(c, cudaStreamCreateWithFlags(&c->wstream,
			  cudaStreamNonBlocking));
			for (cudaEvent_t *e : {&c->ev_wfork, &c->ev_wjoin})
				NB_CK(c, cudaEventCreateWithFlags(e,
				  cudaEventDisableTiming));
		}
	}
	NB_CK(c, c->pT.ensure(np * 16));
	NB_CK(c, c->pL.ensure(np * 16));
	NB_CK(c, c->rng.ensure(np * 8));
	NB_CK(c, c->acc.ensure(npix * 12));
	NB_CK(c, c->buf.ensure(npix * 4));
	NB_CK(c, c->scn.ensure(c->sc.size() * 16));
	NB_CK(c, c->sp.ensure(c->sc.size() * sizeof(ScenePar)));
	NB_CK(c, c->sortbuf.ensure(2 * kSortKeys * sizeof(uint32_t)));
	NB_CK(c, cudaMemsetAsync(c->sortbuf.p, 0, 2 * kSortKeys *
	  sizeof(uint32_t), c->stream));
	c->npaths = (uint32_t)np;
	c->npix = (uint32_t)npix;
	c->nslots = (uint32_t)nslots;
	c->qcap = (uint32_t)q;
	c->have_frame = true;
	drop_graph(c);
	NB_CK(c, cudaMemsetAsync(c->acc.p, 0, npix * 12, c->stream));
	NB_CK(c, cudaMemsetAsync(c->buf.p, 0, npix * 4, c->stream));
	NB_CK(c, cudaStreamSynchronize(c->stream));
	return 0;
}

// Copy accumulation (which & 1) and/or ARGB8 (which & 2) of every scene
// into its rd->acc / rd->buf.
int readback_all(Ctx *c, int which)
{
	if (!c->have_frame)
		return fail(c, RENDGPU_ESTATE, "rendgpu_resaccum must come first");
	NB_CK(c, cudaSetDevice(c->device));
	c->st.d2h_bytes = 0;
	for (const SceneHost &h : c->sc) {
		size_t npix = (size_t)h.W * h.H;
		if ((which & 1) && h.rd->acc) {
			NB_CK(c, cudaMemcpyAsync(h.rd->acc, c->acc.as<float>() +
			  3 * (size_t)h.pix_base, npix * 12, cudaMemcpyDeviceToHost,
			  c->stream));
			c->st.d2h_bytes += npix * 12;
		}
		if ((which & 2) && h.rd->buf) {
			NB_CK(c, cudaMemcpyAsync(h.rd->buf, c->buf.as<uint32_t>() +
			  h.pix_base, npix * 4, cudaMemcpyDeviceToHost, c->stream));
			c->st.d2h_bytes += npix * 4;
		}
	}
	NB_CK(c, cudaStreamSynchronize(c->stream));
	return 0;
}

// ------------------------------------------------------------- tuning --

bool tune_valid(const rendgpu_tune *t)
{
	return t && (t->block == 0 || t->block == 64 || t->block == 128 ||
	  t->block == 256) && (t->stack == 0 || t->stack == 24 ||
	  t->stack == 32 || t->stack == 48 ||
	  (t->force && t->stack == (uint32_t)kStackForced)) && t->sched <= 3 &&
	  t->sort <= 1 && t->fuse <= 2 && t->force <= 1;
}

// Apply launch parameters; a new queue capacity re-sizes the queues (and
// so clears the accumulator).
int set_tune(Ctx *c, const rendgpu_tune *t)
{
	if (!tune_valid(t))
		return fail(c, RENDGPU_EINVAL, "tune: block 0/64/128/256, stack "
		  "0/24/32/48 (8 with force), sched 0..3, force 0/1");
	bool requeue = t->queue != c->tune.queue;
	c->tune.block = t->block;
	c->tune.stack = t->stack;
	c->tune.queue = t->queue;
	c->tune.sched = t->sched;
	c->tune.sort = t->sort;
	c->tune.fuse = t->fuse;
	c->tune.force = t->force;
	drop_graph(c);
	if (requeue && c->have_frame)
		return alloc_frame(c);
	return 0;
}

// The settings in effect (defaults resolved).
rendgpu_tune effective_tune(const Ctx *c)
{
	rendgpu_tune t{};
	t.block = (uint32_t)block_of(c);
	t.stack = c->have_dynamic ? (uint32_t)stack_of(c) : c->tune.stack;
	t.queue = c->tune.queue;
	int sc = sched_of(c);
	t.sched = sc == kSchedStep ? 1u : sc == kSchedPhase ? 2u : 3u;
	t.sort = sorts(c) ? 1u : 0u;
	t.fuse = c->tune.fuse == 2u ? 2u : 1u;
	t.force = c->tune.force;
	return t;
}

// Median device time of `frames` frames with setting t (after one untimed
// frame that also captures the graph).
int tune_measure(Ctx *c, const rendgpu_tune &t, uint32_t frames, float *ms)
{
	int rc = set_tune(c, &t);
	if (rc)
		return rc;
	rc = render_frame(c);
	if (rc)
		return rc;
	std::vector<float> v;
	for (uint32_t f = 0; f < frames; f++) {
		rc = render_frame(c);
		if (rc)
			return rc;
		v.push_back(c->st.ms_frame);
	}
	std::sort(v.begin(), v.end());
	*ms = v[v.size() / 2];
	return 0;
}

// Coordinate-descent autotuner over the traversal schedule, the trace
// block size, the stack depth, the queue capacity and (single-scene path
// frames) ray reordering: each knob in turn
// takes the value with the lowest measured frame time, the others held at
// the best so far.  Frames re-render the current sample index (rd->samples
// is not advanced); the accumulator is cleared afterwards.
int autotune(Ctx *c, uint32_t frames, rendgpu_tune *best_out,
             rendgpu_tune *log, uint32_t cap, uint32_t *nlog)
{
	int rc = ready(c, true);
	if (rc)
		return rc;
	if (c->cfg.mode == RENDGPU_MODE_NRC)
		return fail(c, RENDGPU_EINVAL, "autotune: frames of the radiance "
		  "cache train it; tune in PATH mode");
	frames = std::max(frames, 1u);
	uint32_t flags = c->cfg.flags;
	c->cfg.flags = (flags | RENDGPU_FLAG_TIMING) & ~RENDGPU_FLAG_COUNT;
	uint32_t nl = 0;
	auto run = [&](rendgpu_tune t, float *ms) {
		int r = tune_measure(c, t, frames, ms);
		if (!r && log && nl < cap) {
			log[nl] = t;
			log[nl].ms = *ms;
		}
		if (!r)
			nl++;
		return r;
	};
	rendgpu_tune best = effective_tune(c);
	best.ms = 0.0f;
	float best_ms = 0.0f;
	rc = run(best, &best_ms);
	std::vector<uint32_t> queues;
	for (uint32_t d : {2u, 4u, 8u}) {
		uint32_t q = ((c->nslots / d + 1023u) / 1024u) * 1024u;
		if (q >= 65536u && q < c->nslots)
			queues.push_back(q);
	}
	for (int knob = 0; knob < 5 && !rc; knob++) {
		std::vector<uint32_t> vals;
		if (knob == 0)
			vals = {3u, 1u};
		else if (knob == 1)
			vals = {64u, 128u, 256u};
		else if (knob == 2) {
			for (int st : kStacks)
				if (need_stack(c) <= (uint32_t)st)
					vals.push_back((uint32_t)st);
		} else if (knob == 3) {
			vals = queues;
			vals.push_back(0u);
		} else if (c->sc.size() == 1 && c->cfg.mode != RENDGPU_MODE_NRC) {
			vals = {0u, 1u};
		}
		rendgpu_tune base = best;
		for (uint32_t v : vals) {
			rendgpu_tune t = base;
			uint32_t *field = knob == 0 ? &t.sched : knob == 1 ? &t.block :
			  knob == 2 ? &t.stack : knob == 3 ? &t.queue : &t.sort;
			if (*field == v)
				continue;
			*field = v;
			float ms = 0.0f;
			rc = run(t, &ms);
			if (rc)
				break;
			if (ms < best_ms) {
				best_ms = ms;
				best = t;
			}
		}
	}
	c->cfg.flags = flags;
	if (nlog)
		*nlog = nl;
	if (rc)
		return rc;
	best.ms = best_ms;
	rc = set_tune(c, &best);
	if (rc)
		return rc;
	c->tune.ms = best_ms;
	NB_CK(c, cudaMemsetAsync(c->acc.p, 0, (size_t)c->npix * 12, c->stream));
	NB_CK(c, cudaMemsetAsync(c->buf.p, 0, (size_t)c->npix * 4, c->stream));
	NB_CK(c, cudaStreamSynchronize(c->stream));
	if (best_out)
		*best_out = best;
	return 0;
}

// ------------------------------------------------------ tune store --
//
// Tuned launch parameters persist in a text file, one line per GPU model and
// scene signature:  "<gpu>|<signature> block stack queue sched sort fuse ms".
// The GPU key is the device name, SM count and compute capability; the
// signature hashes (FNV-1a, 64 bit) what the tuned choice depends on: the
// mode and every scene's triangle and instance counts, BVH depths, image size,
// spp and path depth.

std::string tune_gpu_key(const Ctx *c)
{
	cudaDeviceProp p;
	if (cudaGetDeviceProperties(&p, c->device) != cudaSuccess)
		return "unknown";
	std::string name(p.name);
	for (char &ch : name)
		if (ch == ' ' || ch == '|')
			ch = '_';
	return name + ":" + std::to_string(p.multiProcessorCount) + ":" +
	  std::to_string(p.major) + "." + std::to_string(p.minor);
}

std::string tune_signature(const Ctx *c)
{
	uint64_t h = 1469598103934665603ull;
	auto mix = [&h](uint64_t v) {
		for (int i = 0; i < 8; i++) {
			h ^= (v >> (8 * i)) & 0xffu;
			h *= 1099511628211ull;
		}
	};
	mix(c->cfg.mode);
	mix(own_blas(c) ? 1u : 0u);
	mix(c->sc.size());
	for (const SceneHost &s : c->sc) {
		mix(s.ntri);
		mix(s.rd->instcnt);
		mix(s.blas_depth);
		mix(s.tlas_depth);
		mix(s.W);
		mix(s.H);
		mix(s.spp);
		mix(s.depth);
	}
	char buf[24];
	std::snprintf(buf, sizeof(buf), "%016llx", (unsigned long long)h);
	return buf;
}

int tune_save(Ctx *c, const char *path)
{
	int rc = ready(c, true);
	if (rc)
		return rc;
	if (!path)
		return fail(c, RENDGPU_EINVAL, "tune_save: null path");
	std::string key = tune_gpu_key(c) + "|" + tune_signature(c);
	std::vector<std::string> keep;
	if (FILE *f = std::fopen(path, "r")) {
		char line[512];
		while (std::fgets(line, sizeof(line), f)) {
			std::string l(line);
			if (l.compare(0, key.size() + 1, key + " ") != 0)
				keep.push_back(l);
		}
		std::fclose(f);
	}
	rendgpu_tune t = effective_tune(c);
	char row[512];
	std::snprintf(row, sizeof(row), "%s %u %u %u %u %u %u %.6g\n",
	  key.c_str(), t.block, t.stack, t.queue, t.sched, t.sort, t.fuse,
	  (double)c->tune.ms);
	keep.push_back(row);
	std::string tmp = std::string(path) + ".tmp";
	FILE *f = std::fopen(tmp.c_str(), "w");
	if (!f)
		return fail(c, RENDGPU_EINVAL, "tune_save: cannot write " + tmp);
	bool ok = true;
	for (const std::string &l : keep)
		ok = ok && std::fputs(l.c_str(), f) >= 0;
	ok = (std::fclose(f) == 0) && ok;
	if (!ok || std::rename(tmp.c_str(), path) != 0)
		return fail(c, RENDGPU_EINVAL, "tune_save: cannot write " +
		  std::string(path));
	return 0;
}

// 1 when a stored setting for this GPU and scene signature was applied,
// 0 when the file has none (or does not exist).
int tune_load(Ctx *c, const char *path)
{
	int rc = ready(c, true);
	if (rc)
		return rc;
	if (!path)
		return fail(c, RENDGPU_EINVAL, "tune_load: null path");
	std::string key = tune_gpu_key(c) + "|" + tune_signature(c);
	FILE *f = std::fopen(path, "r");
	if (!f)
		return 0;
	char line[512];
	rendgpu_tune t{};
	bool found = false;
	while (!found && std::fgets(line, sizeof(line), f)) {
		std::string l(line);
		if (l.compare(0, key.size() + 1, key + " ") != 0)
			continue;
		double ms = 0.0;
		found = std::sscanf(line + key.size() + 1, "%u %u %u %u %u %u %lf",
		  &t.block, &t.stack, &t.queue, &t.sched, &t.sort, &t.fuse,
		  &ms) == 7;
		t.ms = (float)ms;
	}
	std::fclose(f);
	if (!found)
		return 0;
	rc = set_tune(c, &t);
	if (rc)
		return rc;
	c->tune.ms = t.ms;
	return 1;
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
unsigned long long g_noalloc_ctx[64]; // context id the address belongs to

// Id of the current CUDA context (cuCtxGetCurrent + cuCtxGetId, reached
// through the runtime's driver entry points so the library needs no link
// against libcuda).  A device reset ends the context; the next one has a new
// id and loads the module, and with it the array, again, possibly at another
// address.  0 when the id is not available.
unsigned long long current_ctx_id()
{
	typedef int (*GetCurrent)(void **);
	typedef int (*GetId)(void *, unsigned long long *);
	static GetCurrent get_current = nullptr;
	static GetId get_id = nullptr;
	static bool tried = false;
	if (!tried) {
		tried = true;
		cudaDriverEntryPointQueryResult q;
		if (cudaGetDriverEntryPoint("cuCtxGetCurrent",
		  reinterpret_cast<void **>(&get_current), cudaEnableDefault, &q) !=
		  cudaSuccess || q != cudaDriverEntryPointSuccess)
			get_current = nullptr;
		if (cudaGetDriverEntryPoint("cuCtxGetId",
		  reinterpret_cast<void **>(&get_id), cudaEnableDefault, &q) !=
		  cudaSuccess || q != cudaDriverEntryPointSuccess)
			get_id = nullptr;
	}
	void *ctx = nullptr;
	unsigned long long id = 0;
	if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx ||
	    get_id(ctx, &id) != 0)
		return 0;
	return id;
}

// Device address of the scratch array on the current device `dev`: looked
// up on the first use in each CUDA context of the device (a device reset
// makes a new context), cached otherwise.
int noalloc_scratch(Ctx *c, int dev, unsigned char **base)
{
	if (dev < 0 || dev >= 64)
		return fail(c, RENDGPU_EINVAL, "device ordinal above 63");
	std::lock_guard<std::mutex> lk(g_noalloc_mu);
	unsigned long long id = current_ctx_id();
	if (!g_noalloc_addr[dev] || id != g_noalloc_ctx[dev]) {
		void *p = nullptr;
		cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		if (e != cudaSuccess || !p)
			return cuda_fail(c, e, "cudaGetSymbolAddress(scratch)");
		g_noalloc_addr[dev] = p;
		g_noalloc_ctx[dev] = id;
	}
	*base = static_cast<unsigned char *>(g_noalloc_addr[dev]);
	return 0;
}

// Count and work counter of one ray-batch call (hdr[0], hdr[2]), written on
// the device so the call needs no host-to-device copy.  hdr[1] is left
// alone: in a context's berr it is the sticky device-error count that
// rendgpu_sync and the host-pointer calls read and clear.
__global__ void k_call_begin(uint32_t *hdr, uint32_t n)
{
	if (threadIdx.x == 0) {
		hdr[0] = n;
		hdr[2] = 0u;
	}
}

} // namespace
} // namespace nb

using namespace nb;

extern "C" {

int rendgpu_init(struct rdata *rdp, const struct rendgpu_cfg *cfg)
{
	if (!rdp)
		return RENDGPU_EINVAL;
	if (find_ctx(rdp))
		return RENDGPU_ESTATE;
	Ctx *c = nullptr;
	nb_rdata *rd = reinterpret_cast<nb_rdata *>(rdp);
	int rc = new_ctx(&rd, 1, nullptr, cfg, &c);
	if (rc)
		return rc;
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
	return upload_static_all(c);
}

int rendgpu_upload_dynamic(struct rdata *rdp)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	int rc = upload_dynamic_all(c);
	if (!rc && rebuilds_tlas(c))
		rc = rebuild_tlas_tight(c);
	return rc;
}

int rendgpu_resaccum(struct rdata *rdp)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	return alloc_frame(c);
}

int rendgpu_clraccum(struct rdata *rdp)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	if (!c->have_frame)
		return fail(c, RENDGPU_ESTATE, "rendgpu_resaccum must come first");
	NB_CK(c, cudaSetDevice(c->device));
	NB_CK(c, cudaMemsetAsync(c->acc.p, 0, (size_t)c->npix * 12, c->stream));
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
	return readback_all(c, which);
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
	// berr: [0] count, [1] device errors (sticky until read), [2] work
	uint32_t *b = c->berr.as<uint32_t>();
	k_call_begin<<<1, 32, 0, c->stream>>>(b, n);
	NB_CK(c, cudaGetLastError());
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
	uint32_t *b = c->berr.as<uint32_t>();
	k_call_begin<<<1, 32, 0, c->stream>>>(b, n);
	NB_CK(c, cudaGetLastError());
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
	k_call_begin<<<1, 32, 0, c->stream>>>(hdr, n);
	NB_CK(c, cudaGetLastError());
	const float4 *r4 = static_cast<const float4 *>(rays);
	// abandoned rays count into the context's device-error word (allocated
	// with the context), which rendgpu_sync reports
	rc = launch_trace(c, r4, hdr, hdr + 2, raw, c->berr.as<uint32_t>() + 1,
	  nullptr);
	if (rc)
		return rc;
	k_refine<<<grid_for(c, n, 256), 256, 0, c->stream>>>(scene_of(c), r4,
	  hdr, raw, static_cast<float4 *>(hits));
	NB_CK(c, cudaGetLastError());
	return 0;
}

// Read and clear the context's device-error word (after the stream's work
// so far); it counts every device error since the last read.
static int take_device_errors(Ctx *c, uint32_t *e)
{
	*e = 0;
	NB_CK(c, cudaMemcpyAsync(e, c->berr.as<uint32_t>() + 1, 4,
	  cudaMemcpyDeviceToHost, c->stream));
	NB_CK(c, cudaStreamSynchronize(c->stream));
	if (*e)
		NB_CK(c, cudaMemsetAsync(c->berr.as<uint32_t>() + 1, 0, 4,
		  c->stream));
	return 0;
}

static int batch_errors(Ctx *c)
{
	uint32_t e = 0;
	int rc = take_device_errors(c, &e);
	if (rc)
		return rc;
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
	if (!c->mlp_ready) {
		int rc = nrc_reset(c, c->cfg.seed);
		if (rc)
			return rc;
	}
	k_nrc_encode<<<grid_for(c, n, 128), 128, 0, c->stream>>>(raw, n, c->box,
	  static_cast<__nv_bfloat16 *>(feats), grid_of(c));
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
	if (n && (misaligned16(feats) || misaligned16(out)))
		return fail(c, RENDGPU_EINVAL,
		  "feats and out must be non-null 16-byte aligned device pointers");
	NB_CK(c, cudaSetDevice(c->device));
	return nrc_infer(c, feats, n, reinterpret_cast<float4 *>(out));
}

int rendgpu_check_bounded_wait(struct rdata *rdp, uint32_t cycles,
                               uint32_t *out)
{
	Ctx *c = find_ctx(rdp);
	if (!c || !out)
		return RENDGPU_EINVAL;
	if (cycles == 0 || cycles > (1u << 31))
		return fail(c, RENDGPU_EINVAL, "cycles must be in 1..2^31");
	NB_CK(c, cudaSetDevice(c->device));
	NB_CK(c, c->waitchk.ensure(4 * sizeof(uint32_t)));
	k_wait_check<<<1, 32, 0, c->stream>>>(cycles, c->waitchk.as<uint32_t>());
	NB_CK(c, cudaGetLastError());
	NB_CK(c, cudaMemcpyAsync(out, c->waitchk.p, 3 * sizeof(uint32_t),
	  cudaMemcpyDeviceToHost, c->stream));
	NB_CK(c, cudaStreamSynchronize(c->stream));
	return 0;
}

int rendgpu_nrc_query_device(struct rdata *rdp, const float *entries,
                             uint32_t n, float *radiance, uint32_t npath)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	if (!c->mlp_ready)
		return fail(c, RENDGPU_ESTATE, "rendgpu_nrc_reset must come first");
	if (!c->have_dynamic)
		return fail(c, RENDGPU_ESTATE, "upload_dynamic must come first");
	if (n && (misaligned16(entries) || misaligned16(radiance)))
		return fail(c, RENDGPU_EINVAL,
		  "entries and radiance must be non-null 16-byte aligned device "
		  "pointers");
	NB_CK(c, cudaSetDevice(c->device));
	return nrc_query(c, reinterpret_cast<const float4 *>(entries), nullptr, n,
	  reinterpret_cast<float4 *>(radiance), npath,
	  c->berr.as<uint32_t>() + 1, false);
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
	if (n && (misaligned16(feats) || misaligned16(targets)))
		return fail(c, RENDGPU_EINVAL,
		  "feats and targets must be non-null 16-byte aligned device pointers");
	NB_CK(c, cudaSetDevice(c->device));
	return nrc_train(c, feats, reinterpret_cast<const float4 *>(targets), n,
	  update, grad, loss);
}

int rendgpu_nrc_train_raw_device(struct rdata *rdp, const float *raw,
                                 const float *targets, uint32_t n, int update,
                                 float *grad, float *grid_grad, float *loss)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	if (!c->mlp_ready)
		return fail(c, RENDGPU_ESTATE, "rendgpu_nrc_reset must come first");
	if (!c->have_dynamic)
		return fail(c, RENDGPU_ESTATE, "upload_dynamic must come first");
	if (n && (!raw || misaligned16(targets) ||
	  (grid_grad && misaligned16(grid_grad))))
		return fail(c, RENDGPU_EINVAL, "raw must be a non-null device "
		  "pointer, targets (and grid_grad) 16-byte aligned");
	if (n == 0)
		return 0;
	NB_CK(c, cudaSetDevice(c->device));
	NB_CK(c, c->rfeat.ensure((size_t)n * 128));
	k_nrc_encode<<<grid_for(c, n, 128), 128, 0, c->stream>>>(raw, n, c->box,
	  c->rfeat.as<__nv_bfloat16>(), grid_of(c));
	NB_CK(c, cudaGetLastError());
	GridSrc gs;
	gs.raw = raw;
	gs.box = c->box;
	gs.g_out = grid_grad;
	int rc = nrc_train(c, c->rfeat.p, reinterpret_cast<const float4 *>(
	  targets), n, update, grad, loss, nullptr, 0, 0, &gs);
	if (rc == 0 && grid_grad && !nrc_grid(c))
		NB_CK(c, cudaMemsetAsync(grid_grad, 0, kGridParams * 4, c->stream));
	return rc;
}

int rendgpu_nrc_grid(struct rdata *rdp, float *host, int write)
{
	Ctx *c = find_ctx(rdp);
	if (!c || !host)
		return RENDGPU_EINVAL;
	if (!c->mlp_ready)
		return fail(c, RENDGPU_ESTATE, "rendgpu_nrc_reset must come first");
	NB_CK(c, cudaSetDevice(c->device));
	if (write)
		NB_CK(c, cudaMemcpyAsync(c->grid_t.p, host, kGridParams * 4,
		  cudaMemcpyHostToDevice, c->stream));
	else
		NB_CK(c, cudaMemcpyAsync(host, c->grid_t.p, kGridParams * 4,
		  cudaMemcpyDeviceToHost, c->stream));
	NB_CK(c, cudaStreamSynchronize(c->stream));
	return 0;
}

int rendgpu_relmse_device(struct rdata *rdp, const float *ref, double *out)
{
	Ctx *c = find_ctx(rdp);
	if (!c || !ref || !out)
		return RENDGPU_EINVAL;
	if (!c->have_frame)
		return fail(c, RENDGPU_ESTATE, "rendgpu_resaccum must come first");
	NB_CK(c, cudaSetDevice(c->device));
	uint32_t n = c->sc[0].W * c->sc[0].H * 3u;
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
	// device errors of the asynchronous calls since the last check
	uint32_t e = 0;
	int rc = take_device_errors(c, &e);
	if (rc)
		return rc;
	c->st.device_errors = e;
	if (e)
		return fail(c, RENDGPU_EDEVICE, "device error in an asynchronous "
		  "call (" + std::to_string(e) + " abandoned rays or timed-out "
		  "tensor-core waits)");
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
	const SceneHost &h = c->sc[0];
	uint32_t n = (uint32_t)h.lights.size();
	if (c->dyn_active) {
		// the table of the last device-side update
		NB_CK(c, cudaSetDevice(c->device));
		uint32_t m = out ? std::min(n, cap) : 0u;
		if (m)
			NB_CK(c, cudaMemcpyAsync(out, c->lights.as<nb_glight>() +
			  h.light_off, (size_t)m * sizeof(nb_glight),
			  cudaMemcpyDeviceToHost, c->stream));
		float area = 0.0f;
		NB_CK(c, cudaMemcpyAsync(&area, c->dyn_area.p, sizeof(float),
		  cudaMemcpyDeviceToHost, c->stream));
		NB_CK(c, cudaStreamSynchronize(c->stream));
		if (total_area)
			*total_area = area;
		return (int)n;
	}
	if (out) {
		uint32_t m = n < cap ? n : cap;
		std::memcpy(out, h.lights.data(), (size_t)m *
		  sizeof(nb_glight));
	}
	if (total_area)
		*total_area = h.light_area;
	return (int)n;
}

int rendgpu_update_instances_device(struct rdata *rdp,
                                    const float *glob_device, uint32_t n,
                                    uint32_t flags)
{
	return update_instances(find_ctx(rdp), glob_device, n, flags);
}

int rendgpu_update_instances(struct rdata *rdp, const float *glob,
                             uint32_t n, uint32_t flags)
{
	Ctx *c = find_ctx(rdp);
	int rc = ready(c, false);
	if (rc)
		return rc;
	if (!glob || n != c->sc[0].rd->instcnt || c->batch)
		return fail(c, RENDGPU_EINVAL, "update: n must equal rd->instcnt "
		  "of a single-scene context");
	NB_CK(c, cudaSetDevice(c->device));
	NB_CK(c, cudaMemcpyAsync(c->dyn_glob.p, glob, (size_t)n * 64,
	  cudaMemcpyHostToDevice, c->stream));
	rc = update_instances(c, c->dyn_glob.as<float>(), n, flags);
	c->st.h2d_bytes = (uint64_t)n * 64;
	return rc;
}

int rendgpu_blas_host(struct rdata *rdp, uint32_t triofs, uint32_t tricnt,
                      void *nodes, uint32_t node_cap, void *tris,
                      uint32_t tri_cap, uint32_t info[3])
{
	if (!rdp || !info || tricnt == 0)
		return RENDGPU_EINVAL;
	const nb_rdata *rd = reinterpret_cast<const nb_rdata *>(rdp);
	if (!rd->tris || !rd->insts)
		return RENDGPU_EINVAL;
	// rdata holds no triangle count: the range must be an instance's mesh
	bool known = false;
	for (uint32_t i = 0; i < rd->instcnt && !known; i++)
		known = rd->insts[i].triofs == triofs &&
		  rd->insts[i].tricnt == tricnt;
	if (!known)
		return RENDGPU_EINVAL;
	blas_out b;
	std::string err;
	if (!build_blas(rd, triofs, tricnt, blas_params(), &b, &err))
		return RENDGPU_EINVAL;
	info[0] = (uint32_t)b.nodes.size();
	info[1] = (uint32_t)b.tris.size();
	info[2] = b.depth;
	if (nodes && node_cap >= b.nodes.size())
		std::memcpy(nodes, b.nodes.data(), b.nodes.size() * sizeof(nb_qnode));
	if (tris && tri_cap >= b.tris.size())
		std::memcpy(tris, b.tris.data(), b.tris.size() * sizeof(nb_gtri));
	return 0;
}

int rendgpu_get_instances(struct rdata *rdp, float *xf, float *wbox,
                          uint32_t cap, uint32_t info[3])
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	if (!c->have_dynamic || c->batch)
		return fail(c, RENDGPU_ESTATE, "upload_dynamic of a single-scene "
		  "context must come first");
	if ((wbox || info) && !c->dyn_active)
		return fail(c, RENDGPU_ESTATE, "world boxes and build info exist "
		  "after a device-side update");
	NB_CK(c, cudaSetDevice(c->device));
	uint32_t n = std::min(cap, c->sc[0].rd->instcnt);
	std::vector<float4> gi(4 * (size_t)n), wb(2 * (size_t)n);
	if (xf && n)
		NB_CK(c, cudaMemcpyAsync(gi.data(), c->insts.p, (size_t)n * 64,
		  cudaMemcpyDeviceToHost, c->stream));
	if (wbox && n)
		NB_CK(c, cudaMemcpyAsync(wb.data(), c->dyn_wbox.p, (size_t)n * 32,
		  cudaMemcpyDeviceToHost, c->stream));
	if (info)
		NB_CK(c, cudaMemcpyAsync(info, c->dyn_info.p, 3 * sizeof(uint32_t),
		  cudaMemcpyDeviceToHost, c->stream));
	NB_CK(c, cudaStreamSynchronize(c->stream));
	for (uint32_t i = 0; i < n; i++) {
		if (xf)
			std::memcpy(xf + 12 * (size_t)i, &gi[4 * (size_t)i], 48);
		if (wbox) {
			const float4 &l = wb[2 * (size_t)i], &h = wb[2 * (size_t)i + 1];
			float v[6] = {l.x, l.y, l.z, h.x, h.y, h.z};
			std::memcpy(wbox + 6 * (size_t)i, v, sizeof(v));
		}
	}
	return (int)n;
}

static int set_resolve(Ctx *c, uint32_t op, float exposure)
{
	if (op > RENDGPU_RESOLVE_ACES || !(exposure > 0.0f) ||
	    !(exposure < FLT_MAX))
		return fail(c, RENDGPU_EINVAL, "resolve: op 0..2, exposure > 0");
	for (SceneHost &h : c->sc) {
		h.resolve = op;
		h.exposure = exposure;
	}
	return 0;
}

int rendgpu_set_resolve(struct rdata *rdp, uint32_t op, float exposure)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	return set_resolve(c, op, exposure);
}

int rendgpu_batch_set_resolve(struct rendgpu_batch *b, uint32_t op,
                              float exposure)
{
	Ctx *c = find_batch(b);
	if (!c)
		return RENDGPU_EINVAL;
	return set_resolve(c, op, exposure);
}

int rendgpu_capture(struct rdata *rdp, uint32_t bounce_mask, uint32_t cap)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	if (bounce_mask && (cap == 0u || cap > (1u << 24)))
		return fail(c, RENDGPU_EINVAL, "capture: cap must be 1..2^24");
	NB_CK(c, cudaSetDevice(c->device));
	drop_graph(c); // the captured launch sequence changes
	c->cap_mask = bounce_mask;
	c->cap_n = bounce_mask ? cap : 0u;
	if (!bounce_mask)
		return 0;
	size_t bytes = (size_t)__builtin_popcount(bounce_mask) *
	  cap_slot_bytes(cap);
	NB_CK(c, c->capbuf.ensure(bytes));
	NB_CK(c, cudaMemsetAsync(c->capbuf.p, 0, bytes, c->stream));
	return 0;
}

int rendgpu_captured(struct rdata *rdp, uint32_t bounce,
                     struct rendgpu_ray *rays, struct rendgpu_hit *hits,
                     struct rendgpu_ray *shadow, uint32_t counts[4])
{
	Ctx *c = find_ctx(rdp);
	if (!c || !counts)
		return RENDGPU_EINVAL;
	if (!captures(c, bounce))
		return fail(c, RENDGPU_EINVAL, "bounce " + std::to_string(bounce) +
		  " is not captured (rendgpu_capture)");
	NB_CK(c, cudaSetDevice(c->device));
	CapSlot cs = cap_slot(c, bounce);
	NB_CK(c, cudaMemcpyAsync(counts, cs.counts, 4 * sizeof(uint32_t),
	  cudaMemcpyDeviceToHost, c->stream));
	NB_CK(c, cudaStreamSynchronize(c->stream));
	uint32_t m = std::min(counts[0], c->cap_n);
	uint32_t ms = std::min(counts[2], c->cap_n);
	if (rays && m)
		NB_CK(c, cudaMemcpyAsync(rays, cs.rays, (size_t)m * 32,
		  cudaMemcpyDeviceToHost, c->stream));
	if (hits && m)
		NB_CK(c, cudaMemcpyAsync(hits, cs.hits, (size_t)m * 16,
		  cudaMemcpyDeviceToHost, c->stream));
	if (shadow && ms)
		NB_CK(c, cudaMemcpyAsync(shadow, cs.shadow, (size_t)ms * 32,
		  cudaMemcpyDeviceToHost, c->stream));
	NB_CK(c, cudaStreamSynchronize(c->stream));
	return 0;
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

int rendgpu_set_tune(struct rdata *rdp, const struct rendgpu_tune *t)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	NB_CK(c, cudaSetDevice(c->device));
	return set_tune(c, t);
}

int rendgpu_get_tune(struct rdata *rdp, struct rendgpu_tune *t)
{
	Ctx *c = find_ctx(rdp);
	if (!c || !t)
		return RENDGPU_EINVAL;
	*t = effective_tune(c);
	return 0;
}

int rendgpu_autotune(struct rdata *rdp, uint32_t frames,
                     struct rendgpu_tune *best, struct rendgpu_tune *log,
                     uint32_t cap, uint32_t *nlog)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	NB_CK(c, cudaSetDevice(c->device));
	return autotune(c, frames, best, log, cap, nlog);
}

int rendgpu_batch_init(struct rdata *const *rds, uint32_t n,
                       const uint32_t *max_depth,
                       const struct rendgpu_cfg *cfg,
                       struct rendgpu_batch **out)
{
	if (!out || !cfg)
		return RENDGPU_EINVAL;
	Ctx *c = nullptr;
	int rc = new_ctx(reinterpret_cast<nb_rdata *const *>(rds), n, max_depth,
	  cfg, &c);
	if (rc)
		return rc;
	c->batch = true;
	rendgpu_batch *b = reinterpret_cast<rendgpu_batch *>(c);
	std::lock_guard<std::mutex> lk(g_mu);
	g_batches.insert(b);
	*out = b;
	return 0;
}

int rendgpu_batch_release(struct rendgpu_batch *b)
{
	Ctx *c = find_batch(b);
	if (!c)
		return RENDGPU_EINVAL;
	{
		std::lock_guard<std::mutex> lk(g_mu);
		g_batches.erase(b);
	}
	cudaSetDevice(c->device);
	cudaStreamSynchronize(c->stream);
	free_ctx(c);
	return 0;
}

int rendgpu_batch_upload_static(struct rendgpu_batch *b)
{
	Ctx *c = find_batch(b);
	return c ? upload_static_all(c) : RENDGPU_EINVAL;
}

int rendgpu_batch_upload_dynamic(struct rendgpu_batch *b)
{
	Ctx *c = find_batch(b);
	return c ? upload_dynamic_all(c) : RENDGPU_EINVAL;
}

int rendgpu_batch_resaccum(struct rendgpu_batch *b)
{
	Ctx *c = find_batch(b);
	return c ? alloc_frame(c) : RENDGPU_EINVAL;
}

int rendgpu_batch_clraccum(struct rendgpu_batch *b)
{
	Ctx *c = find_batch(b);
	if (!c)
		return RENDGPU_EINVAL;
	if (!c->have_frame)
		return fail(c, RENDGPU_ESTATE, "resaccum must come first");
	NB_CK(c, cudaSetDevice(c->device));
	NB_CK(c, cudaMemsetAsync(c->acc.p, 0, (size_t)c->npix * 12, c->stream));
	return 0;
}

int rendgpu_batch_render(struct rendgpu_batch *b)
{
	Ctx *c = find_batch(b);
	if (!c)
		return RENDGPU_EINVAL;
	NB_CK(c, cudaSetDevice(c->device));
	c->last = 0;
	int rc = render_frame(c);
	if (rc)
		return rc;
	for (size_t i = 0; i < c->sc.size(); i++)
		__atomic_fetch_add(&c->sc[i].rd->rays, (unsigned int)(
		  c->scn_host[2 * i] + c->scn_host[2 * i + 1]), __ATOMIC_SEQ_CST);
	return 0;
}

int rendgpu_batch_readback(struct rendgpu_batch *b, int which)
{
	Ctx *c = find_batch(b);
	return c ? readback_all(c, which) : RENDGPU_EINVAL;
}

int rendgpu_batch_get_stats(struct rendgpu_batch *b,
                            struct rendgpu_stats *total,
                            struct rendgpu_scene_stats *per, uint32_t n)
{
	Ctx *c = find_batch(b);
	if (!c)
		return RENDGPU_EINVAL;
	if (total) {
		c->st.device_bytes = held_bytes(c);
		c->st.max_stack = need_stack(c);
		*total = c->st;
	}
	for (uint32_t i = 0; per && i < n && i < c->sc.size(); i++) {
		const SceneHost &h = c->sc[i];
		per[i].closest_rays = i < c->scn_host.size() / 2 ?
		  c->scn_host[2 * i] : 0;
		per[i].shadow_rays = i < c->scn_host.size() / 2 ?
		  c->scn_host[2 * i + 1] : 0;
		per[i].paths = (uint64_t)h.W * h.H * h.spp;
		per[i].pixels = (uint64_t)h.W * h.H;
	}
	return 0;
}

int rendgpu_batch_set_tune(struct rendgpu_batch *b,
                           const struct rendgpu_tune *t)
{
	Ctx *c = find_batch(b);
	if (!c)
		return RENDGPU_EINVAL;
	NB_CK(c, cudaSetDevice(c->device));
	return set_tune(c, t);
}

int rendgpu_batch_get_tune(struct rendgpu_batch *b, struct rendgpu_tune *t)
{
	Ctx *c = find_batch(b);
	if (!c || !t)
		return RENDGPU_EINVAL;
	*t = effective_tune(c);
	return 0;
}

int rendgpu_tune_save(struct rdata *rdp, const char *path)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	return tune_save(c, path);
}

int rendgpu_tune_load(struct rdata *rdp, const char *path)
{
	Ctx *c = find_ctx(rdp);
	if (!c)
		return RENDGPU_EINVAL;
	NB_CK(c, cudaSetDevice(c->device));
	return tune_load(c, path);
}

int rendgpu_batch_tune_save(struct rendgpu_batch *b, const char *path)
{
	Ctx *c = find_batch(b);
	if (!c)
		return RENDGPU_EINVAL;
	return tune_save(c, path);
}

int rendgpu_batch_tune_load(struct rendgpu_batch *b, const char *path)
{
	Ctx *c = find_batch(b);
	if (!c)
		return RENDGPU_EINVAL;
	NB_CK(c, cudaSetDevice(c->device));
	return tune_load(c, path);
}

int rendgpu_batch_autotune(struct rendgpu_batch *b, uint32_t frames,
                           struct rendgpu_tune *best,
                           struct rendgpu_tune *log, uint32_t cap,
                           uint32_t *nlog)
{
	Ctx *c = find_batch(b);
	if (!c)
		return RENDGPU_EINVAL;
	NB_CK(c, cudaSetDevice(c->device));
	return autotune(c, frames, best, log, cap, nlog);
}

int rendgpu_batch_get_stream(struct rendgpu_batch *b, void **stream)
{
	Ctx *c = find_batch(b);
	if (!c || !stream)
		return RENDGPU_EINVAL;
	*stream = (void *)c->stream;
	return 0;
}

int rendgpu_batch_last_error(struct rendgpu_batch *b)
{
	Ctx *c = find_batch(b);
	return c ? c->last : RENDGPU_EINVAL;
}

const char *rendgpu_batch_strerror(struct rendgpu_batch *b)
{
	Ctx *c = find_batch(b);
	return c ? c->msg.c_str() : "not a live batch handle";
}

} // extern "C"
