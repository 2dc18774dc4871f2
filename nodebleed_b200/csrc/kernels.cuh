// Wavefront path-tracing kernels (sm_100a).
//
// One frame = gen, then per bounce: closest-hit trace of the ray queue,
// shade (which appends next-bounce rays and shadow rays with warp-aggregated
// atomics), any-hit trace of the shadow queue; finally accumulate.  Every
// kernel is a grid-stride loop over a count it reads from device memory, so
// the whole frame is a fixed launch sequence (capturable in a CUDA graph).
//
// The per-path arithmetic follows the CPU oracle operation by operation
// (camera jitter, shading normal, next-event estimation, cosine bounce, PCG32
// streams, sin/cos polynomials), compiled without contraction, so a path whose
// hits agree with the oracle's produces the same bits.

#ifndef NB_KERNELS_CUH
#define NB_KERNELS_CUH

#include "nrc.cuh"
#include "trace.cuh"

namespace nb {

constexpr float kEps2 = 1e-3f;          // util.h:8 EPS2
constexpr float kInvPi = 0.318309886f;  // util.h:11 INV_PI

struct FrameDev {
	// queues: 2 float4 per ray: (o, tmax) (d, path as bits)
	float4   *q[2];
	float4   *hits;    // (t, u, v, id bits)
	float4   *shadow;  // 2 float4: (o, tfar) (d, path)
	float4   *scol;    // shadow contribution (c, 0)
	float4   *pT;      // (T.rgb, spec flag)
	float4   *pL;      // (L.rgb, 0)
	uint2    *rng;     // PCG32 state
	float    *acc;     // W*H*3
	uint32_t *buf;     // W*H ARGB8
	uint32_t *cnt;     // [0],[1] ray queues, [2] shadow, [3] errors,
	                   // [4] closest-hit work counter, [5] shadow work,
	                   // [6] shadow launches, [8+k] / [24+k] closest /
	                   // shadow rays of bounce k
	unsigned long long *rays; // [0] closest, [1] shadow
	unsigned long long *scn;  // per scene: [2s] closest, [2s+1] shadow rays
	uint32_t  npaths, npix;   // all scenes
	// neural radiance cache (mode 2): queries (4 float4: (pos, path),
	// (wo, T.x), (n, T.y), (albedo, T.z)) counted in cnt[40], training
	// records (6 float4: (pos, path), wo, n, albedo, L before, T) in cnt[41]
	float4   *nq;
	float4   *nrec;
	uint32_t  nq_cap, nrec_cap;
	uint32_t *ncnt; // [0] queries, [1] records (cnt + 40 of the frame's
	                // first wave; every wave appends to the same arrays)
};

// Path flags kept in the bits of pT.w.
constexpr uint32_t kPathSpec = 1u;   // arrived by a mirror bounce
constexpr uint32_t kPathTrain = 2u;  // unbiased cache-training path

// Frame-wide arguments; everything per scene (camera, seed, sizes, depth,
// the cache's training-path stride) is in the ScenePar table.
struct FrameArgs {
	uint32_t depth;   // bounces of the launch sequence: max over scenes
	uint32_t mode;    // 0 path, 1 primary, 2 path with radiance cache
	uint32_t nrc_end; // mode 2: from this bounce on, training paths end in
	                  // the cache too (self-training); 0xffffffff: never
	                  // (warm-up frames)
};

// ------------------------------------------------------------- sampling --

__device__ __forceinline__ uint32_t pcg_next(uint64_t &st, uint64_t inc)
{
	uint64_t old = st;
	st = old * 6364136223846793005ull + inc;
	uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
	uint32_t rot = (uint32_t)(old >> 59u);
	return (xs >> rot) | (xs << ((32u - rot) & 31u));
}

__device__ __forceinline__ uint64_t pcg_inc(uint32_t path)
{
	return ((uint64_t)path << 1u) | 1u;
}

__device__ __forceinline__ uint64_t pcg_start(uint64_t seed, uint32_t frame,
                                              uint32_t path)
{
	uint64_t inc = pcg_inc(path), st = 0;
	pcg_next(st, inc);
	st += seed + 0x9e3779b97f4a7c15ull * ((uint64_t)frame + 1u);
	pcg_next(st, inc);
	return st;
}

__device__ __forceinline__ float rnd01(uint64_t &st, uint64_t inc)
{
	return __fmul_rn((float)(pcg_next(st, inc) >> 8), 0x1p-24f);
}

// sin and cos of 2*pi*u, u in [0,1): quadrant from 4u, Taylor polynomials
// of sin/cos(pi/2 f) on [0,1) (same constants and order as the oracle).
__device__ __forceinline__ void sincos2pi(float u, float *s, float *c)
{
	float u4 = __fmul_rn(u, 4.0f);
	int q = (int)u4;
	float f = __fsub_rn(u4, (float)q);
	float f2 = __fmul_rn(f, f);
	float sp = __fmul_rn(f, __fadd_rn(1.57079633f, __fmul_rn(f2,
	  __fadd_rn(-0.645964098f, __fmul_rn(f2, __fadd_rn(0.0796926262f,
	  __fmul_rn(f2, __fadd_rn(-0.00468175414f, __fmul_rn(f2,
	  __fadd_rn(0.000160441185f, __fmul_rn(f2, -3.59884324e-06f)))))))))));
	float cp = __fadd_rn(1.0f, __fmul_rn(f2, __fadd_rn(-1.23370055f,
	  __fmul_rn(f2, __fadd_rn(0.253669508f, __fmul_rn(f2,
	  __fadd_rn(-0.0208634808f, __fmul_rn(f2, __fadd_rn(0.000919260275f,
	  __fmul_rn(f2, __fadd_rn(-2.52020424e-05f,
	  __fmul_rn(f2, 4.71087478e-07f))))))))))));
	switch (q & 3) {
	case 0: *s = sp; *c = cp; break;
	case 1: *s = cp; *c = -sp; break;
	case 2: *s = -sp; *c = -cp; break;
	default: *s = -cp; *c = sp; break;
	}
}

// GGX (Trowbridge-Reitz) microfacet conductor, alpha = roughness (Walter et
// al. 2007): Smith G1 for GGX and Schlick's Fresnel with F0 = albedo.  Same
// operation order as the CPU oracle.
__device__ __forceinline__ float ggx_g1(float a2, float nv)
{
	return __fdiv_rn(__fmul_rn(2.0f, nv), __fadd_rn(nv, __fsqrt_rn(
	  __fadd_rn(a2, __fmul_rn(__fsub_rn(1.0f, a2), __fmul_rn(nv, nv))))));
}

__device__ __forceinline__ void schlick(const float f0[3], float c,
                                        float out[3])
{
	float m = __fsub_rn(1.0f, c);
	float m2 = __fmul_rn(m, m);
	float m5 = __fmul_rn(__fmul_rn(m2, m2), m);
	for (int a = 0; a < 3; a++)
		out[a] = __fadd_rn(f0[a], __fmul_rn(__fsub_rn(1.0f, f0[a]), m5));
}

__device__ __forceinline__ float dot3(const float a[3], const float b[3])
{
	return __fadd_rn(__fadd_rn(__fmul_rn(a[0], b[0]), __fmul_rn(a[1], b[1])),
	  __fmul_rn(a[2], b[2]));
}

// Orthonormal basis around n (rend.c:3126-3133).
__device__ __forceinline__ void onb(const float n[3], float ta[3],
                                    float tb[3])
{
	float sgn = copysignf(1.0f, n[2]);
	float oa = __fdiv_rn(-1.0f, __fadd_rn(sgn, n[2]));
	float ob = __fmul_rn(__fmul_rn(n[0], n[1]), oa);
	ta[0] = __fadd_rn(1.0f, __fmul_rn(__fmul_rn(__fmul_rn(sgn, n[0]), n[0]),
	  oa));
	ta[1] = __fmul_rn(sgn, ob);
	ta[2] = __fmul_rn(-sgn, n[0]);
	tb[0] = ob;
	tb[1] = __fadd_rn(sgn, __fmul_rn(__fmul_rn(n[1], n[1]), oa));
	tb[2] = -n[1];
}

// Warp-aggregated append: returns this lane's slot in the queue.
__device__ __forceinline__ uint32_t append(uint32_t *counter, bool want)
{
	uint32_t mask = __ballot_sync(__activemask(), want);
	if (!want)
		return 0;
	uint32_t lane = threadIdx.x & 31u;
	uint32_t leader = __ffs(mask) - 1;
	uint32_t base = 0;
	if (lane == leader)
		base = atomicAdd(counter, (uint32_t)__popc(mask));
	base = __shfl_sync(mask, base, leader);
	return base + __popc(mask & ((1u << lane) - 1u));
}

// Warp-aggregated count of the lanes with `want` into ctr[2 * scene + which]
// (lanes of one warp mostly share a scene).
__device__ __forceinline__ void count_scene(unsigned long long *ctr,
                                            uint32_t scene, uint32_t which,
                                            bool want)
{
	uint32_t mask = __ballot_sync(__activemask(), want);
	if (!want)
		return;
	uint32_t peers = __match_any_sync(mask, scene);
	if ((threadIdx.x & 31u) == (uint32_t)__ffs(peers) - 1u)
		atomicAdd(ctr + 2u * scene + which,
		  (unsigned long long)__popc(peers));
}

// Pixel of queue slot i: 8x4 pixel tiles, spp consecutive samples.
__device__ __forceinline__ bool tile_pixel(uint32_t i, uint32_t W,
                                           uint32_t H, uint32_t spp,
                                           uint32_t *x, uint32_t *y,
                                           uint32_t *s)
{
	uint32_t p = i / spp;
	*s = i - p * spp;
	uint32_t tile = p >> 5, in = p & 31u;
	uint32_t tpr = (W + 7u) >> 3;
	*x = (tile % tpr) * 8u + (in & 7u);
	*y = (tile / tpr) * 4u + (in >> 3);
	return *x < W && *y < H;
}

// --------------------------------------------------------------- kernels --

// Camera rays (rend.c:3293-3402, one lane) and path state for the camera
// slots [slot_lo, slot_hi) of all scenes (one wave of the ray queue).
__global__ void __launch_bounds__(256) k_gen(DScene S, FrameDev F,
                                             FrameArgs A, uint32_t slot_lo,
                                             uint32_t slot_hi)
{
	if (blockIdx.x == 0 && threadIdx.x == 0)
		F.cnt[4] = 0u;
	for (uint32_t i0 = slot_lo + blockIdx.x * blockDim.x; i0 < slot_hi;
	     i0 += gridDim.x * blockDim.x) {
		uint32_t i = i0 + threadIdx.x;
		uint32_t x = 0, y = 0, smp = 0, sc = 0;
		bool live = i < slot_hi;
		if (live)
			sc = scene_search(S, i, [](const ScenePar *p) {
				return __ldg(&p->slot_base); });
		const ScenePar *P = S.sp + sc;
		uint32_t W = __ldg(&P->W), spp = __ldg(&P->spp);
		live = live && tile_pixel(i - __ldg(&P->slot_base), W,
		  __ldg(&P->H), spp, &x, &y, &smp);
		uint32_t lpath = (y * W + x) * spp + smp;
		uint32_t path = __ldg(&P->path_base) + lpath;
		float o[3] = {0, 0, 0}, d[3] = {0, 0, 1};
		uint64_t st = 0;
		if (live) {
			ScenePar C = *P;
			uint64_t inc = pcg_inc(lpath);
			st = pcg_start(C.seed, C.frame, lpath);
			float u0 = rnd01(st, inc), u1 = rnd01(st, inc);
			float sx = __fadd_rn((float)x, __fsub_rn(u0, 0.5f));
			float sy = __fadd_rn((float)y, __fsub_rn(u1, 0.5f));
			sx = __fmaf_rn(sx, C.rw, -0.5f);
			sy = __fmaf_rn(sy, C.rh, -0.5f);
			sx = __fmul_rn(sx, C.fovfdist);
			sy = __fmul_rn(sy, C.fovfdist);
			sx = __fmul_rn(sx, C.aspect);
			float ups[3], riup[3], td[3];
			for (int a = 0; a < 3; a++) {
				ups[a] = __fmul_rn(C.up[a], sy);
				riup[a] = __fmaf_rn(C.ri[a], sx, -ups[a]);
			}
			if (C.tanfangle > 0.0f) {
				float u2 = rnd01(st, inc), u3 = rnd01(st, inc);
				float rad = __fsqrt_rn(u2), sn, cs;
				sincos2pi(u3, &sn, &cs);
				float lx = __fmul_rn(cs, rad), ly = __fmul_rn(sn, rad);
				for (int a = 0; a < 3; a++) {
					o[a] = __fmaf_rn(__fmaf_rn(C.ri[a], lx,
					  __fmul_rn(C.up[a], ly)), C.focrad, C.eye[a]);
					float fe = __fmaf_rn(C.fwd[a], C.fdist, C.eye[a]);
					td[a] = __fsub_rn(__fadd_rn(fe, riup[a]), o[a]);
				}
			} else {
				for (int a = 0; a < 3; a++) {
					o[a] = C.eye[a];
					td[a] = __fmaf_rn(C.fwd[a], C.fdist, riup[a]);
				}
			}
			float l2 = __fmaf_rn(td[0], td[0], __fmaf_rn(td[1], td[1],
			  __fmul_rn(td[2], td[2])));
			float il = __fdiv_rn(1.0f, __fsqrt_rn(l2));
			for (int a = 0; a < 3; a++)
				d[a] = __fmul_rn(td[a], il);
			uint32_t flags = (A.mode == 2u && (lpath + C.nrc_offset) %
			  C.nrc_stride == 0u) ? kPathTrain : 0u;
			F.pT[path] = make_float4(1.0f, 1.0f, 1.0f,
			  __uint_as_float(flags));
			F.pL[path] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
			F.rng[path] = make_uint2((uint32_t)st, (uint32_t)(st >> 32));
		}
		uint32_t slot = append(&F.cnt[0], live);
		if (live) {
			F.q[0][2u * slot] = make_float4(o[0], o[1], o[2], FLT_MAX);
			F.q[0][2u * slot + 1u] = make_float4(d[0], d[1], d[2],
			  __uint_as_float(path));
		}
	}
}

// Closest-hit trace of a ray queue (count in *count): raw hits.
// COUNT adds visit / triangle-test counts to counts[0..1]; SCHED picks the
// traversal schedule.  Blocks of 64, 128 or 256 threads (the launch bound
// keeps 64 registers per thread for each).
template <int SCHED, int STACK, bool COUNT>
__global__ void __launch_bounds__(256, 4) k_trace(DScene S, const float4 *rays,
                                               const uint32_t *count,
                                               uint32_t *work, float4 *hits,
                                               uint32_t *errs,
                                               unsigned long long *nrays,
                                               unsigned long long *counts)
{
	extern __shared__ uint2 sstk[];
	uint32_t n = *count;
	if (blockIdx.x == 0 && threadIdx.x == 0 && nrays)
		atomicAdd(nrays, (unsigned long long)n);
	SinkRaw sink{hits, errs, COUNT ? counts : nullptr};
	trace_persistent<SCHED, false, STACK, COUNT>(S, rays, n, work,
	  sstk + threadIdx.x, blockDim.x, sink);
}

// Any-hit trace of API rays: occl[i] = hit in (0, tmax).
template <int SCHED, int STACK>
__global__ void __launch_bounds__(256, 4) k_occluded(DScene S,
                                                  const float4 *rays,
                                                  const uint32_t *count,
                                                  uint32_t *work, uint8_t *occl,
                                                  uint32_t *errs)
{
	extern __shared__ uint2 sstk[];
	SinkOccl sink{occl, errs};
	trace_persistent<SCHED, true, STACK, false>(S, rays, *count, work,
	  sstk + threadIdx.x, blockDim.x, sink);
}

// Unoccluded shadow rays add their carried contribution to the path.
struct SinkShadow {
	const float4 *rays;
	const float4 *scol;
	float4       *pL;
	uint32_t     *errs;
	__device__ void operator()(uint32_t i, const Trav &T, uint32_t err)
	{
		if (err) {
			atomicAdd(errs, 1u);
			return;
		}
		if (T.found)
			return;
		uint32_t path = __float_as_uint(rays[2u * i + 1u].w);
		float4 c = scol[i];
		float4 L = pL[path];
		L.x = __fadd_rn(L.x, c.x);
		L.y = __fadd_rn(L.y, c.y);
		L.z = __fadd_rn(L.z, c.z);
		pL[path] = L;
	}
};

template <int SCHED, int STACK>
__global__ void __launch_bounds__(256, 4) k_shadow(DScene S, FrameDev F,
                                                  uint32_t k)
{
	extern __shared__ uint2 sstk[];
	uint32_t n = F.cnt[2];
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		atomicAdd(&F.rays[1], (unsigned long long)n);
		if (k < 16u)
			atomicAdd(&F.cnt[24u + k], n); // shadow rays of bounce k
	}
	SinkShadow sink{F.shadow, F.scol, F.pL, &F.cnt[3]};
	trace_persistent<SCHED, true, STACK, false>(S, F.shadow, n, &F.cnt[5],
	  sstk + threadIdx.x, blockDim.x, sink);
}

// Closest-hit trace of queue `rays` (bounce k) and, in the same launch and
// the same persistent loop, the shadow rays of bounce ks = k - 1: lanes take
// shadow rays once the closest-hit queue is drained, so the two queues'
// last, slowest rays overlap instead of ending two launches.  The shadow
// rays' contributions land in pL before bounce k is shaded, as with
// separate launches.  Ylitie schedule only.
template <int STACK, bool COUNT>
__global__ void __launch_bounds__(256, 4) k_trace_fused(DScene S, FrameDev F,
                                                     const float4 *rays,
                                                     const uint32_t *count,
                                                     uint32_t ks)
{
	extern __shared__ uint2 sstk[];
	uint32_t n = *count, ns = F.cnt[2];
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		atomicAdd(&F.rays[0], (unsigned long long)n);
		atomicAdd(&F.rays[1], (unsigned long long)ns);
		if (ks < 16u)
			atomicAdd(&F.cnt[24u + ks], ns); // shadow rays of bounce ks
	}
	SinkRaw sink{F.hits, &F.cnt[3], COUNT ? F.rays + 2 : nullptr};
	SinkShadow ss{F.shadow, F.scol, F.pL, &F.cnt[3]};
	trace_two<STACK, COUNT>(S, rays, n, F.shadow, ns, &F.cnt[4],
	  sstk + threadIdx.x, blockDim.x, sink, ss);
}

// Raw hits -> the reference's hit record (t, u, v, tri << 12 | inst).
__global__ void __launch_bounds__(256) k_refine(DScene S, const float4 *rays,
                                                const uint32_t *count,
                                                const float4 *raw,
                                                float4 *hits)
{
	uint32_t n = *count;
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
	     i += gridDim.x * blockDim.x) {
		float4 a = rays[2u * i], b = rays[2u * i + 1u];
		float4 h = raw[i];
		THit th{h.x, __float_as_uint(h.y), __float_as_uint(h.z)};
		hits[i] = finish_hit(S, a.x, a.y, a.z, b.x, b.y, b.z, th);
	}
}

// Radiance-cache position of a vertex: in its scene's box, clamped to
// [0,1], with the scene's feature code added to x (nrc_encode decodes it;
// its box is then the identity), and the path index.
__device__ __forceinline__ float4 nrc_entry_pos(const ScenePar *P,
                                                const float pos[3],
                                                uint32_t path)
{
	float v[3];
	for (int a = 0; a < 3; a++)
		v[a] = fminf(fmaxf(__fmul_rn(__fsub_rn(pos[a], __ldg(&P->nrc_lo[a])),
		  __ldg(&P->nrc_inv[a])), 0.0f), 1.0f);
	return make_float4(__fadd_rn(v[0], __ldg(&P->nrc_off)), v[1], v[2],
	  __uint_as_float(path));
}

// Shade the hits of queue `cur` at bounce k; append next rays to queue
// 1-cur and shadow rays to the shadow queue.
__global__ void __launch_bounds__(256) k_shade(DScene S, FrameDev F,
                                               FrameArgs A, uint32_t cur,
                                               uint32_t k)
{
	uint32_t n = F.cnt[cur];
	const float4 *rays = F.q[cur];
	float4 *next = F.q[cur ^ 1u];
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		F.cnt[4] = 0u;
		F.cnt[5] = 0u;
		if (k < 16u)
			atomicAdd(&F.cnt[8u + k], n); // closest-hit rays of bounce k
	}
	for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < n;
	     i0 += gridDim.x * blockDim.x) {
		uint32_t i = i0 + threadIdx.x;
		bool live = i < n;
		bool want_ray = false, want_shadow = false;
		float no[3] = {0, 0, 0}, nd[3] = {0, 0, 0};
		float so[3] = {0, 0, 0}, sd[3] = {0, 0, 0}, sc[3] = {0, 0, 0};
		float tfar = 0.0f;
		uint32_t path = 0, sidx = 0;
		if (live) {
			float4 ra = rays[2u * i], rb = rays[2u * i + 1u];
			float4 h = F.hits[i];
			if (h.x != FLT_MAX) {
				THit th{h.x, __float_as_uint(h.y), __float_as_uint(h.z)};
				h = finish_hit(S, ra.x, ra.y, ra.z, rb.x, rb.y, rb.z, th);
			}
			path = __float_as_uint(rb.w);
			sidx = scene_of_path(S, path);
			const ScenePar *P = S.sp + sidx;
			uint32_t lpath = path - __ldg(&P->path_base);
			uint32_t depth = __ldg(&P->depth);
			float4 T = F.pT[path];
			float4 L = F.pL[path];
			if (h.x == FLT_MAX) {
				L.x = __fadd_rn(L.x, __fmul_rn(T.x, __ldg(&P->bg[0])));
				L.y = __fadd_rn(L.y, __fmul_rn(T.y, __ldg(&P->bg[1])));
				L.z = __fadd_rn(L.z, __fmul_rn(T.z, __ldg(&P->bg[2])));
				F.pL[path] = L;
			} else {
				uint32_t id = __float_as_uint(h.w);
				uint32_t inst = id & NB_INST_ID_MASK;
				uint32_t prim = id >> NB_INST_ID_BITS;
				const float4 *ip = S.insts + 4u * inst;
				float4 m0 = __ldg(ip), m1 = __ldg(ip + 1);
				float4 m2 = __ldg(ip + 2);
				uint32_t triofs = __float_as_uint(__ldg(ip + 3).y);
				const nb_rnrm *rn = S.nrms + triofs + prim;
				const float4 *rnv = reinterpret_cast<const float4 *>(rn);
				float4 n0 = __ldg(rnv), n1 = __ldg(rnv + 1);
				float4 n2 = __ldg(rnv + 2);
				uint32_t mtlid = __float_as_uint(n0.w);
				const float4 *mv = reinterpret_cast<const float4 *>(
				  S.mtls + mtlid);
				float4 mc = __ldg(mv), mf = __ldg(mv + 1);
				uint32_t mflags = __float_as_uint(mf.z);
				float col[3] = {mc.x, mc.y, mc.z};
				// shading normal (rend.c:3109 with the transpose)
				float u = h.y, v = h.z;
				float w = __fsub_rn(__fsub_rn(1.0f, u), v);
				float nn[3];
				nn[0] = __fadd_rn(__fmul_rn(n1.x, u), __fadd_rn(
				  __fmul_rn(n2.x, v), __fmul_rn(n0.x, w)));
				nn[1] = __fadd_rn(__fmul_rn(n1.y, u), __fadd_rn(
				  __fmul_rn(n2.y, v), __fmul_rn(n0.y, w)));
				nn[2] = __fadd_rn(__fmul_rn(n1.z, u), __fadd_rn(
				  __fmul_rn(n2.z, v), __fmul_rn(n0.z, w)));
				float mm[3];
				mm[0] = __fadd_rn(__fadd_rn(__fmul_rn(m0.x, nn[0]),
				  __fmul_rn(m1.x, nn[1])), __fmul_rn(m2.x, nn[2]));
				mm[1] = __fadd_rn(__fadd_rn(__fmul_rn(m0.y, nn[0]),
				  __fmul_rn(m1.y, nn[1])), __fmul_rn(m2.y, nn[2]));
				mm[2] = __fadd_rn(__fadd_rn(__fmul_rn(m0.z, nn[0]),
				  __fmul_rn(m1.z, nn[1])), __fmul_rn(m2.z, nn[2]));
				float ml = __fadd_rn(__fadd_rn(__fmul_rn(mm[0], mm[0]),
				  __fmul_rn(mm[1], mm[1])), __fmul_rn(mm[2], mm[2]));
				float il = __fdiv_rn(1.0f, __fsqrt_rn(ml));
				float n[3] = {__fmul_rn(mm[0], il), __fmul_rn(mm[1], il),
				  __fmul_rn(mm[2], il)};
				if (A.mode == 1u) {
					// rend.c:3435-3441
					L.x = __fmul_rn(__fmul_rn(__fadd_rn(n[0], 1.0f),
					  0.5f), col[0]);
					L.y = __fmul_rn(__fmul_rn(__fadd_rn(n[1], 1.0f),
					  0.5f), col[1]);
					L.z = __fmul_rn(__fmul_rn(__fadd_rn(n[2], 1.0f),
					  0.5f), col[2]);
					F.pL[path] = L;
				} else {
					float d[3] = {rb.x, rb.y, rb.z};
					float pos[3] = {__fmaf_rn(d[0], h.x, ra.x),
					  __fmaf_rn(d[1], h.x, ra.y),
					  __fmaf_rn(d[2], h.x, ra.z)};
					float dn = __fadd_rn(__fadd_rn(__fmul_rn(n[0], d[0]),
					  __fmul_rn(n[1], d[1])), __fmul_rn(n[2], d[2]));
					bool front = dn < 0.0f;
					if (!front) {
						n[0] = __fmul_rn(n[0], -1.0f);
						n[1] = __fmul_rn(n[1], -1.0f);
						n[2] = __fmul_rn(n[2], -1.0f);
					}
					uint2 rs = F.rng[path];
					uint64_t st = (uint64_t)rs.x | ((uint64_t)rs.y << 32);
					uint64_t inc = pcg_inc(lpath);
					float rl = rnd01(st, inc), ra_ = rnd01(st, inc);
					float rb_ = rnd01(st, inc), r0 = rnd01(st, inc);
					float r1 = rnd01(st, inc);
					F.rng[path] = make_uint2((uint32_t)st,
					  (uint32_t)(st >> 32));
					uint32_t pflags = __float_as_uint(T.w);
					bool spec = (pflags & kPathSpec) != 0u;
					bool train = (pflags & kPathTrain) != 0u;
					bool emissive = (mflags & NB_FLAG_EMISSIVE) != 0u;
					bool glossy = mc.w >= 0.5f && mf.x > 0.0f;
					bool mirror = mc.w >= 0.5f && !glossy;
					bool queried = false;
					if (A.mode == 2u && k >= 1u && !emissive) {
						// rendering paths end at vertex 2 (the first
						// vertex after the primary hit, mirrors
						// included); training paths at bounce nrc_end.
						// The cache supplies their remaining radiance.
						bool end = k >= A.nrc_end || !train;
						if (end) {
							// radiance cache query: the path ends here
							uint32_t qi = atomicAdd(&F.ncnt[0], 1u);
							if (qi < F.nq_cap) {
								float4 *q = F.nq + 4u * qi;
								q[0] = nrc_entry_pos(P, pos, path);
								q[1] = make_float4(-d[0], -d[1], -d[2], T.x);
								q[2] = make_float4(n[0], n[1], n[2], T.y);
								q[3] = make_float4(col[0], col[1], col[2],
								  T.z);
							}
							queried = true;
						}
						if (train && !end) {
							uint32_t ri = atomicAdd(&F.ncnt[1], 1u);
							if (ri < F.nrec_cap) {
								float4 *q = F.nrec + 6u * ri;
								q[0] = nrc_entry_pos(P, pos, path);
								q[1] = make_float4(-d[0], -d[1], -d[2], 0.0f);
								q[2] = make_float4(n[0], n[1], n[2], 0.0f);
								q[3] = make_float4(col[0], col[1], col[2],
								  0.0f);
								q[4] = make_float4(L.x, L.y, L.z, 0.0f);
								q[5] = make_float4(T.x, T.y, T.z, 0.0f);
							}
						}
					}
					if (queried) {
						// the cache supplies the rest of the path
					} else if (emissive) {
						if ((k == 0u || spec) && front) {
							L.x = __fadd_rn(L.x, __fmul_rn(T.x, col[0]));
							L.y = __fadd_rn(L.y, __fmul_rn(T.y, col[1]));
							L.z = __fadd_rn(L.z, __fmul_rn(T.z, col[2]));
							F.pL[path] = L;
						}
					} else if (mirror) {
						// perfect mirror
						float dd = __fadd_rn(__fadd_rn(__fmul_rn(d[0],
						  n[0]), __fmul_rn(d[1], n[1])),
						  __fmul_rn(d[2], n[2]));
						float s2 = __fmul_rn(2.0f, dd);
						for (int a = 0; a < 3; a++) {
							nd[a] = __fsub_rn(d[a], __fmul_rn(n[a], s2));
							no[a] = __fmaf_rn(nd[a], kEps2, pos[a]);
						}
						T.x = __fmul_rn(T.x, col[0]);
						T.y = __fmul_rn(T.y, col[1]);
						T.z = __fmul_rn(T.z, col[2]);
						T.w = __uint_as_float(pflags | kPathSpec);
						F.pT[path] = T;
						want_ray = k + 1u < depth;
					} else {
						T.w = __uint_as_float(pflags & ~kPathSpec);
						float wo[3] = {__fmul_rn(d[0], -1.0f),
						  __fmul_rn(d[1], -1.0f), __fmul_rn(d[2], -1.0f)};
						float nwo = dot3(n, wo);
						float a2 = __fmul_rn(mf.x, mf.x);
						uint32_t nl = __ldg(&P->light_cnt);
						if (glossy && !(nwo > 0.0f))
							nl = 0u; // the path ends here
						if (nl) {
							// pick an emitting triangle by area
							const float4 *lt = S.lights +
							  5u * __ldg(&P->light_off);
							uint32_t lo = 0, hi = nl - 1u;
							while (lo < hi) {
								uint32_t mid = (lo + hi) >> 1;
								float cdf = __ldg(&lt[5u * mid + 3u]).w;
								if (rl < cdf)
									hi = mid;
								else
									lo = mid + 1u;
							}
							const float4 *lp = lt + 5u * lo;
							float4 l0 = __ldg(lp), l1 = __ldg(lp + 1);
							float4 l2 = __ldg(lp + 2), l3 = __ldg(lp + 3);
							// v0 = l0.xyz, e0 = (l0.w, l1.x, l1.y),
							// e1 = (l1.z, l1.w, l2.x), n = (l2.y, l2.z, l2.w)
							// emit = l3.xyz
							float su = __fsqrt_rn(ra_);
							float b1 = __fmul_rn(su, __fsub_rn(1.0f, rb_));
							float b2 = __fmul_rn(su, rb_);
							float e0[3] = {l0.w, l1.x, l1.y};
							float e1[3] = {l1.z, l1.w, l2.x};
							float lv0[3] = {l0.x, l0.y, l0.z};
							float lnm[3] = {l2.y, l2.z, l2.w};
							float ld[3];
							for (int a = 0; a < 3; a++) {
								float p = __fadd_rn(__fadd_rn(lv0[a],
								  __fmul_rn(e0[a], b1)),
								  __fmul_rn(e1[a], b2));
								ld[a] = __fsub_rn(p, pos[a]);
							}
							float l2s = __fadd_rn(__fadd_rn(
							  __fmul_rn(ld[0], ld[0]),
							  __fmul_rn(ld[1], ld[1])),
							  __fmul_rn(ld[2], ld[2]));
							float ldist = __fsqrt_rn(l2s);
							float ilr = __fdiv_rn(1.0f, ldist);
							for (int a = 0; a < 3; a++)
								ld[a] = __fmul_rn(ld[a], ilr);
							float ndotl = __fadd_rn(__fadd_rn(
							  __fmul_rn(n[0], ld[0]),
							  __fmul_rn(n[1], ld[1])),
							  __fmul_rn(n[2], ld[2]));
							float cosl = -__fadd_rn(__fadd_rn(
							  __fmul_rn(lnm[0], ld[0]),
							  __fmul_rn(lnm[1], ld[1])),
							  __fmul_rn(lnm[2], ld[2]));
							tfar = __fsub_rn(ldist, __fmul_rn(2.0f, kEps2));
							if (ndotl > 0.0f && cosl > 0.0f &&
							    tfar > 0.0f) {
								float em[3] = {l3.x, l3.y, l3.z};
								float tc[3] = {T.x, T.y, T.z};
								float fr[3] = {col[0], col[1], col[2]};
								float wgt;
								if (glossy) {
									// F D G / (4 n.wo n.l) n.l cosl
									// area / l^2
									float hv[3] = {__fadd_rn(wo[0], ld[0]),
									  __fadd_rn(wo[1], ld[1]),
									  __fadd_rn(wo[2], ld[2])};
									float hil = __fdiv_rn(1.0f,
									  __fsqrt_rn(dot3(hv, hv)));
									for (int a = 0; a < 3; a++)
										hv[a] = __fmul_rn(hv[a], hil);
									float nh = dot3(n, hv);
									float lh = dot3(ld, hv);
									float dd = __fadd_rn(__fmul_rn(
									  __fmul_rn(nh, nh),
									  __fsub_rn(a2, 1.0f)), 1.0f);
									float Dm = __fdiv_rn(__fmul_rn(a2,
									  kInvPi), __fmul_rn(dd, dd));
									float G = __fmul_rn(ggx_g1(a2, nwo),
									  ggx_g1(a2, ndotl));
									wgt = __fmul_rn(__fdiv_rn(
									  __fmul_rn(Dm, G),
									  __fmul_rn(4.0f, nwo)), cosl);
									wgt = __fmul_rn(wgt,
									  __ldg(&P->light_area));
									wgt = __fdiv_rn(wgt, l2s);
									schlick(col, lh, fr);
								} else {
									wgt = __fmul_rn(ndotl, cosl);
									wgt = __fmul_rn(wgt, __fmul_rn(
									  kInvPi, __ldg(&P->light_area)));
									wgt = __fdiv_rn(wgt, l2s);
								}
								for (int a = 0; a < 3; a++) {
									sc[a] = __fmul_rn(__fmul_rn(
									  __fmul_rn(tc[a], fr[a]), em[a]),
									  wgt);
									so[a] = __fmaf_rn(ld[a], kEps2,
									  pos[a]);
									sd[a] = ld[a];
								}
								want_shadow = true;
							}
						}
						if (glossy && k + 1u < depth && nwo > 0.0f) {
							// microfacet normal from D(m) (m.n), reflect
							// wo; weight F G1(wo) G1(wi) (wo.m) /
							// ((n.wo) (n.m))
							float ct2 = __fdiv_rn(__fsub_rn(1.0f, r1),
							  __fadd_rn(1.0f, __fmul_rn(__fsub_rn(a2, 1.0f),
							  r1)));
							float ct = __fsqrt_rn(ct2);
							float s2 = __fsub_rn(1.0f, ct2);
							float st = __fsqrt_rn(s2 > 0.0f ? s2 : 0.0f);
							float sn, cs;
							sincos2pi(r0, &sn, &cs);
							float ta[3], tb[3], m[3];
							onb(n, ta, tb);
							float mx = __fmul_rn(st, cs);
							float my = __fmul_rn(st, sn);
							for (int a = 0; a < 3; a++)
								m[a] = __fadd_rn(__fadd_rn(
								  __fmul_rn(ta[a], mx),
								  __fmul_rn(tb[a], my)),
								  __fmul_rn(n[a], ct));
							float wom = dot3(wo, m);
							float s2w = __fmul_rn(2.0f, wom);
							for (int a = 0; a < 3; a++)
								nd[a] = __fsub_rn(__fmul_rn(m[a], s2w),
								  wo[a]);
							float nwi = dot3(n, nd);
							if (wom > 0.0f && nwi > 0.0f) {
								float w = __fdiv_rn(__fmul_rn(__fmul_rn(
								  ggx_g1(a2, nwo), ggx_g1(a2, nwi)), wom),
								  __fmul_rn(nwo, ct));
								float F[3];
								schlick(col, wom, F);
								T.x = __fmul_rn(__fmul_rn(T.x, F[0]), w);
								T.y = __fmul_rn(__fmul_rn(T.y, F[1]), w);
								T.z = __fmul_rn(__fmul_rn(T.z, F[2]), w);
								for (int a = 0; a < 3; a++)
									no[a] = __fmaf_rn(nd[a], kEps2, pos[a]);
								want_ray = true;
							}
						} else if (!glossy && k + 1u < depth) {
							float sn, cs;
							sincos2pi(r0, &sn, &cs);
							float s1 = __fsqrt_rn(r1);
							float lx = __fmul_rn(cs, s1);
							float ly = __fmul_rn(sn, s1);
							float lz = __fsqrt_rn(__fsub_rn(1.0f, r1));
							// onb (rend.c:3126)
							float sgn = copysignf(1.0f, n[2]);
							float oa = __fdiv_rn(-1.0f, __fadd_rn(sgn, n[2]));
							float ob = __fmul_rn(__fmul_rn(n[0], n[1]), oa);
							float ta[3] = {__fadd_rn(1.0f, __fmul_rn(
							  __fmul_rn(__fmul_rn(sgn, n[0]), n[0]), oa)),
							  __fmul_rn(sgn, ob), __fmul_rn(-sgn, n[0])};
							float tb[3] = {ob, __fadd_rn(sgn, __fmul_rn(
							  __fmul_rn(n[1], n[1]), oa)), -n[1]};
							for (int a = 0; a < 3; a++) {
								nd[a] = __fadd_rn(__fadd_rn(
								  __fmul_rn(ta[a], lx),
								  __fmul_rn(tb[a], ly)),
								  __fmul_rn(n[a], lz));
								no[a] = __fmaf_rn(nd[a], kEps2, pos[a]);
							}
							T.x = __fmul_rn(T.x, col[0]);
							T.y = __fmul_rn(T.y, col[1]);
							T.z = __fmul_rn(T.z, col[2]);
							want_ray = true;
						}
						F.pT[path] = T;
					}
				}
			}
		}
		if (S.nscenes > 1u) {
			count_scene(F.scn, sidx, 0u, live);
			count_scene(F.scn, sidx, 1u, want_shadow);
		}
		uint32_t rs_ = append(&F.cnt[cur ^ 1u], want_ray);
		if (want_ray) {
			next[2u * rs_] = make_float4(no[0], no[1], no[2], FLT_MAX);
			next[2u * rs_ + 1u] = make_float4(nd[0], nd[1], nd[2],
			  __uint_as_float(path));
		}
		uint32_t ss = append(&F.cnt[2], want_shadow);
		if (want_shadow) {
			F.shadow[2u * ss] = make_float4(so[0], so[1], so[2], tfar);
			F.shadow[2u * ss + 1u] = make_float4(sd[0], sd[1], sd[2],
			  __uint_as_float(path));
			F.scol[ss] = make_float4(sc[0], sc[1], sc[2], 0.0f);
		}
	}
}

// ---------------------------------------------------------- reordering --
//
// Counting sort of a ray queue by a 12-bit key: direction octant (3 bits)
// over a 3-bit-per-axis cell of the origin in the scene box, so rays of a
// warp share their child order and nearby geometry.  Order within a key is
// arbitrary; every path's result is independent of queue order.

constexpr uint32_t kSortKeys = 4096;

__device__ __forceinline__ uint32_t ray_key(float4 a, float4 b,
                                            const NrcBox &B)
{
	uint32_t oct = (b.x < 0.0f ? 1u : 0u) | (b.y < 0.0f ? 2u : 0u) |
	  (b.z < 0.0f ? 4u : 0u);
	float p[3] = {a.x, a.y, a.z};
	uint32_t cell = 0;
	for (int k = 0; k < 3; k++) {
		float u = (p[k] - B.lo[k]) * B.inv[k] * 8.0f;
		int c = (int)fminf(fmaxf(u, 0.0f), 7.0f);
		cell |= (uint32_t)c << (3 * k);
	}
	return (oct << 9) | cell;
}

// Histogram of the keys of queue `q` (count *n) into hist (kSortKeys).
__global__ void __launch_bounds__(256) k_sort_hist(const float4 *q,
                                                   const uint32_t *n,
                                                   NrcBox B, uint32_t *hist)
{
	__shared__ uint32_t h[kSortKeys];
	for (uint32_t i = threadIdx.x; i < kSortKeys; i += blockDim.x)
		h[i] = 0u;
	__syncthreads();
	uint32_t cnt = *n;
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
	     i += gridDim.x * blockDim.x)
		atomicAdd(&h[ray_key(q[2u * i], q[2u * i + 1u], B)], 1u);
	__syncthreads();
	for (uint32_t i = threadIdx.x; i < kSortKeys; i += blockDim.x)
		if (h[i])
			atomicAdd(&hist[i], h[i]);
}

// Exclusive scan of hist into offs; hist cleared for the next use
// (one block of 1024 threads, 4 keys each).
__global__ void __launch_bounds__(1024) k_sort_scan(uint32_t *hist,
                                                    uint32_t *offs)
{
	__shared__ uint32_t part[1024];
	uint32_t t = threadIdx.x;
	uint32_t v[4], s = 0;
	for (int k = 0; k < 4; k++) {
		v[k] = hist[4u * t + k];
		hist[4u * t + k] = 0u;
		s += v[k];
	}
	part[t] = s;
	__syncthreads();
	for (uint32_t d = 1; d < 1024u; d <<= 1) {
		uint32_t x = t >= d ? part[t - d] : 0u;
		__syncthreads();
		part[t] += x;
		__syncthreads();
	}
	uint32_t base = part[t] - s;
	for (int k = 0; k < 4; k++) {
		offs[4u * t + k] = base;
		base += v[k];
	}
}

// Scatter queue `src` (count *n) to `dst` in key order; *ndst = *n.
__global__ void __launch_bounds__(256) k_sort_scatter(const float4 *src,
                                                      const uint32_t *n,
                                                      NrcBox B,
                                                      uint32_t *offs,
                                                      float4 *dst,
                                                      uint32_t *ndst)
{
	uint32_t cnt = *n;
	if (blockIdx.x == 0 && threadIdx.x == 0)
		*ndst = cnt;
	for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < cnt;
	     i0 += gridDim.x * blockDim.x) {
		uint32_t i = i0 + threadIdx.x;
		bool live = i < cnt;
		float4 a = make_float4(0, 0, 0, 0), b = a;
		uint32_t key = 0xffffffffu;
		if (live) {
			a = src[2u * i];
			b = src[2u * i + 1u];
			key = ray_key(a, b, B);
		}
		// one atomic per run of equal keys in the warp
		uint32_t act = __ballot_sync(0xffffffffu, live);
		if (live) {
			uint32_t peers = __match_any_sync(act, key);
			uint32_t leader = __ffs(peers) - 1;
			uint32_t lane = threadIdx.x & 31u;
			uint32_t base = 0;
			if (lane == leader)
				base = atomicAdd(&offs[key], (uint32_t)__popc(peers));
			base = __shfl_sync(peers, base, leader);
			uint32_t pos = base + __popc(peers & ((1u << lane) - 1u));
			dst[2u * pos] = a;
			dst[2u * pos + 1u] = b;
		}
	}
}

// Parity capture: an even sample (stride ceil(n / cap)) of at most `cap`
// entries of a queue whose count n is on the device.  With raw hits, each
// sampled ray's closest hit is refined into the reference's record exactly
// as k_shade refines it.  out_n[0] = entries written, out_n[1] = n.
__global__ void __launch_bounds__(256) k_capture(DScene S, const float4 *rays,
                                                 const uint32_t *count,
                                                 const float4 *raw,
                                                 uint32_t cap,
                                                 float4 *out_rays,
                                                 float4 *out_hits,
                                                 uint32_t *out_n)
{
	uint32_t n = *count;
	uint32_t stride = n > cap ? (n + cap - 1u) / cap : 1u;
	uint32_t m = n ? (n - 1u) / stride + 1u : 0u;
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		out_n[0] = m;
		out_n[1] = n;
	}
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m;
	     i += gridDim.x * blockDim.x) {
		uint32_t j = i * stride;
		float4 a = rays[2u * j], b = rays[2u * j + 1u];
		out_rays[2u * i] = a;
		out_rays[2u * i + 1u] = b;
		if (out_hits) {
			float4 h = raw[j];
			THit th{h.x, __float_as_uint(h.y), __float_as_uint(h.z)};
			out_hits[i] = finish_hit(S, a.x, a.y, a.z, b.x, b.y, b.z, th);
		}
	}
}

// relMSE of the accumulated image (acc / samples) against a reference
// image: mean over pixels and channels of (x - r)^2 / (r^2 + 0.01),
// accumulated in FP64 (the only double-precision arithmetic on the device).
__global__ void __launch_bounds__(256) k_relmse(const float *acc, float inv,
                                                const float *ref,
                                                uint32_t n, double *out)
{
	double s = 0.0;
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
	     i += gridDim.x * blockDim.x) {
		double x = (double)acc[i] * (double)inv, r = ref[i];
		double d = x - r;
		s += d * d / (r * r + 0.01);
	}
	for (int o = 16; o > 0; o >>= 1)
		s += __shfl_down_sync(0xffffffffu, s, o);
	__shared__ double part[8];
	if ((threadIdx.x & 31) == 0)
		part[threadIdx.x >> 5] = s;
	__syncthreads();
	if (threadIdx.x == 0) {
		double t = 0.0;
		for (int w = 0; w < (int)(blockDim.x >> 5); w++)
			t += part[w];
		atomicAdd(out, t);
	}
}

// Tonemapped 8-bit channel of a linear radiance value x (exposure applied):
// op 1 = Reinhard x / (1 + x), op 2 = the fitted ACES curve of Narkowicz
// (2015), x (2.51 x + 0.03) / (x (2.43 x + 0.59) + 0.14) clamped to [0, 1];
// then the sRGB transfer function (IEC 61966-2-1) and rounding to the
// nearest of 0..255.  Negative and NaN inputs give 0.
__device__ __forceinline__ uint32_t tonemap8(float x, uint32_t op)
{
	float v = x > 0.0f ? x : 0.0f;
	if (op == 1u) {
		v = __fdiv_rn(v, __fadd_rn(1.0f, v));
	} else {
		float num = __fmul_rn(v, __fadd_rn(__fmul_rn(2.51f, v), 0.03f));
		float den = __fadd_rn(__fmul_rn(v, __fadd_rn(__fmul_rn(2.43f, v),
		  0.59f)), 0.14f);
		v = fminf(__fdiv_rn(num, den), 1.0f);
	}
	float s = v <= 0.0031308f ? __fmul_rn(12.92f, v) :
	  __fsub_rn(__fmul_rn(1.055f, powf(v, 1.0f / 2.4f)), 0.055f);
	int q = __float2int_rn(__fmul_rn(s, 255.0f));
	return (uint32_t)min(max(q, 0), 255);
}

// acc += sum over the pixel's samples; ARGB8 resolve (rend.c:3565-3580), or
// a tonemapped resolve (rendgpu_set_resolve).
// Pixels of all scenes: acc and buf hold the scenes' images back to back.
__global__ void __launch_bounds__(256) k_accum(DScene S, FrameDev F)
{
	for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < F.npix;
	     p += gridDim.x * blockDim.x) {
		uint32_t sc = scene_search(S, p, [](const ScenePar *q) {
			return __ldg(&q->pix_base); });
		const ScenePar *P = S.sp + sc;
		uint32_t spp = __ldg(&P->spp);
		float inv = __ldg(&P->inv);
		const float4 *pl = F.pL + __ldg(&P->path_base) +
		  (size_t)(p - __ldg(&P->pix_base)) * spp;
		float sx = 0.0f, sy = 0.0f, sz = 0.0f;
		for (uint32_t s = 0; s < spp; s++) {
			float4 L = pl[s];
			sx = __fadd_rn(sx, L.x);
			sy = __fadd_rn(sy, L.y);
			sz = __fadd_rn(sz, L.z);
		}
		float ax = __fadd_rn(F.acc[3u * p], sx);
		float ay = __fadd_rn(F.acc[3u * p + 1u], sy);
		float az = __fadd_rn(F.acc[3u * p + 2u], sz);
		F.acc[3u * p] = ax;
		F.acc[3u * p + 1u] = ay;
		F.acc[3u * p + 2u] = az;
		uint32_t op = __ldg(&P->resolve);
		uint32_t cx, cy, cz;
		if (op == 0u) {
			// the reference's pack: wraps instead of clamping
			cx = (uint32_t)__fmul_rn(255.0f, __fmul_rn(ax, inv));
			cy = (uint32_t)__fmul_rn(255.0f, __fmul_rn(ay, inv));
			cz = (uint32_t)__fmul_rn(255.0f, __fmul_rn(az, inv));
		} else {
			float e = __fmul_rn(inv, __ldg(&P->exposure));
			cx = tonemap8(__fmul_rn(ax, e), op);
			cy = tonemap8(__fmul_rn(ay, e), op);
			cz = tonemap8(__fmul_rn(az, e), op);
		}
		F.buf[p] = 0xff000000u | (cx & 0xffu) << 16 | (cy & 0xffu) << 8 |
		  (cz & 0xffu);
	}
}

} // namespace nb

#endif
