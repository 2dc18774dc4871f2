/*
 * rendgpu.h - C ABI of the B200 path-tracing core for nodebleed.
 *
 * A drop-in beside the reference renderer API (rend.h:149-162).  The
 * application keeps its own host side: scene import, `struct rdata`
 * (rend.h:119-147), rend_init, rend_prepstatic / rend_prepdynamic (the BVH8
 * build) and rend_resaccum.  It then hands the same `struct rdata *` to the
 * calls below, which upload the BVH/triangles/instances in a GPU layout and
 * render on the GPU.  `rendgpu_render` has the thrd_start_t shape of
 * `rend_render` (rend.c:3603), so a frame loop that does
 *     for i < nthreads: thrd_create(&t[i], rend_render, &rd);
 * can do the same with rendgpu_render: the first caller renders the frame,
 * later callers of the same frame return at once (rd->blknum is the claim,
 * as in rend.c:3623).  The caller then resets blknum/rays and bumps samples
 * exactly as main.c:424-426 does.
 *
 * All calls return 0 on success or a negative RENDGPU_E* code; nothing
 * exits or asserts.  rendgpu_strerror() describes the last error.
 * Pointers in signatures are host pointers unless the name says _device.
 */
#ifndef RENDGPU_H
#define RENDGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

struct rdata; /* rend.h:119-147, layout mirrored in nb_rdata.h */

enum rendgpu_status {
	RENDGPU_OK = 0,
	RENDGPU_EINVAL = -1,   /* bad argument or state */
	RENDGPU_ENOMEM = -2,   /* device or host allocation failed */
	RENDGPU_ECUDA = -3,    /* CUDA runtime error */
	RENDGPU_ELIMIT = -4,   /* scene exceeds a documented limit */
	RENDGPU_ESTATE = -5,   /* call order (init/upload/resaccum) violated */
	RENDGPU_EDEVICE = -6,  /* device-side error flag (e.g. stack overflow) */
	RENDGPU_ENODEV = -7    /* no CUDA device */
};

enum rendgpu_mode {
	RENDGPU_MODE_PATH = 0,    /* path tracing: NEE + cosine/mirror bounces */
	RENDGPU_MODE_PRIMARY = 1, /* reference live shading: (n+1)/2 * albedo */
	RENDGPU_MODE_NRC = 2      /* path tracing ended by the radiance cache at
	                             vertex 2, the first vertex after the primary
	                             hit; 2^16 training paths per frame, unbiased
	                             up to bounce reserved[2] (default 3) where
	                             the cache ends them too (self-training),
	                             train it: a frame's records train the
	                             cache during the next frame, beside its
	                             traversal and before its queries */
};

enum rendgpu_flags {
	RENDGPU_FLAG_TIMING = 1u << 0, /* record per-kernel CUDA events */
	RENDGPU_FLAG_COUNT = 1u << 1,  /* count node visits / triangle tests of
	                                  the closest-hit traces (slower) */
	RENDGPU_FLAG_GRAPH = 1u << 2   /* capture the frame's launch sequence
	                                  into a CUDA graph once and replay it
	                                  (always on for batches; ignored in
	                                  NRC mode); with TIMING only ms_frame
	                                  is recorded */
};

struct rendgpu_cfg {
	uint32_t size;       /* sizeof(struct rendgpu_cfg) */
	uint32_t max_depth;  /* closest-hit rays per path (>= 1) */
	uint32_t mode;       /* enum rendgpu_mode */
	uint32_t flags;      /* enum rendgpu_flags */
	uint64_t seed;       /* PCG32 seed of the path streams */
	int32_t  device;     /* CUDA device ordinal */
	uint32_t block;      /* threads per block of the trace kernels: 64,
	                        128 or 256 (0 = 256); see rendgpu_tune */
	uint32_t sched;      /* traversal schedule: 0 = default, 1 = step,
	                        2 = phase, 3 = ylitie (see trace.cuh) */
	uint32_t reserved[7]; /* [0]: float bits of the cache's Adam learning
	                         rate (0 = 1e-2); [1]: radiance-cache warm-up
	                         frames of unbiased tracing (0 = 1); [2]: bounce
	                         at which training paths end in the cache after
	                         the warm-up (0 = 3); [3]: cache training steps
	                         of 16384 samples per frame (0 = 6); [4] bit 0:
	                         keep the TLAS rendgpu_upload_dynamic converts
	                         from rd->bnodes instead of the device rebuild
	                         over tight instance boxes; [4] bit 1: keep the
	                         BLASes rendgpu_upload_static converts from
	                         rd->bnodes instead of building its own (SAH
	                         binary build collapsed to 8-wide nodes by
	                         cost); [4] bit 2: one wave of all paths
	                         where two concurrent waves would run (see
	                         rendgpu_tune.queue); [4] bit 3: the upload-time
	                         device TLAS rebuild splits level by level,
	                         greedily into 8 children, instead of building
	                         one CTA's binary SAH tree collapsed by cost
	                         (see RENDGPU_UPDATE_COLLAPSE); [5] bit 0: no hash
	                         grid in the cache's position encoding; [6]:
	                         cache training paths per frame (0 = 65536) */
};

/* A ray for the batch calls: origin, tmax, direction (32 bytes). */
struct rendgpu_ray {
	float ox, oy, oz, tmax;
	float dx, dy, dz, pad;
};

/* A hit: t (FLT_MAX on a miss), barycentrics u/v of v1/v2, and
 * id = tri << 12 | inst as in rend.c:890 (16 bytes). */
struct rendgpu_hit {
	float    t, u, v;
	uint32_t id;
};

struct rendgpu_stats {
	uint64_t rays;           /* closest + shadow rays of the last frame */
	uint64_t closest_rays;
	uint64_t shadow_rays;
	uint32_t trace_launches; /* closest-hit trace launches of the frame */
	uint32_t launches;       /* all kernel launches of the frame */
	float    ms_frame;       /* device time of the frame (TIMING flag) */
	float    ms_trace;       /* sum over closest-hit trace launches (fused
	                            launches also trace the previous bounce's
	                            shadow rays; see rendgpu_tune.fuse) */
	float    ms_shadow;      /* sum over separate shadow (any-hit) launches */
	float    ms_shade;       /* gen + shade + accumulate */
	uint32_t device_errors;  /* rays abandoned by a device error */
	uint32_t max_stack;      /* traversal stack entries the scene needs */
	uint64_t device_bytes;   /* device memory held by this context */
	uint64_t h2d_bytes;      /* host->device bytes of the last upload/render */
	uint64_t d2h_bytes;      /* device->host bytes of the last readback */
	uint64_t node_visits;    /* closest-hit node visits (COUNT flag) */
	uint64_t tri_tests;      /* closest-hit triangle tests (COUNT flag) */
	uint32_t bounce_closest[16]; /* closest-hit rays per bounce */
	uint32_t bounce_shadow[16];  /* shadow rays per bounce */
	uint32_t nrc_queries;    /* radiance-cache queries of the frame */
	uint32_t nrc_records;    /* training vertices recorded in the frame */
	float    ms_nrc;         /* cache inference + training (TIMING flag) */
	float    nrc_loss;       /* loss of the last training step in the frame
	                            (radiance-cache frames train on the previous
	                            frame's records; 0 in the first frame) */
};

/* Launch parameters of a context (rendgpu_set_tune / rendgpu_autotune).
 * Zero fields take the defaults. */
struct rendgpu_tune {
	uint32_t block;  /* threads per block of the trace kernels: 64, 128
	                    or 256 (default) */
	uint32_t stack;  /* traversal stack entries per thread in shared memory:
	                    24, 32 or 48; a depth below the scene's need (TLAS +
	                    BLAS depth + 2) gives the smallest that fits */
	uint32_t queue;  /* ray-queue capacity in camera slots: a frame runs in
	                    waves of this many paths through all bounces, one
	                    after another.  0 = the default: single-scene
	                    contexts of at least 2^20 slots run two
	                    waves of half the slots each, concurrently on two
	                    streams, so that each wave's launch tails overlap
	                    the other's work (cfg.reserved[4] bit 2 turns this
	                    off); others one wave of all paths.  Images do not
	                    depend on the waves. */
	uint32_t sched;  /* traversal schedule as rendgpu_cfg.sched (0 = cfg's) */
	float    ms;     /* autotune: median device ms per frame measured */
	uint32_t sort;   /* 1: reorder each bounce's rays by direction octant
	                    and origin cell before tracing (single-scene
	                    PATH/PRIMARY contexts); 0: queue order */
	uint32_t fuse;   /* 1: trace each bounce's shadow rays in the launch of
	                    the next bounce's closest hits (2 launches per
	                    bounce instead of 3); 2: separate launches;
	                    0: the default (fused) */
	uint32_t force;  /* 1: use `stack` as given even where the scene needs
	                    more (8 is then accepted too, for the ray-batch calls
	                    only): rays that overflow it are abandoned and
	                    reported, which tests the overflow handling; 0: the
	                    stack always fits (default) */
};

/* Per-scene counts of a batch frame. */
struct rendgpu_scene_stats {
	uint64_t closest_rays;
	uint64_t shadow_rays;
	uint64_t paths;   /* width * height * spp */
	uint64_t pixels;
};

/* Create the GPU context of `rd` (one per rdata).  Replaces nothing in the
 * reference; pairs with rend_init (rend.c:3000). */
int rendgpu_init(struct rdata *rd, const struct rendgpu_cfg *cfg);

/* Free everything of `rd`'s GPU context (pairs with rend_release,
 * rend.c:3025). */
int rendgpu_release(struct rdata *rd);

/* After rend_prepstatic (rend.c:3033): upload every BLAS reachable from
 * rd->insts, triangles, normals and materials.  The BLASes are built by the
 * library on the host's cores (binary SAH tree collapsed to the GPU node
 * layout; rendgpu_blas_host shows one), or converted node for node from the
 * reference's with cfg.reserved[4] bit 1.  A mesh with a NaN or infinite
 * vertex fails the built form with RENDGPU_EINVAL. */
int rendgpu_upload_static(struct rdata *rd);

/* After rend_prepdynamic (rend.c:3073): upload the TLAS, the instance
 * transforms and the light table.  The TLAS in rd->bnodes is checked and
 * converted (RENDGPU_EINVAL on a malformed tree; the context then needs a
 * successful upload before it traces again).  A single-scene context then
 * rebuilds it on the device over tight instance boxes (every vertex after
 * the instance's matrix instead of its root box's 8 corners), no deeper
 * than the converted tree: the same hits, fewer instances entered.
 * cfg.reserved[4] bit 0 keeps the converted tree. */
int rendgpu_upload_dynamic(struct rdata *rd);

/* After rend_resaccum (rend.c:3092): size the device accumulator and the
 * path/ray queues for rd->width x rd->height x rd->spp. */
int rendgpu_resaccum(struct rdata *rd);

/* Zero the device accumulator (rend_clraccum, rend.c:3103). */
int rendgpu_clraccum(struct rdata *rd);

/* Render one frame of rd->spp samples per pixel into the device
 * accumulator (rend_render, rend.c:3603).  rd->samples keys the random
 * streams and normalises the ARGB8 resolve, rd->rays receives the ray
 * count.  Returns 0 (int, thrd_start_t shape); errors are reported by
 * rendgpu_last_error(). */
int rendgpu_render(void *rd);

/* Copy the device accumulator to rd->acc and/or the ARGB8 image to rd->buf
 * (which = 1: acc, 2: buf, 3: both); NULL host pointers are skipped. */
int rendgpu_readback(struct rdata *rd, int which);

/* Closest hits of n host rays (ray exchange with intersect_tlas,
 * rend.c:1976); hits to host memory. */
int rendgpu_trace_rays(struct rdata *rd, const struct rendgpu_ray *rays,
                       uint32_t n, struct rendgpu_hit *hits);

/* Occlusion of n host rays up to their tmax (intersect_any_tlas,
 * rend.c:2883): occl[i] = 1 if anything is hit in (0, tmax). */
int rendgpu_occluded(struct rdata *rd, const struct rendgpu_ray *rays,
                     uint32_t n, uint8_t *occl);

/* Device-pointer forms of the two calls above, on the context's stream;
 * return without synchronising.  A ray the device had to abandon (a
 * traversal stack overflow; the upload's depth check makes this unreachable
 * for trees it accepts) comes back as a miss from the closest-hit form and as
 * occluded from the occlusion form, and counts into the context's
 * device-error word, which rendgpu_sync reports and clears. */
int rendgpu_trace_rays_device(struct rdata *rd, const void *rays_device,
                              uint32_t n, void *hits_device);
int rendgpu_occluded_device(struct rdata *rd, const void *rays_device,
                            uint32_t n, void *occl_device);

/* Closest hits of n device rays into device hits, like
 * rendgpu_trace_rays_device, but the call allocates no device memory.
 * No counterpart in the reference (it has no device memory at all).  It
 * exists for callers that cannot let a library call cudaMalloc or cudaFree
 * while they run: applications that hand out all device memory from their
 * own arena sized at start-up, and frame loops that cannot absorb the device
 * synchronisation an allocation or free can imply.  Its scratch (the raw hits
 * of at most RENDGPU_NOALLOC_MAX_RAYS rays plus three counters, 4 MiB +
 * 256 B) is one static device array that every GPU loading the library keeps
 * until the process exits.  n above the maximum returns RENDGPU_ELIMIT.
 * The first call in each CUDA context of a device (after a device reset,
 * again) looks up the array's device address (cudaGetSymbolAddress); make
 * that first call before any stream capture.
 * All calls share the array: calls whose work overlaps on the GPU (two
 * contexts, two streams, or two host threads) race on it; calls on one
 * context are ordered by its stream.  Rays the device had to abandon come
 * back as misses and count into the context's device-error word (allocated
 * with the context, not by this call), which rendgpu_sync reports as
 * RENDGPU_EDEVICE.  Returns without synchronising. */
#define RENDGPU_NOALLOC_MAX_RAYS (1u << 18)
int rendgpu_trace_rays_device_noalloc(struct rdata *rd,
                                      const void *rays_device, uint32_t n,
                                      void *hits_device);

/* Neural radiance cache (no counterpart in the reference).  A 64-input MLP
 * with 5 hidden layers of 64 ReLU units and 3 linear outputs, BF16 on the
 * tensor cores with FP32 master weights and Adam (beta 0.9/0.99, eps 1e-15).
 * Parameters: RENDGPU_NRC_PARAMS floats, layer l (0..4: 64x64, 5: 8x64 of
 * which 3 rows are used) stored [out][in] at offset l * 4096.
 * The position also goes through a trainable multiresolution hash grid
 * (Mueller et al. 2022): 8 levels of 2^17 entries of 2 FP32 features,
 * RENDGPU_NRC_GRID_PARAMS floats, level l at offset l * 262144, entry e at
 * 2 e; lattices of 16, 28, 52, 95, 172, 312, 565 and 1024 cells per axis
 * over the scene box, levels 0 and 1 indexed densely (x + (r+1)(y + (r+1)
 * z)), the others by (x ^ 2654435761 y ^ 805459861 z) mod 2^17.  Its Adam
 * steps are lazy: entries a batch does not touch keep their state.
 * cfg.reserved[5] bit 0 turns the grid off (its features are then 0). */
#define RENDGPU_NRC_PARAMS (5 * 4096 + 8 * 64)
#define RENDGPU_NRC_GRID_PARAMS (8 * 131072 * 2)

/* (Re)initialise the weights (Xavier uniform from `seed`), zero Adam. */
int rendgpu_nrc_reset(struct rdata *rd, uint64_t seed);
/* Copy the FP32 master weights out (write = 0) or in (write = 1). */
int rendgpu_nrc_weights(struct rdata *rd, float *host, int write);
/* Copy the hash grid out (write = 0) or in (write = 1). */
int rendgpu_nrc_grid(struct rdata *rd, float *host, int write);
/* 12 floats per query (world position, outgoing direction, normal,
 * albedo) -> 64 BF16 features: 0..15 the hash grid's features of the
 * position in the scene box (level l at 2l, 2l+1), 16..33 the position's
 * sin/cos(2^k pi x), k = 0..2, per axis, 34..41 the encoded direction,
 * 42..44 the normal mapped to [0,1], 45..47 the albedo, the rest zero.
 * Initialises the cache from cfg->seed if rendgpu_nrc_reset has not. */
int rendgpu_nrc_encode_device(struct rdata *rd, const float *raw_device,
                              uint32_t n, void *feats_device);
/* MLP outputs (r, g, b, 0) per query (tcgen05 tensor cores, TMEM
 * accumulators).  The device buffers of the infer and train calls must be
 * 16-byte aligned (RENDGPU_EINVAL otherwise). */
int rendgpu_nrc_infer_device(struct rdata *rd, const void *feats_device,
                             uint32_t n, float *out_device);
/* Diagnostic of the device-side timeout (no counterpart in the reference).
 * Every wait of the tensor-core kernels on their own UMMAs gives up after
 * 2^31 SM clock cycles (about 1.1 s at 1965 MHz) and is then reported as
 * RENDGPU_EDEVICE.  This call runs such a wait limited to `cycles`
 * (1..2^31) on a barrier nothing completes, then on one that completes:
 * out[0] = 1 if the first timed out, out[1] = 1 if the second succeeded,
 * out[2] = clock cycles the timed-out wait took.  Synchronises; the
 * context stays usable. */
int rendgpu_check_bounded_wait(struct rdata *rd, uint32_t cycles,
                               uint32_t *out);
/* The frame's cache lookup in one pass: for each of n queries, 4 float4 at
 * entries_device + 16 i hold (position, path index as uint32 bits),
 * (outgoing direction, throughput r), (normal, throughput g), (albedo,
 * throughput b); the query is encoded as rendgpu_nrc_encode_device does,
 * run through the MLP as rendgpu_nrc_infer_device does, and
 * radiance_device[4 path .. + 2] += throughput * max(output, 0).  Queries
 * whose path index is npath or more are skipped; two queries of one path
 * in a call race.  Device buffers 16-byte aligned (RENDGPU_EINVAL
 * otherwise); needs rendgpu_upload_dynamic (the encoding's scene box). */
int rendgpu_nrc_query_device(struct rdata *rd, const float *entries_device,
                             uint32_t n, float *radiance_device,
                             uint32_t npath);
/* Gradient of the relative L2 loss mean((y-t)^2 / (y^2 + 0.01)) over a
 * batch (targets: 4 floats per query, the 4th unused); update = 1 takes
 * one Adam step.  grad_device (RENDGPU_NRC_PARAMS floats) and loss_host
 * may be NULL; a non-NULL loss_host synchronises. */
int rendgpu_nrc_train_device(struct rdata *rd, const void *feats_device,
                             const float *targets_device, uint32_t n,
                             int update, float *grad_device, float *loss_host);
/* The same from raw inputs (12 floats per query, as for
 * rendgpu_nrc_encode_device): encoded with the current grid, and the grid
 * trained too: grid_grad_device (RENDGPU_NRC_GRID_PARAMS floats, may be
 * NULL) receives its gradient, update = 1 also takes the grid's Adam
 * step.  Needs rendgpu_upload_dynamic (the scene box). */
int rendgpu_nrc_train_raw_device(struct rdata *rd, const float *raw_device,
                                 const float *targets_device, uint32_t n,
                                 int update, float *grad_device,
                                 float *grid_grad_device, float *loss_host);

/* relMSE of this context's accumulated image (acc / rd->samples) against a
 * reference image (W*H*3 floats, device memory): mean over pixels and
 * channels of (x - r)^2 / (r^2 + 0.01), reduced in FP64 on the device. */
int rendgpu_relmse_device(struct rdata *rd, const float *ref_device,
                          double *out);

/* Wait for all work of the context.  Returns RENDGPU_EDEVICE when one of
 * the asynchronous _device calls since the last check (the no-alloc trace
 * included) met a device error (rays abandoned, or a tensor-core wait of the
 * cache that timed out); stats.device_errors then holds their number.  The
 * check reads and clears the context's device-error word, as the
 * host-pointer trace calls also do. */
int rendgpu_sync(struct rdata *rd);

/* The cudaStream_t every call of this context runs on (for callers that
 * order their own work or CUDA events against it). */
int rendgpu_get_stream(struct rdata *rd, void **stream);

/* Statistics of the last rendgpu_render / trace call. */
int rendgpu_get_stats(struct rdata *rd, struct rendgpu_stats *st);

/* The light table uploaded by rendgpu_upload_dynamic: n entries of 20
 * floats (v0, e0, e1, n, emit, cdf, area, pad x3); returns the count, or a
 * negative code.  `out` may be NULL to query the count. */
int rendgpu_get_lights(struct rdata *rd, float *out, uint32_t cap,
                       float *total_area);

/* Device-side scene update.  It replaces the host steps the reference's
 * frame loop runs whenever a transform changed (main.c:257-264): upd_rinsts
 * (main.c:117-157: each instance's world->object matrix as the inverse of
 * its object->world matrix, mat4.c:299, and its world box from the 8
 * transformed corners of its BLAS root box), rend_prepdynamic
 * (rend.c:3073-3090: the TLAS build, build_bvh8 rend.c:458-709) and, for the
 * path tracer, the world-space light table; the device does all three
 * from the new matrices alone, so a moving scene never round-trips through
 * host memory.  glob: n row-major 4x4 object->world matrices (tfmat.glob) in
 * rd->insts order, n = rd->instcnt, 4-byte aligned; the _device form takes
 * device memory, the other copies n * 64 bytes from host memory first.
 * The world->object matrices and world boxes are bit-identical to the host
 * bridge's.  The TLAS is this library's own device build (binned SAH, at
 * most as deep as the TLAS rendgpu_upload_dynamic uploaded, so the
 * traversal stack still fits); hits do not depend on its shape.  flags:
 * RENDGPU_UPDATE_REFIT keeps the last device build's topology and only
 * recomputes its boxes (faster, looser as instances move; the first update
 * always builds).  Single-scene contexts; needs rendgpu_upload_dynamic once
 * (which again makes the host-built TLAS current).  rd->insts and rd->aabbs
 * on the host are not touched.  A singular matrix zeroes that instance (it
 * is never hit) and counts into the device-error word (rendgpu_sync).  The
 * radiance cache keeps the encoding box of the upload.  Returns without
 * synchronising. */
#define RENDGPU_UPDATE_REFIT 1u
/* RENDGPU_UPDATE_TIGHT: bound each instance by every vertex of its mesh
 * after the new matrix instead of the 8 transformed corners of its BLAS root
 * box (a rotated instance's corner box can be much larger), and build or
 * refit the TLAS over those boxes; rendgpu_get_instances then reports them. */
#define RENDGPU_UPDATE_TIGHT 2u
/* How an update builds the TLAS.  By default scenes of up to 2048
 * instances get one CTA's binary SAH tree collapsed into 8-wide nodes by
 * cost, as the upload-time rebuild does, and larger ones a greedy 8-way
 * split level by level over all SMs.  Measured: 0.57 against 0.43 ms for
 * 1026 instances, the collapsed tree then 2.5% faster to traverse (scale
 * frame); 1.7 against 0.8 ms for 4096 instances, no faster to traverse
 * (stress frame).  RENDGPU_UPDATE_COLLAPSE / RENDGPU_UPDATE_LEVELS choose
 * one of them whatever the size (not both). */
#define RENDGPU_UPDATE_COLLAPSE 4u
#define RENDGPU_UPDATE_LEVELS 8u
int rendgpu_update_instances_device(struct rdata *rd,
                                    const float *glob_device, uint32_t n,
                                    uint32_t flags);
int rendgpu_update_instances(struct rdata *rd, const float *glob, uint32_t n,
                             uint32_t flags);
/* The device's instance records after the last upload or update (for
 * checks): xf[12 i ..] = world->object 3x4 of instance i; wbox[6 i ..] =
 * its world box (min xyz, max xyz) and info = (TLAS nodes, TLAS depth,
 * build overflow flag) of the last device-side update, which must exist
 * when wbox or info is asked for.  Any pointer may be NULL.  Returns the
 * number of instances copied (<= cap).  Synchronises. */
int rendgpu_get_instances(struct rdata *rd, float *xf, float *wbox,
                          uint32_t cap, uint32_t info[3]);
/* The BLAS rendgpu_upload_static builds for the mesh rd->tris[triofs ..
 * triofs + tricnt), which must be the triangle range of one of rd's
 * instances, built in host memory only (no device, no context; for
 * checks of the tree): nodes in the GPU layout (struct nb_qnode of
 * gpulayout.h, 80 bytes, root first, node_cap of them) and triangles
 * (struct nb_gtri, 48 bytes, tri_cap of them); info = (nodes, triangles,
 * depth).  Buffers that are too small (or NULL) are left untouched, so a
 * first call with NULLs returns the sizes.  No counterpart in the reference,
 * whose build is rend.c:458-709. */
int rendgpu_blas_host(struct rdata *rd, uint32_t triofs, uint32_t tricnt,
                      void *nodes, uint32_t node_cap, void *tris,
                      uint32_t tri_cap, uint32_t info[3]);

/* 8-bit resolve of the frame image (rd->buf through rendgpu_readback),
 * done in the accumulation pass of every later frame.  The reference packs
 * 255 * acc / samples per channel and lets values above 1 wrap
 * (accum_pckt, rend.c:3574-3577); that stays the default.  The tonemapped
 * forms (no counterpart in the reference) scale by `exposure`, apply
 * Reinhard x / (1 + x) or the fitted ACES curve of Narkowicz (2015), then
 * the sRGB transfer function, and round to the nearest 8-bit value. */
enum rendgpu_resolve_op {
	RENDGPU_RESOLVE_WRAP = 0,     /* the reference's wrapping pack */
	RENDGPU_RESOLVE_REINHARD = 1,
	RENDGPU_RESOLVE_ACES = 2
};
int rendgpu_set_resolve(struct rdata *rd, uint32_t op, float exposure);

/* Ray capture for parity checks (no counterpart in the reference, whose
 * rays never leave the CPU; it lets a test re-trace the very rays a GPU frame
 * traced with intersect_tlas / intersect_any_tlas, rend.c:1976/2883).  With
 * bounce_mask != 0, every later frame records for each bounce k < 32 whose
 * bit is set: an even sample (stride ceil(n / cap)) of at most `cap` of the
 * closest-hit rays traced at bounce k, together with the hits the frame
 * found for them (refined, as rendgpu_trace_rays returns them), and an even
 * sample of at most `cap` of the shadow rays shading generated at bounce k.
 * Only the first wave of camera slots is captured (rendgpu_tune.queue).
 * Each captured bounce adds two small launches; bounce_mask = 0 stops it. */
int rendgpu_capture(struct rdata *rd, uint32_t bounce_mask, uint32_t cap);
/* The last frame's capture of bounce k.  rays / hits / shadow hold `cap`
 * entries each (any may be NULL; a ray's pad word carries its path index);
 * counts[0] = closest rays returned, [1] = closest rays the first wave
 * traced at bounce k, [2] = shadow rays returned, [3] = shadow rays the
 * first wave generated at bounce k.
 * Synchronises. */
int rendgpu_captured(struct rdata *rd, uint32_t bounce,
                     struct rendgpu_ray *rays, struct rendgpu_hit *hits,
                     struct rendgpu_ray *shadow, uint32_t counts[4]);

/* Last error of any call on this thread's most recent context. */
int         rendgpu_last_error(struct rdata *rd);
const char *rendgpu_strerror(struct rdata *rd);

/* Launch parameters (no counterpart in the reference).  set_tune with a new
 * queue capacity re-sizes the queues and clears the accumulator; get_tune
 * reports the settings in effect.  rendgpu_autotune renders `frames` timed
 * frames (after one untimed) per candidate, tuning the schedule, the block
 * size, the stack depth and the queue capacity one at a time (coordinate
 * descent), keeps the fastest, and clears the accumulator; rd->samples is
 * not advanced.  Every measured setting with its ms goes to log[0..cap)
 * and their number to *nlog (either may be NULL).  Not in NRC mode. */
int rendgpu_set_tune(struct rdata *rd, const struct rendgpu_tune *t);
int rendgpu_get_tune(struct rdata *rd, struct rendgpu_tune *t);
int rendgpu_autotune(struct rdata *rd, uint32_t frames,
                     struct rendgpu_tune *best, struct rendgpu_tune *log,
                     uint32_t cap, uint32_t *nlog);
/* Tuned settings kept across runs (the reference fixes its variants at
 * compile time, rend.c:3597-3599).  tune_save stores the settings in effect
 * (and the last autotune's ms) in a text file under this GPU model (name, SM
 * count, compute capability) and this context's scene signature (a hash of
 * the mode and of every scene's triangle and instance counts, BVH depths,
 * image size, spp and path depth), replacing an older line of the same key.
 * tune_load applies the stored line of the same key and returns 1, or
 * returns 0 when the file or the line does not exist.  Both need
 * rendgpu_resaccum first. */
int rendgpu_tune_save(struct rdata *rd, const char *path);
int rendgpu_tune_load(struct rdata *rd, const char *path);

/* Batches (no counterpart in the reference, which renders one rdata per
 * rend_render): n scenes of uneven triangle counts, resolutions, spp and
 * depths rendered by one launch sequence over shared ray queues, captured
 * once into a CUDA graph and replayed every frame.  Each rdata is prepared
 * by the application exactly as for rendgpu_init (rend_prepstatic,
 * rend_prepdynamic, rend_resaccum); max_depth[i] bounds scene i's paths
 * (NULL: cfg->max_depth for all).  Every scene's image is bit-identical to
 * the same scene rendered alone with the same cfg.  At most 4096 instances
 * over all scenes (hit ids keep 12 instance bits).  In RENDGPU_MODE_NRC one
 * radiance cache serves the batch: each scene's positions are encoded in
 * its own box, and scenes 2..15 get an input feature of their own (scene
 * 16 shares scene 2's); the warm-up frame is bit-identical to each scene's
 * alone, later frames depend on what all scenes trained.  Cache frames are
 * launched directly, not from a graph.
 * batch_render renders one frame of every scene (rd->samples of each keys
 * its random streams; the caller bumps samples afterwards, as main.c does)
 * and adds each scene's rays to its rd->rays. */
struct rendgpu_batch;
int rendgpu_batch_init(struct rdata *const *rds, uint32_t n,
                       const uint32_t *max_depth,
                       const struct rendgpu_cfg *cfg,
                       struct rendgpu_batch **out);
int rendgpu_batch_release(struct rendgpu_batch *b);
int rendgpu_batch_upload_static(struct rendgpu_batch *b);
int rendgpu_batch_upload_dynamic(struct rendgpu_batch *b);
int rendgpu_batch_resaccum(struct rendgpu_batch *b);
int rendgpu_batch_clraccum(struct rendgpu_batch *b);
int rendgpu_batch_render(struct rendgpu_batch *b);
int rendgpu_batch_readback(struct rendgpu_batch *b, int which);
/* Totals of the last frame, and per-scene counts into per[0..n). */
int rendgpu_batch_get_stats(struct rendgpu_batch *b,
                            struct rendgpu_stats *total,
                            struct rendgpu_scene_stats *per, uint32_t n);
int rendgpu_batch_set_tune(struct rendgpu_batch *b,
                           const struct rendgpu_tune *t);
int rendgpu_batch_get_tune(struct rendgpu_batch *b, struct rendgpu_tune *t);
int rendgpu_batch_autotune(struct rendgpu_batch *b, uint32_t frames,
                           struct rendgpu_tune *best,
                           struct rendgpu_tune *log, uint32_t cap,
                           uint32_t *nlog);
/* rendgpu_tune_save / rendgpu_tune_load for a batch (its signature covers
 * every scene). */
int rendgpu_batch_tune_save(struct rendgpu_batch *b, const char *path);
int rendgpu_batch_tune_load(struct rendgpu_batch *b, const char *path);
int rendgpu_batch_get_stream(struct rendgpu_batch *b, void **stream);
/* rendgpu_set_resolve for every scene of the batch. */
int rendgpu_batch_set_resolve(struct rendgpu_batch *b, uint32_t op,
                              float exposure);
int         rendgpu_batch_last_error(struct rendgpu_batch *b);
const char *rendgpu_batch_strerror(struct rendgpu_batch *b);

#ifdef __cplusplus
}
#endif

#endif
