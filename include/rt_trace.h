/* rt_trace.h — C ABI of the B200 software ray-traversal engine.
 *
 * The engine takes over renderlab's software BVH traversal: the ray-query seam that its non-RT
 * GI, shadow and reflection passes call (shaders/gi_rays_software.wgsl:280-291 and
 * shaders/reflections_software_bvh4.wgsl:140-207), over the packed u32 geometry buffers that
 * src/gi_bvh.rs and src/reflection_software.rs write. Scenes are uploaded as those words,
 * verbatim; rays go in as 32-byte records and hits come out as the seam's hit records.
 *
 * Conventions: every function returns rt_status; on failure rt_get_last_error() describes it.
 * Device pointers are CUDA device addresses on the context's device; `stream` is a
 * cudaStream_t (NULL: the legacy default stream). No call traps or hangs the GPU: stack
 * overflows and device waits are bounded and reported through rt_get_stats().
 */
#ifndef RT_TRACE_H
#define RT_TRACE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RT_ABI_VERSION 1u

typedef enum rt_status {
  RT_OK = 0,
  RT_ERR_INVALID_ARG = 1,    /* null pointer, bad size, unknown enum */
  RT_ERR_LAYOUT = 2,         /* packed words fail validation (src/gi_bvh.rs:33-36 InvalidInput) */
  RT_ERR_OOM = 3,            /* device or host allocation refused / over the HBM budget */
  RT_ERR_STACK_OVERFLOW = 4, /* a traversal stack was full; the push was dropped and counted */
  RT_ERR_TIMEOUT = 5,        /* a bounded device or host wait gave up */
  RT_ERR_CUDA = 6,           /* a CUDA runtime call failed (src/lib.rs:138-160 Error::Fault) */
  RT_ERR_BUSY = 7,           /* the serving queue is full or closed */
  RT_ERR_UNSUPPORTED = 8     /* option not available for this layout / kernel */
} rt_status;

/* The two packed layouts. */
typedef enum rt_layout {
  RT_LAYOUT_GI = 0,         /* gi_geometry: 16-word header, 32-word instances (src/gi_bvh.rs:19-25) */
  RT_LAYOUT_REFLECTION = 1, /* rl_geometry: 8-word header, 24-word instances (reflection_software.rs:38-42) */
  RT_LAYOUT_REFLECTION_BVH2 = 2 /* the legacy median BVH2 reflection layout (reflection_software.rs:170-264,
                                   reflections_software.wgsl), as geometry dumps carry it; PLAIN kernel only */
} rt_layout;

/* Query modes: gi_traverse's mode argument (gi_rays_software.wgsl:214-217). For the reflection
 * layout CLOSEST is rs_closest and either any-hit mode is rs_blocked. */
typedef enum rt_mode {
  RT_CLOSEST = 0,     /* gi_closest / rs_closest */
  RT_ANY_SKY = 1,     /* gi_visible (any hit; instances flagged "casts no shadow" skipped) */
  RT_ANY_CASTERS = 2  /* gi_visible_within / rs_blocked */
} rt_mode;

/* Traversal kernels. PLAIN is the loop-for-loop transcription of the WGSL (bit-exact with it);
 * FAST runs the same arithmetic in a scheduled kernel (bit-exact with PLAIN); WIDE8 traverses
 * the engine's compressed 8-wide BVH with watertight triangle tests and an FP64 re-test of
 * near ties (same hit ids except near ties; t within 1e-5 relative of FP64). */
typedef enum rt_kernel {
  RT_KERNEL_PLAIN = 0,
  RT_KERNEL_FAST = 1,
  RT_KERNEL_WIDE8 = 2,
  RT_KERNEL_WIDE8_PACKET = 3 /* WIDE8 walked by warp-wide packets of 32 consecutive rays (top level and
                                BLAS), for coherent batches; WIDE8's results */
} rt_kernel;

/* One ray, 32 bytes: origin, tmin, direction (need not be unit length), tmax. */
typedef struct rt_ray {
  float o[3];
  float tmin;
  float d[3];
  float tmax;
} rt_ray;

/* Reflection closest hit, 20 bytes: t and the hardware ray-query record
 * (placement slot + 1, primitive, u bits, v bits); rec[0] == 0 is a miss
 * (reflections_software_bvh4.wgsl:42,90). */
typedef struct rt_hit {
  float t;
  uint32_t rec[4];
} rt_hit;

/* GI closest hit, 40 bytes: GiHit (gi_rays_software.wgsl:19). inst == 0xffffffff is a miss;
 * tri holds the three position indices, or (primitive, 0, 0) for meshes with a primitive table;
 * normal is unit_normal of the source-winding normal in world space. */
typedef struct rt_gi_hit {
  float t;
  uint32_t inst;
  uint32_t tri[3];
  float bary[2];
  float normal[3];
} rt_gi_hit;

/* Any-hit results are one uint32 per ray: 1 when something blocks the ray, else 0
 * (gi_visible returns the negation). */

/* Where the WIDE8 per-ray walk keeps each lane's node-group stack (rt_tuning.wide8_stack,
 * rt_plan_desc.stack; 0 there means unchanged / the context's choice). No counterpart in the
 * reference, whose WGSL loops keep a fixed array per invocation. */
#define RT_STACK_LOCAL 1u  /* 32 entries a lane in local memory, cached by L1 (the default) */
#define RT_STACK_SHARED 2u /* 16 entries a lane in shared memory: only for scenes whose 8-wide trees are
                            * at most 16 levels deep (else RT_ERR_UNSUPPORTED) */
/* Launch parameters the autotuner chooses (renderlab_b200.tune); zero fields keep defaults. */
typedef struct rt_tuning {
  uint32_t fast_refill;  /* FAST: idle lanes (1-32) a persistent warp waits for before taking more rays */
  uint32_t wide8_refill; /* WIDE8: the same */
  uint32_t wide8_stack;  /* WIDE8: RT_STACK_LOCAL or RT_STACK_SHARED */
  uint32_t wide8_entries; /* WIDE8: leaves per instance (1-1024) of the 8-wide top level that later
                           * rt_scene_prepare calls build: 1 enters each instance at its BLAS root;
                           * more split the instances' BLASes into world-space entries (default 256) */
  uint32_t reserved[4];
} rt_tuning;

typedef struct rt_ctx rt_ctx;
typedef struct rt_scene rt_scene;
typedef struct rt_blas rt_blas;

typedef struct rt_stats {
  uint64_t rays_traced;
  uint64_t stack_overflows; /* pushes dropped because a stack was full */
  uint64_t launches;
  uint64_t scene_bytes;     /* device bytes held by uploaded scenes */
} rt_stats;

/* ---- context ---- */
uint32_t rt_abi_version(void);
rt_status rt_ctx_create(int device, rt_ctx** out);
void rt_ctx_destroy(rt_ctx* ctx);
const char* rt_get_last_error(const rt_ctx* ctx);
rt_status rt_get_stats(rt_ctx* ctx, rt_stats* out);
rt_status rt_ctx_set_tuning(rt_ctx* ctx, const rt_tuning* tuning);
rt_status rt_ctx_get_tuning(const rt_ctx* ctx, rt_tuning* out);
/* Runs a small device kernel that reports the device's arithmetic conventions (signed-zero
 * min/max, correctly rounded reciprocal and square root) as 16 result words. */
rt_status rt_selftest(rt_ctx* ctx, uint32_t out[16]);

/* ---- scenes: packed words in, device-resident scene out ----
 * Replaces the renderer's `queue.write_buffer` of gi_geometry / rl_geometry
 * (gi_cache.rs:4480-4484, primary_ray_gpu.rs:3672-3709). The words are validated (ranges,
 * acyclic trees) before upload so that no traversal can read outside them. */
rt_status rt_scene_upload(rt_ctx* ctx, rt_layout layout, const uint32_t* words, size_t n_words,
                          rt_scene** out);
/* Rewrites the leading words (header, instance records, top level) of an uploaded scene, as
 * the renderer does each frame when transforms change. The mesh words must be unchanged. */
/* The upload's admission check alone, on the host (no device needed). info: instances,
 * top-level base, root, distinct triangles, distinct BLAS nodes, deepest BLAS, deepest top
 * level, 0. */
rt_status rt_scene_validate(rt_layout layout, const uint32_t* words, size_t n_words, uint32_t info[8],
                            char* err, size_t err_len);
rt_status rt_scene_update_records(rt_ctx* ctx, rt_scene* scene, const uint32_t* words,
                                  size_t n_words);
/* Builds the derived layout a kernel needs (RT_KERNEL_WIDE8: the compressed 8-wide BVH over the
 * scene's triangles, built on the host threads and uploaded). PLAIN and FAST need nothing. */
rt_status rt_scene_prepare(rt_ctx* ctx, rt_scene* scene, rt_kernel kernel);
/* Chooses the WIDE8 top level's entries per instance for this scene by measurement: for each
 * budget (NULL / 0 budgets: 1, 4, 16, 64, 256; each 1-1024), rebuilds only the 8-wide top level
 * and times a WIDE8 pass over `probe` seeded incoherent rays in the scene's world box (0:
 * 65,536; half closest-hit with uniform directions, half any-hit toward uniform points of the
 * box), then keeps the fastest, which the scene's later rt_scene_prepare calls also use, and
 * reports it in *chosen (0 for a scene without a top level, which is left as it is). Few large
 * instances favour 1 (each instance entered at its BLAS root); many small, deeply overlapping
 * ones favour more. Needs rt_scene_prepare(scene, RT_KERNEL_WIDE8) first; synchronous; the
 * scene's top level is rebuilt in place, so no other call may trace the scene meanwhile. No
 * counterpart in the reference, whose top level is the packed BVH4 over instance boxes
 * (src/instance_bvh.rs:162-460). */
rt_status rt_scene_tune_top(rt_ctx* ctx, rt_scene* scene, const uint32_t* budgets, uint32_t n_budgets,
                            uint32_t probe, uint32_t* chosen);
/* Levels of the deepest 8-wide BLAS (after rt_scene_prepare for WIDE8, else RT_ERR_UNSUPPORTED):
 * RT_STACK_SHARED needs at most 16. */
rt_status rt_scene_wide8_depth(const rt_scene* scene, uint32_t* depth);
/* Builds the 8-wide layout of these words on the host, as rt_scene_prepare does, and checks what
 * the WIDE8 kernels rely on: indices in range, each triangle in exactly one leaf, every child box
 * enclosing the triangles below it in exact arithmetic, empty
 * slots inverted, node exponents in the decodable range. No device needed. info: 8-wide nodes,
 * triangles, deepest level, distinct BLAS. No counterpart in the reference (its runtime BVH is
 * the 4-wide one). */
rt_status rt_wide8_check(rt_layout layout, const uint32_t* words, size_t n_words, uint32_t info[4], char* err,
                         size_t err_len);
rt_status rt_scene_release(rt_ctx* ctx, rt_scene* scene);
size_t rt_scene_device_bytes(const rt_scene* scene);

/* ---- traversal ----
 * rt_trace: the seam. d_rays holds n rt_ray; d_hits receives n rt_gi_hit (GI closest),
 * n rt_hit (reflection closest) or n uint32 (any-hit). Asynchronous on `stream`; allocates
 * nothing. */
rt_status rt_trace(rt_ctx* ctx, const rt_scene* scene, rt_mode mode, const rt_ray* d_rays,
                   void* d_hits, uint32_t n, void* stream);
/* rt_trace with an explicit kernel (rt_kernel) and, for FAST / WIDE8, an optional device
 * permutation (d_order[i] is the ray traced by thread i; NULL: identity). */
rt_status rt_trace_ex(rt_ctx* ctx, const rt_scene* scene, rt_mode mode, rt_kernel kernel,
                      const rt_ray* d_rays, const uint32_t* d_order, void* d_hits, uint32_t n,
                      void* stream);
/* Ray order keys for rt_order_rays. */
typedef enum rt_ray_order {
  RT_ORDER_NONE = 0,
  RT_ORDER_ORIGIN = 1,            /* Morton code of the origin in the scene's bounds */
  RT_ORDER_OCTANT_ORIGIN = 2,     /* direction octant, then the origin's Morton code */
  RT_ORDER_DIRECTION_ORIGIN = 3   /* octahedral direction cell, then a coarse origin code */
} rt_ray_order;
/* Writes to d_order (n uint32) a permutation of the rays that groups nearby, alike rays, for
 * rt_trace_ex. Uses the context's ordering scratch (allocated on first use, or sized ahead by
 * rt_ctx_reserve). Asynchronous on `stream`. */
rt_status rt_order_rays(rt_ctx* ctx, const rt_scene* scene, const rt_ray* d_rays, uint32_t n, rt_ray_order key,
                        uint32_t* d_order, void* stream);
/* GPU refit of the BLAS that instance `instance` uses (near_field::refit_bvh, near_field.rs:445-478,
 * on the device): the same vertices and triangles at new positions. GI layout: d_positions (3
 * floats a vertex, n_positions of them) replaces the BLAS's position words. Reflection layout: the
 * pre-edged triangles are rewritten from d_positions through d_indices (the mesh's triangle list,
 * as given to rt_blas_build). The node boxes are refit bottom-up with the host refit's arithmetic:
 * the words equal those of rt_blas_refit + rt_pack_scene. Asynchronous on `stream` (the first call
 * per BLAS reads its topology synchronously). Every instance of the BLAS sees the change. The
 * instance records and the top level are not touched: when the geometry leaves its records' world
 * boxes, rewrite them with rt_scene_update_records, as the reference refits and re-places its
 * instances. The scene's derived WIDE8 layout is dropped (rt_scene_prepare builds it again). */
rt_status rt_scene_refit(rt_ctx* ctx, rt_scene* scene, uint32_t instance, const float* d_positions,
                         uint32_t n_positions, const uint32_t* d_indices, uint32_t n_indices, void* stream);
/* Copies words [first, first + n) of the scene's device buffer to host memory (synchronous). */
rt_status rt_scene_read_words(rt_ctx* ctx, const rt_scene* scene, size_t first, size_t n, uint32_t* out);

/* ---- The GI cache's ray producers --------------------------------------------------------
 * A cache cell (32 bytes) as gi_cache.wgsl keeps it: query point, cell edge, octahedral normal
 * (pack2x16snorm) and the key word whose high 24 bits turn the cell's directions. */
typedef struct rt_gi_cell {
  float q[3];
  float edge;
  uint32_t normal;
  uint32_t key_b;
  uint32_t pad[2];
} rt_gi_cell;
#define RT_GI_DIRECTIONS 64u /* rays a cell */
#define RT_GI_ROTATE 4u      /* GI_F_ROTATE: turn each cell's directions by its key */
/* The cells' fixed directions as rays (gi_direction about gi_basis of the normal, from the
 * query point offset along it by gi_origin_offset; tmin 0, tmax 1e20): ray k of cell c is
 * d_rays[c * 64 + k] (gi_cache.wgsl:1046-1068, gi_cells.wgsl:463-487). */
rt_status rt_gi_cell_rays(rt_ctx* ctx, const rt_gi_cell* d_cells, uint32_t n_cells, uint32_t flags, rt_ray* d_rays,
                          void* stream);
/* The same rays traced against a GI-layout scene by the FAST kernel, generated in its ray refill
 * (no ray buffer): RT_CLOSEST gives the gather's rt_gi_hit per item (gi_gather_software.wgsl:89-94),
 * RT_ANY_SKY one uint32 per item, 1 when blocked (gi_ray's visibility, gi_cache.wgsl:1562-1575,
 * keeps the negation as a bit). Results at d_hits[c * 64 + k]. */
rt_status rt_trace_gi_cells(rt_ctx* ctx, const rt_scene* scene, rt_mode mode, const rt_gi_cell* d_cells,
                            uint32_t n_cells, uint32_t flags, void* d_hits, void* stream);
/* The GI cache's per-light visibility (gi_light, shaders/gi_cache.wgsl:2040-2077): for every cell
 * and light, whether the light reaches the cell (gi_light_affects, :2028-2036: lit, in front of
 * the cell's surface, within range, inside a spot cone) and, if so, whether gi_visible_within
 * finds nothing on the ray from the cell's offset origin (the gather rays' origin) toward it
 * (gi_light_direction, :1977-1983; tmax the light's distance, 1e20 for a directional light).
 * The rays are made inside the traversal's ray refill (no ray buffer). d_words receives
 * ceil(n_lights / 32) words a cell: bit l % 32 of word l / 32 set when light l reaches the cell
 * and its ray is clear. kernel: RT_KERNEL_FAST (bit-exact with the reference arithmetic) or
 * RT_KERNEL_WIDE8 (after rt_scene_prepare). The cache state around gi_light -- its shade queue,
 * the light-reuse and moved-caster shortcuts -- is the renderer's and not part of this call. */
typedef struct rt_gi_light { /* light_cluster.wgsl:10, 80 bytes */
  float position_range[4];
  float travel_outer[4];
  float rgb_inner[4];
  uint32_t kind[4]; /* kind[0]: 0 directional, 1 point, 2 spot */
  float source[4];
} rt_gi_light;
rt_status rt_trace_gi_lights(rt_ctx* ctx, const rt_scene* scene, rt_kernel kernel, const rt_gi_cell* d_cells,
                             uint32_t n_cells, const rt_gi_light* d_lights, uint32_t n_lights, uint32_t* d_words,
                             void* stream);

/* ---- Many batches in one launch ----------------------------------------------------------
 * Uneven ray batches of one scene, each with its own buffers and mode, traced by ONE persistent
 * launch that hands out rays from the concatenation of the batches. Per batch, the results are
 * exactly those rt_trace_ex would write for it alone with the same kernel. No counterpart in the
 * reference (its passes dispatch one compute shader per ray buffer). */
typedef struct rt_batch {
  const rt_ray* d_rays; /* device rays */
  void* d_hits;         /* device results: as rt_trace for this batch's mode */
  uint32_t n;
  rt_mode mode;
} rt_batch;
#define RT_MAX_BATCHES 4096u
/* Stream-ordered; the batch table is staged through the context (h_batches may be reused on
 * return). kernel: RT_KERNEL_FAST or RT_KERNEL_WIDE8 (one persistent launch), or RT_KERNEL_PLAIN
 * (one launch per batch, for comparison and for workloads too short to fill a persistent grid).
 * At most RT_MAX_BATCHES batches. */
rt_status rt_trace_batches(rt_ctx* ctx, const rt_scene* scene, rt_kernel kernel, const rt_batch* h_batches,
                           uint32_t n_batches, void* stream);

/* A prepared many-batch launch: its batch table resident on the device, an optional ray sort, and
 * the whole launch captured once in a CUDA graph and replayed by rt_plan_launch. The batches'
 * buffers must stay valid for the plan's life; their contents may change between launches (the
 * plan re-sorts on every launch). Launches of one plan must not overlap (they share its ray
 * counter): issue them on one stream. */
typedef struct rt_plan rt_plan;
typedef struct rt_plan_desc {
  rt_kernel kernel;   /* RT_KERNEL_FAST or RT_KERNEL_WIDE8; RT_KERNEL_PLAIN: a launch per batch */
  uint32_t refill;    /* idle lanes (1-32) before a warp takes more rays; 0: the context's tuning */
  rt_ray_order order; /* sort the launch's rays first (RT_ORDER_NONE: no sort; PLAIN takes none) */
  uint32_t graph;     /* 1: replay a captured CUDA graph; 0: launch directly */
  uint32_t stack;     /* WIDE8: RT_STACK_LOCAL or RT_STACK_SHARED; 0: the context's tuning */
} rt_plan_desc;
rt_status rt_plan_create(rt_ctx* ctx, const rt_scene* scene, const rt_batch* h_batches, uint32_t n_batches,
                         const rt_plan_desc* desc, rt_plan** out);
rt_status rt_plan_launch(rt_plan* plan, void* stream);
/* Rays the plan traces per launch and device bytes it holds (table, counter, sort scratch). */
rt_status rt_plan_info(const rt_plan* plan, uint64_t* rays, uint64_t* device_bytes);
rt_status rt_plan_destroy(rt_plan* plan);

/* ---- Serving ---------------------------------------------------------------------------
 * A request loop over several device-resident scenes: requests (host ray buffers of any size,
 * any mode) are submitted from any thread at any time and their hits written back to the
 * caller's host buffers. Scenes are admitted only while scenes plus launch slots fit
 * hbm_budget (else RT_ERR_OOM). A worker thread fills each free launch slot (launch_rays rays
 * of device buffers, its own stream) with chunks of pending requests of one scene in arrival
 * order and traces it with one many-batch launch of `kernel`; requests that arrive while slots
 * are busy join the next free slot, and the slots' copies and launches overlap on the device.
 * Each ray's result equals that of the same ray traced alone with the same kernel. No
 * counterpart in the reference (its passes trace inside the frame). Buffers of a request must
 * stay valid until rt_server_wait returns for it; pinned host buffers keep the copies
 * asynchronous. */
typedef struct rt_server rt_server;
typedef struct rt_server_desc {
  uint64_t hbm_budget;  /* device bytes for scenes + launch slots */
  uint32_t launch_rays; /* rays a launch slot holds (a request larger than this spans slots) */
  uint32_t slots;       /* launch slots in flight at once (1-64) */
  rt_kernel kernel;     /* RT_KERNEL_PLAIN, RT_KERNEL_FAST or RT_KERNEL_WIDE8 (scenes prepared on add,
                         * and a scene with a top level gets its entries tuned by rt_scene_tune_top) */
} rt_server_desc;
typedef struct rt_server_stats {
  uint64_t requests;    /* finished since the last reset */
  uint64_t rays;        /* traced since the last reset */
  uint64_t launches;
  double p50_ms, p99_ms, max_ms; /* request latency, submit to hits in host memory */
  double wall_s;        /* since the last reset */
  uint64_t device_bytes; /* resident scenes + launch slots */
  uint64_t pending;     /* requests with rays not yet on the device */
} rt_server_stats;
rt_status rt_server_create(rt_ctx* ctx, const rt_server_desc* desc, rt_server** out);
rt_status rt_server_add_scene(rt_server* srv, rt_layout layout, const uint32_t* words, size_t n_words, uint32_t* id);
rt_status rt_server_remove_scene(rt_server* srv, uint32_t id); /* RT_ERR_BUSY while it has requests */
rt_status rt_server_submit(rt_server* srv, uint32_t scene, rt_mode mode, const rt_ray* h_rays, uint32_t n,
                           void* h_hits, uint64_t* ticket);
/* Waits for a request (timeout_ms < 0: no limit); RT_ERR_TIMEOUT leaves it waitable again.
 * Returns the request's status and forgets the ticket. */
rt_status rt_server_wait(rt_server* srv, uint64_t ticket, int32_t timeout_ms);
rt_status rt_server_get_stats(rt_server* srv, rt_server_stats* out, int reset);
/* Failure injection on the host, for tests of the serving loop's error path: the next `launches`
 * slot launches fail with `status` (not RT_OK) before anything of them is enqueued, as a failing
 * copy or launch call would (the reference's Error::Fault, src/lib.rs:138-160). Every request
 * with rays in such a slot finishes with that status; the slot returns to service and later
 * requests run normally. 0 launches clears it. No device fault is involved. */
rt_status rt_server_fail_next(rt_server* srv, uint32_t launches, rt_status status);
/* Finishes every submitted request, then frees the slots and releases the scenes. */
rt_status rt_server_destroy(rt_server* srv);

/* Host-buffer form: copies rays in and hits out through the context's pinned staging and
 * device buffers (grown on first use, or sized ahead by rt_ctx_reserve), pipelined in chunks
 * over four streams. Returns when the hits are in h_hits. */
rt_status rt_trace_host(rt_ctx* ctx, const rt_scene* scene, rt_mode mode, rt_kernel kernel,
                        const rt_ray* h_rays, void* h_hits, uint32_t n);
/* Several host-buffer batches, each with its own mode and kernel, in one pipeline: the chunks of
 * all batches go through the same two streams in order, so one batch's first copy overlaps the
 * previous batch's last kernel (a frame's shadow, GI and reflection rays in one call). Returns
 * when every batch's hits are in its h_hits. No counterpart in the reference (its passes
 * dispatch on the GPU queue). */
typedef struct rt_host_batch {
  const rt_ray* h_rays;
  void* h_hits;
  uint32_t n;
  rt_mode mode;
  rt_kernel kernel;
} rt_host_batch;
rt_status rt_trace_host_batches(rt_ctx* ctx, const rt_scene* scene, const rt_host_batch* batches,
                                uint32_t n_batches);
rt_status rt_ctx_reserve(rt_ctx* ctx, uint32_t max_rays);
/* rt_trace_ex in an instrumented build that counts, over the batch, into counts[8]:
 * rays, top-level nodes, instance box tests, BLAS nodes, leaves, triangles tested, f64
 * re-tests, f64 final refinements (RT_KERNEL_WIDE8; the bit-exact kernels visit exactly what
 * the reference traversal visits). Synchronous. */
rt_status rt_trace_counted(rt_ctx* ctx, const rt_scene* scene, rt_mode mode, rt_kernel kernel,
                           const rt_ray* d_rays, void* d_hits, uint32_t n, uint64_t counts[8]);

/* Read bandwidth of the context's device in GB/s, for the traversal's roofline (no counterpart in
 * the reference): 16-byte loads that bypass L1 stream `reps` times over a device buffer of
 * `bytes` (at least 1 MiB), timed with CUDA events after one warm pass. A buffer well inside the
 * 126 MB L2 measures L2's read bandwidth, one far larger than L2 measures HBM's. Synchronous;
 * allocates and frees the buffer. */
rt_status rt_read_bandwidth(rt_ctx* ctx, uint64_t bytes, uint32_t reps, double* gbs);

/* ---- allocation-free traversal ----
 * No counterpart in the reference: renderlab always traverses inside its own renderer.
 * rt_trace_static is the FAST traversal for a caller that cannot allocate device memory -- an
 * engine whose frame loop forbids cudaMalloc, or one that keeps the packed words in its own
 * device buffer and creates no rt_ctx. It allocates nothing: the kernel's scratch (its ray
 * counter and overflow count) is a static 256-byte device array that each GPU loading the
 * library holds until exit. d_words must be words rt_scene_validate accepted, copied to the
 * device by the caller (16-byte aligned); n is at most RT_STATIC_MAX_RAYS, larger batches are
 * refused with RT_ERR_INVALID_ARG, as are d_rays / d_words off a 16-byte boundary and d_hits off a
 * 4-byte one. Hits are written as rt_trace writes them. The first call on
 * a device looks up the array's device address; make it before any stream capture. Every call
 * reuses (and first zeroes) the same array, so calls that overlap on the GPU race. */
#define RT_STATIC_MAX_RAYS (1u << 31)
rt_status rt_trace_static(rt_layout layout, const uint32_t* d_words, size_t n_words, rt_mode mode,
                          const rt_ray* d_rays, void* d_hits, uint32_t n, void* stream);
/* The pushes the last rt_trace_static call on the current device dropped on a full traversal
 * stack (its results may then miss hits), read from the same static array once `stream` has
 * finished. The next rt_trace_static call on the device zeroes the count. Synchronous. */
rt_status rt_trace_static_stack_drops(void* stream, uint64_t* out);

/* ---- host builders (the CPU side of the path: crates/asset/src/near_field.rs:172-541,
 * src/instance_bvh.rs:162-460, src/gi_bvh.rs, src/reflection_software.rs) ---- */
#define RT_BUILD_SAH 0u    /* build_bvh_sah (near_field.rs:184): binned SAH, median past depth 15 */
#define RT_BUILD_MEDIAN 1u /* build_bvh (near_field.rs:172) */
rt_status rt_blas_build(const float* positions, uint32_t n_positions, const uint32_t* indices,
                        uint32_t n_indices, uint32_t build_flags, rt_blas** out);
/* The same build on the context's device (binned SAH or median splits level by level, node
 * boxes quantised bottom-up on the device): host arrays in, a host BLAS out whose nodes, leaves,
 * indices and leaf sources equal rt_blas_build's word for word, including the median rebuild of
 * an SAH tree past 15 node levels. At most 2^29 triangles. Synchronous, on a stream of its own;
 * it holds the context's lock while it builds, so other calls on the same context wait. */
rt_status rt_blas_build_device(rt_ctx* ctx, const float* positions, uint32_t n_positions, const uint32_t* indices,
                               uint32_t n_indices, uint32_t build_flags, rt_blas** out);
/* info: nodes, leaves, positions, indices, root, depth */
rt_status rt_blas_info(const rt_blas* blas, uint32_t info[6]);
/* The 16-word runtime node records (gi_bvh.rs:191-203), 16 * nodes words. */
rt_status rt_blas_nodes(const rt_blas* blas, uint32_t* out);
/* The reordered triangle-list indices (near_field.rs:380-400), `indices` words. */
rt_status rt_blas_indices(const rt_blas* blas, uint32_t* out);
/* refit_bvh (near_field.rs:445-478): same vertices, new positions. */
rt_status rt_blas_refit(rt_blas* blas, const float* positions, uint32_t n_positions);
void rt_blas_free(rt_blas* blas);

/* One placement for the packers. model: object-to-world, 3 rows of 4; rows: the world-to-object
 * rows the record carries (words 0-11). GI: near_base is word 23 and extra words 24-31
 * (identity, map, map length, flags bit0 = casts no shadow, -, placement); word 28 (primitive
 * table) is derived. Reflection: slot is word 21, casts_shadow selects word 22. */
typedef struct rt_instance {
  float model[12];
  float rows[12];
  uint32_t mesh;
  uint32_t slot;
  uint32_t casts_shadow;
  uint32_t near_base;
  uint32_t extra[8];
} rt_instance;

/* Packs meshes and instances into the layout's words (gi_bvh.rs:151-274 + gi_cache.rs:4388-4488;
 * reflection_software.rs:285-388 + primary_ray_gpu.rs:3640-3662), with the instance top level
 * (instance_bvh.rs:162-220; tlas_mode -1 default (>= 40 instances), 0 off, 1 on).
 * mesh_primitives[m] != 0 adds the GI primitive table for mesh m (source indices given).
 * Call with out_words NULL to learn the size in *n_words. */
rt_status rt_pack_scene(rt_layout layout, const rt_blas* const* meshes, uint32_t n_meshes,
                        const float* const* mesh_positions, const uint32_t* const* mesh_indices,
                        const uint32_t* mesh_n_indices, const uint32_t* mesh_primitives,
                        const rt_instance* instances, uint32_t n_instances, int tlas_mode,
                        uint32_t* out_words, size_t* n_words);

/* The object box rt_pack_scene places for a mesh (6 floats: lo xyz, hi xyz): GI, every position
 * of the BLAS (gi_bvh.rs:70); reflection, the vertices of the source triangle list
 * (reflection_software.rs:336-346). */
rt_status rt_object_box(rt_layout layout, const rt_blas* blas, const float* positions, const uint32_t* indices,
                        uint32_t n_indices, float box[6]);
/* Moved instances, on the host: every instance's record gets its new rows and world box (the
 * packer's arithmetic over mesh_boxes[instances[i].mesh], 6 floats a mesh), the top level is
 * refit over the new boxes with header word 3 counting refits, and rebuilt once 64 refits have
 * been made (instance_bvh::place for a moved set), and reflection scene bounds are recomputed.
 * The instances are the scene's, in record order, none singular; the rest of each record stays.
 * rt_scene_move_instances does the same on the device. */
rt_status rt_move_instances_host(rt_layout layout, uint32_t* words, size_t n_words, const rt_instance* instances,
                                 uint32_t n, const float* mesh_boxes, uint32_t n_meshes);
/* The same on an uploaded scene, on the device (records, top-level refit one launch per level,
 * the rebuild after 64 refits, scene bounds), with rt_move_instances_host's words bit for bit:
 * the per-frame instance update of the reference (instance_words + instance_bvh::place,
 * src/instance_bvh.rs:162-275) without a host round trip. Host arrays; it reads the scene's
 * header and, on the first call, the top level's topology, synchronously. */
rt_status rt_scene_move_instances(rt_ctx* ctx, rt_scene* scene, const rt_instance* instances, uint32_t n,
                                  const float* mesh_boxes, uint32_t n_meshes, void* stream);

/* Instance top level alone (instance_bvh.rs:346-366): boxes are 6 floats (lo xyz, hi xyz).
 * Call with out NULL to learn the size. */
rt_status rt_tlas_build(const float* boxes, uint32_t n, int sah, uint32_t* out, size_t* n_words);
rt_status rt_tlas_refit(uint32_t* nodes, size_t n_words, const float* boxes, uint32_t n);
/* rt_tlas_build (SAH, with the median rebuild of a tree too deep for a 48-entry stack, or
 * median) run on the context's device: host boxes in, the same node words out. Synchronous, on a
 * stream of its own; it holds the context's lock while it builds. */
rt_status rt_tlas_build_device(rt_ctx* ctx, const float* boxes, uint32_t n, int sah, uint32_t* out, size_t* n_words);

/* The BLAS's positions (xyz a vertex, as given to rt_blas_build or decoded), 3 * positions floats. */
rt_status rt_blas_positions(const rt_blas* blas, float* out);

/* ---- cooked files: loading cooked scenes (far-field cuts) straight into the engine ----
 * RLB cluster BVH (crates/asset/src/cluster_bvh/codec.rs:4-188, checked as Bvh::validate,
 * crates/asset/src/cluster_bvh.rs:170-333) and RNF near field (crates/asset/src/near_field.rs:
 * 540-660, NearField::validate :106-133). A rejected file returns RT_ERR_LAYOUT and, when err is
 * not NULL, the reference's message in err (at most err_len bytes, NUL-terminated). Sizes follow
 * the NULL-out convention: out NULL -> *n_bytes is the size; too small -> RT_ERR_INVALID_ARG. */
#define RT_RLB_MAX_BYTES 150000000ull /* cluster_bvh::Limits::default */
#define RT_RNF_MAX_BYTES 160000000ull /* near_field::Limits::default */

/* A BLAS as an RLB file, written as the near-field builder writes its cluster BVH
 * (near_field.rs:206-262): one zero-error level over every leaf. */
rt_status rt_blas_encode_rlb(const rt_blas* blas, uint64_t max_bytes, uint8_t* out, size_t* n_bytes, char* err,
                             size_t err_len);
/* cluster_bvh::decode, then level `level`'s root over the file's records (gi_bvh.rs:62-78:
 * Blas::new). The BLAS packs and traces as one built here. */
rt_status rt_rlb_decode(const uint8_t* bytes, size_t n_bytes, uint64_t max_bytes, uint32_t level, rt_blas** out,
                        char* err, size_t err_len);

typedef struct rt_rnf rt_rnf;
typedef struct rt_rnf_settings {
  float lod_error, reach, skip;
  uint32_t bins; /* 0, 8, 16 or 32; a mask is bins * bins / 32 words */
} rt_rnf_settings;
typedef struct rt_rnf_placement {
  uint32_t mesh;
  float transform[16];   /* column-major, the exact bits the masks were cooked under */
  const uint32_t* masks; /* per mesh position: front side then back side, bins^2/32 words each */
  uint64_t n_masks;
} rt_rnf_placement;
rt_status rt_rnf_decode(const uint8_t* bytes, size_t n_bytes, uint64_t max_bytes, rt_rnf** out, char* err,
                        size_t err_len);
rt_status rt_rnf_info(const rt_rnf* field, rt_rnf_settings* settings, uint8_t source[32], uint32_t* n_meshes,
                      uint32_t* n_placements);
/* Mesh `mesh`'s far-field cut as a BLAS (a copy: free it with rt_blas_free). */
rt_status rt_rnf_mesh(const rt_rnf* field, uint32_t mesh, rt_blas** out);
/* Placement k; its masks point into the field and live until rt_rnf_free. */
rt_status rt_rnf_placement_get(const rt_rnf* field, uint32_t k, rt_rnf_placement* out);
rt_status rt_rnf_encode(const rt_rnf_settings* settings, const uint8_t source[32], const rt_blas* const* meshes,
                        uint32_t n_meshes, const rt_rnf_placement* placements, uint32_t n_placements,
                        uint64_t max_bytes, uint8_t* out, size_t* n_bytes, char* err, size_t err_len);
/* GI words for the field's meshes and the given instances (rows and the model as rt_pack_scene
 * takes them, mesh = the field's mesh index): each mesh's placements with masks are appended
 * after the records (gi_bvh.rs:150-227), and an instance whose model has exactly a placement's
 * transform bits gets that placement's mask base in word 23 (gi_bvh.rs:95-104,
 * gi_cache.rs:3225-3250); other instances get 0. */
rt_status rt_rnf_pack_gi(const rt_rnf* field, const rt_instance* instances, uint32_t n_instances, int tlas_mode,
                         uint32_t* out_words, size_t* n_words);
/* A mask-free field as one world-space BLAS (gi_cache.rs:1234-1268): every placement's cut moved
 * by its transform, mirrored windings reversed, built with RT_BUILD_SAH; bases[k] (n_placements
 * entries) is placement k's first position. Traced as one identity instance. */
rt_status rt_rnf_world(const rt_rnf* field, rt_blas** out, uint32_t* bases);
void rt_rnf_free(rt_rnf* field);

#ifdef __cplusplus
}
#endif
#endif /* RT_TRACE_H */
